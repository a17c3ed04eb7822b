"""The CPU oracle against the reference's own code (golden vectors made by
oracle/_ref from the reference sources) and against its known answers."""
import json
import os

import numpy as np
import pytest

import pyoracle as po
from helpers import changes_from_golden, er_graph, oracle_graph


def _run(c, schedule):
    g = po.Graph(int(c["n"][0]))
    assert g.load_edges(c["a"], c["b"]) == po.OK
    assert g.set_colors(c["colors"]) == po.OK
    rc, st = g.apply_batch(changes_from_golden(c), int(c["variant"][0]), schedule, iter_cap=2000)
    return rc, st, g


@pytest.mark.parametrize("schedule,tag", [(po.SERIAL, "serial"), (po.SNAPSHOT, "snapshot")])
def test_oracle_matches_reference_code(golden, schedule, tag):
    bad = []
    for c in golden:
        rc, st, g = _run(c, schedule)
        want_it, want_status = c[f"{tag}_iters"]
        if not (np.array_equal(g.colors(), c[f"{tag}_colors"]) and st.iterations == want_it
                and st.status == want_status):
            bad.append(c["name"])
    assert not bad, f"oracle differs from the reference code on {bad[:10]}"


def test_sample_fixture_known_answers(golden):
    by = {c["name"]: c for c in golden}
    # serial schedule of the reference's own sample run (one thread)
    assert by["sample_hi"]["serial_colors"].tolist() == [2, 2, 1, 1, 0, 0, 2, 2, 3, 1]
    assert by["sample_hb"]["serial_colors"].tolist() == [1, 0, 2, 2, 1, 0, 2, 3, 4, 2]
    for nm in ("sample_hi", "sample_hb"):
        for tag in ("serial", "snapshot"):
            rc, st, g = _run(by[nm], po.SERIAL if tag == "serial" else po.SNAPSHOT)
            assert g.conflicts() == 0


def test_snapshot_is_thread_count_independent():
    n, a, b = er_graph(3000, 12, seed=5)
    rng = np.random.default_rng(3)
    col = rng.integers(0, 6, n).astype(np.int32)
    x = rng.integers(0, n, 4000)
    y = rng.integers(0, n, 4000)
    keep = x != y
    ch = po.as_changes(x[keep], y[keep], rng.integers(0, 2, 4000)[keep])
    outs = []
    for th in (1, 4):
        po.set_threads(th)
        for v in (po.HI, po.HB):
            g = oracle_graph(n, a, b, col)
            rc, st = g.apply_batch(ch, v, po.SNAPSHOT, iter_cap=100000)
            outs.append((th, v, g.colors().tobytes(), st.iterations))
    po.set_threads(0)
    assert outs[0][2:] == outs[2][2:] and outs[1][2:] == outs[3][2:]


@pytest.mark.parametrize("variant", [po.HI, po.HB])
def test_oracle_proper_after_batch_from_proper_start(variant):
    import dyncolor_b200 as dc

    n, a, b = er_graph(5000, 16, seed=2)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ch = es.sample_batch(500, 500, seed=9)
    g = oracle_graph(n, a, b, col)
    assert g.conflicts() == 0
    rc, st = g.apply_batch(ch, variant, po.SNAPSHOT)
    assert rc == po.OK
    assert g.conflicts() == 0


def test_oracle_rejects_bad_lines():
    g = po.Graph(4)
    assert g.load_edges(np.array([0, 1]), np.array([1, 1])) == po.E_INVAL
    assert g.load_edges(np.array([0, 1]), np.array([1, 2])) == po.OK
    g.set_colors(np.zeros(4, np.int32))
    rc, _ = g.apply_batch(po.as_changes([0], [4], [1]), po.HI)
    assert rc == po.E_INVAL
    rc, _ = g.apply_batch(po.as_changes([2], [2], [0]), po.HI)
    assert rc == po.E_INVAL
    # inst outside {0,1} is ignored, even with bad ids (readin_changes)
    rc, _ = g.apply_batch(po.as_changes([7], [7], [5]), po.HI)
    assert rc == po.OK


@pytest.mark.skipif(not po.ref_available(), reason="reference harness not built here")
def test_oracle_matches_reference_code_live():
    rng = np.random.default_rng(77)
    for trial in range(40):
        n = int(rng.integers(2, 50))
        m = int(rng.integers(0, 3 * n))
        a = rng.integers(0, n, m).astype(np.int32)
        b = rng.integers(0, n, m).astype(np.int32)
        keep = a != b
        a, b = a[keep], b[keep]
        col = rng.integers(0, 6, n).astype(np.int32)
        k = int(rng.integers(0, 2 * n))
        x = rng.integers(0, n, k)
        y = rng.integers(0, n, k)
        keep = x != y
        ch = po.as_changes(x[keep], y[keep], rng.integers(0, 2, k)[keep])
        for v in (po.HI, po.HB):
            for sch in (po.SERIAL, po.SNAPSHOT):
                g = oracle_graph(n, a, b, col)
                rc, st = g.apply_batch(ch, v, sch, iter_cap=2000)
                it, status, rcol = po.run_ref(v, sch, a, b, col, ch, iter_cap=2000)
                assert (it, status) == (st.iterations, st.status)
                assert np.array_equal(rcol, g.colors())


def test_checker_generators_match_the_product_generators():
    """The generators compiled into liboracle.so (used by the benchmark's
    reference arm, which must not load libdyncolor.so) give the same graphs,
    colourings and batches as the product's."""
    import dyncolor_b200 as dc

    n = 1 << 12
    a1, b1 = po.gen_dedup(n, *po.gen_rmat(12, 16 * n, seed=3))
    a2, b2 = dc.dedup(n, *dc.rmat(12, 16 * n, seed=3))
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert np.array_equal(po.gen_greedy_color(n, a1, b1), dc.greedy_color(n, a2, b2))
    x1 = po.GenEdgeSet(n, a1, b1).sample_batch(300, 300, mode=po.INS_RMAT, scale=12, seed=5)
    x2 = dc.EdgeSet(n, a2, b2).sample_batch(300, 300, mode=dc.INS_RMAT, scale=12, seed=5)
    assert np.array_equal(x1.view(np.int32), x2.view(np.int32))
    c1 = po.gen_chung_lu(5000, 2.1, 24.0, 250.0, seed=2)
    c2 = dc.chung_lu(5000, 2.1, 24.0, 250.0, seed=2)
    assert np.array_equal(c1[0], c2[0]) and np.array_equal(c1[1], c2[1])


def test_reference_arm_loads_only_checker_code(tmp_path):
    """bench.py --impl reference builds its inputs with the checker's
    generators and runs the reference's own kernel bodies: libdyncolor.so is
    never mapped into that process."""
    import subprocess
    import sys

    if not po.ref_available():
        pytest.skip("reference harness not built")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    probe = tmp_path / "probe.py"
    probe.write_text(
        "import json, runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--scale', '12', '--batch', '2000', "
        "'--steps', '2', '--warmup', '1', '--ref-sample', '200']\n"
        f"sys.path.insert(0, {root!r})\n"
        "import bench\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'dyncolor': 'libdyncolor' in maps, 'oracle': 'liboracle' in maps}))\n")
    r = subprocess.run([sys.executable, str(probe)], capture_output=True, text=True, cwd=root, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert lines[0]["impl"] == "reference" and lines[0]["value"] > 0
    assert lines[1] == {"dyncolor": False, "oracle": True}

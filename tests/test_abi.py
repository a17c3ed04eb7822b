"""C ABI surface and host-side logic that needs no GPU."""
import ctypes
import os
import re

import numpy as np

import dyncolor_b200 as dc
import pyoracle as po
from helpers import er_graph, oracle_graph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(inc, fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(dcg?_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(dc.LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_options_default_and_status_strings():
    opt = dc.Options()
    assert dc.lib().dc_options_default(ctypes.byref(opt)) == dc.OK
    assert opt.variant == dc.HI and opt.iter_cap > 0 and opt.slack > 1 and opt.unit_slots % 128 == 0
    assert dc.status_str(dc.E_ITER_LIMIT) == "iteration cap reached"
    assert ctypes.sizeof(dc.Stats) == 152 and dc.CHANGE_DTYPE.itemsize == 12


def test_generators_deterministic_and_thread_independent():
    a1, b1 = dc.rmat(12, 20000, seed=7)
    a2, b2 = dc.rmat(12, 20000, seed=7)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    a3, _ = dc.rmat(12, 20000, seed=8)
    assert not np.array_equal(a1, a3)
    assert a1.min() >= 0 and a1.max() < 4096
    x, y = dc.dedup(4096, a1, b1)
    assert np.all(x < y)
    keys = x.astype(np.int64) * 4096 + y
    assert np.all(np.diff(keys) > 0)


def test_rmat_skew_and_config1_size():
    # R-MAT(0.57, 0.19, 0.19, 0.05), scale 16, 16 * 2^16 samples -> ~0.91 M edges
    n = 1 << 16
    a, b = dc.rmat(16, 16 * n, seed=1)
    a, b = dc.dedup(n, a, b)
    assert 880_000 < len(a) < 940_000
    deg = np.bincount(np.concatenate([a, b]), minlength=n)
    assert deg[0] > 50 * deg.mean()


def test_greedy_is_id_order_greedy():
    n, a, b = er_graph(4000, 10, seed=3)
    col = dc.greedy_color(n, a, b)
    g = oracle_graph(n, a, b, col)
    assert g.is_greedy_id_order() and g.conflicts() == 0


def test_chung_lu_shape():
    a, b = dc.chung_lu(20000, 2.1, 24, 2000, seed=1)
    a, b = dc.dedup(20000, a, b)
    deg = np.bincount(np.concatenate([a, b]), minlength=20000)
    assert 15 < deg.mean() < 30
    assert deg.max() > 500


def test_edgeset_batches():
    n, a, b = er_graph(2000, 8, seed=4)
    es = dc.EdgeSet(n, a, b)
    m0 = es.size()
    existing = set(zip(a.tolist(), b.tolist()))
    ch = es.sample_batch(100, 150, mode=dc.INS_UNIFORM, seed=3)
    assert len(ch) == 250 and es.size() == m0 + 50
    dels = ch[ch["inst"] == 0]
    ins = ch[ch["inst"] == 1]
    assert all((min(x, y), max(x, y)) in existing for x, y in zip(dels["node1"], dels["node2"]))
    assert all((min(x, y), max(x, y)) not in existing for x, y in zip(ins["node1"], ins["node2"]))
    assert len({(min(x, y), max(x, y)) for x, y in zip(ins["node1"], ins["node2"])}) == 150
    assert np.all(ins["node1"] != ins["node2"])
    ch2 = es.sample_batch(10, 10, mode=dc.INS_RMAT, scale=11, seed=3)
    assert len(ch2) == 20
    ch3 = es.sample_batch(10, 10, mode=dc.INS_DEGREE, seed=3)
    assert len(ch3) == 20


def test_reference_text_formats(tmp_path):
    from dyncolor_b200 import io

    a = np.array([0, 1, 2], np.int32)
    b = np.array([1, 2, 3], np.int32)
    io.write_graph(tmp_path / "g.txt", a, b)
    x, y = io.read_graph(tmp_path / "g.txt")
    assert np.array_equal(a, x) and np.array_equal(b, y)
    io.write_colors(tmp_path / "c.txt", np.array([3, 1, 0, 2], np.int32))
    assert io.read_colors(tmp_path / "c.txt", 4).tolist() == [3, 1, 0, 2]
    ch = dc.as_changes([0, 1], [2, 3], [1, 0])
    io.write_changes(tmp_path / "x.txt", ch)
    assert np.array_equal(io.read_changes(tmp_path / "x.txt"), ch)

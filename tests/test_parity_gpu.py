"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Colours, iteration counts and step statistics must be bit-exact with the
oracle's snapshot schedule; the golden vectors additionally pin both to the
reference's own kernel code run on the CPU."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from helpers import changes_from_golden, er_graph, oracle_graph, rmat_graph, to_dc_changes

pytestmark = pytest.mark.gpu

VARIANTS = [(dc.HI, po.HI), (dc.HB, po.HB)]


def gpu_ctx(variant, n, a, b, colors, **kw):
    ctx = dc.Context(variant=variant, **kw)
    ctx.load_edges(n, a, b)
    ctx.set_colors(colors)
    return ctx


def check_same(ctx, g, st_gpu, st_orc, stats=True, scanned=True):
    gc, oc = ctx.colors(), g.colors()
    if not np.array_equal(gc, oc):
        bad = np.nonzero(gc != oc)[0]
        raise AssertionError(f"{len(bad)} colours differ, first {bad[:8]} gpu {gc[bad[:8]]} oracle {oc[bad[:8]]}")
    assert st_gpu.iterations == st_orc.iterations
    if stats:
        assert st_gpu.seed_targets == st_orc.seed_targets
        assert st_gpu.frontier_total == st_orc.frontier_total
        if scanned:
            assert st_gpu.slots_scanned == st_orc.slots_scanned


def test_golden_vectors_on_gpu(golden):
    bad = []
    for c in golden:
        variant = int(c["variant"][0])
        n = int(c["n"][0])
        ctx = gpu_ctx(variant, n, c["a"], c["b"], c["colors"], iter_cap=2000)
        ch = to_dc_changes(changes_from_golden(c))
        st = ctx.apply_batch(ch, check=False)
        want_it, want_status = c["snapshot_iters"]
        ok = np.array_equal(ctx.colors(), c["snapshot_colors"]) and st.iterations == want_it
        ok = ok and ((st.status == dc.OK) == (want_status == 0))
        if not ok:
            bad.append(c["name"])
        ctx.close()
    assert not bad, f"GPU differs from the reference code (snapshot) on {bad[:10]}"


@pytest.mark.parametrize("variant,ov", VARIANTS)
@pytest.mark.parametrize("unit_slots", [128, 4096])
def test_random_graphs_multi_batch(variant, ov, unit_slots):
    rng = np.random.default_rng(11 + unit_slots)
    for trial in range(6):
        n, a, b = er_graph(int(rng.integers(50, 3000)), float(rng.integers(2, 40)), seed=trial + 1)
        col = rng.integers(0, int(rng.integers(1, 40)), n).astype(np.int32)
        ctx = gpu_ctx(variant, n, a, b, col, unit_slots=unit_slots, iter_cap=100000)
        g = oracle_graph(n, a, b, col)
        for bi in range(3):
            k = int(rng.integers(0, 3 * n))
            x = rng.integers(0, n, k)
            y = rng.integers(0, n, k)
            keep = x != y
            ch = po.as_changes(x[keep], y[keep], rng.integers(0, 2, k)[keep])
            rc, so = g.apply_batch(ch, ov, po.SNAPSHOT, iter_cap=100000)
            sg = ctx.apply_batch(to_dc_changes(ch), check=False)
            assert (sg.status == dc.OK) == (rc == po.OK)
            # random batches repeat pairs, so slot counts differ from the
            # oracle's multiset rows; colours and steps must not
            check_same(ctx, g, sg, so, scanned=False)
        if variant == dc.HB:
            assert np.array_equal(ctx.prop(), g.prop())
        for v in rng.integers(0, n, 20):
            assert np.array_equal(ctx.neighbors(int(v)), g.neighbors(int(v)))
        ctx.close()


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_rmat16_config_batch(variant, ov):
    """R-MAT scale 16, edge factor 16, greedy id-order colouring, one batch
    of 10,000 deletions of existing edges + 10,000 absent insertions."""
    n, a, b = rmat_graph(16, 16, seed=1)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ch = es.sample_batch(10_000, 10_000, mode=dc.INS_UNIFORM, seed=2)
    ctx = gpu_ctx(variant, n, a, b, col)
    g = oracle_graph(n, a, b, col)
    rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
    sg = ctx.apply_batch(to_dc_changes(ch))
    assert rc == po.OK
    check_same(ctx, g, sg, so)
    assert ctx.validate() == 0 and g.conflicts() == 0
    assert sg.edges_inserted == 10_000 and sg.edges_deleted == 10_000
    assert ctx.info()["edges"] == len(a)


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_rmat_batch_sequence(variant, ov):
    n, a, b = rmat_graph(14, 16, seed=3)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ctx = gpu_ctx(variant, n, a, b, col, slack=1.05)
    g = oracle_graph(n, a, b, col)
    for i in range(5):
        ch = es.sample_batch(3000, 3000, mode=dc.INS_RMAT, scale=14, seed=10 + i)
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so)
        assert ctx.validate() == 0
    assert ctx.info()["edges"] == es.size()


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_hub_rows_and_wide_colour_windows(variant, ov):
    """A star whose centre has 5000 leaves coloured 0..4999: deleting the
    edge to the leaf coloured 4500 makes the centre's mex 4500, beyond the
    first 4096-colour window, across many work units."""
    leaves = 5000
    n = leaves + 1
    a = np.zeros(leaves, np.int32)
    b = np.arange(1, n, dtype=np.int32)
    col = np.concatenate([[leaves], np.arange(leaves)]).astype(np.int32)
    ch = po.as_changes([0, 4501, 17], [4501, 4600, 18], [0, 1, 1])
    for us in (128, 4096):
        ctx = gpu_ctx(variant, n, a, b, col, unit_slots=us)
        g = oracle_graph(n, a, b, col)
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so)
        ctx.close()


def test_saturation_beyond_first_window():
    """HI insEdge compares saturation sizes over every colour; colours above
    4096 must count."""
    n = 9000
    rng = np.random.default_rng(5)
    a = rng.integers(0, n, 40000).astype(np.int32)
    b = rng.integers(0, n, 40000).astype(np.int32)
    keep = a != b
    a, b = a[keep], b[keep]
    col = rng.integers(0, 8000, n).astype(np.int32)
    col[:200] = 7  # many equal colours for the insertions
    x = rng.integers(0, 200, 600)
    y = rng.integers(0, 200, 600)
    keep = x != y
    ch = po.as_changes(x[keep], y[keep], np.ones(keep.sum(), np.int32))
    ctx = gpu_ctx(dc.HI, n, a, b, col)
    g = oracle_graph(n, a, b, col)
    rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
    sg = ctx.apply_batch(to_dc_changes(ch))
    check_same(ctx, g, sg, so, scanned=False)


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_edge_cases(variant, ov):
    n, a, b = er_graph(400, 6, seed=9)
    col = dc.greedy_color(n, a, b)
    ctx = gpu_ctx(variant, n, a, b, col)
    g = oracle_graph(n, a, b, col)
    u, v = int(a[0]), int(b[0])
    w = next(x for x in range(n) if x not in (u, v) and x not in set(g.neighbors(u).tolist()))
    batches = [
        po.as_changes([], [], []),                                  # empty
        po.as_changes([u, u, u], [v, v, v], [0, 0, 0]),              # duplicate deletions
        po.as_changes([u, u], [w, w], [1, 1]),                      # duplicate insertions
        po.as_changes([u, u], [w, w], [0, 1]),                      # delete + insert: delete wins
        po.as_changes([u], [v], [1]),                               # re-insert
        po.as_changes([u], [v], [1]),                               # insert existing edge
        po.as_changes([w, 3], [u, 4], [7, 9]),                      # ignored inst values
        po.as_changes(a[:50], b[:50], np.ones(50, np.int32)),       # insertions of existing edges
        po.as_changes(a[:80], b[:80], np.zeros(80, np.int32)),      # deletion only
    ]
    for ch in batches:
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so, scanned=False)
        for x in (u, v, w):
            assert np.array_equal(ctx.neighbors(x), g.neighbors(x))
    if variant == dc.HB:
        assert np.array_equal(ctx.prop(), g.prop())


def test_invalid_batches_leave_state_untouched():
    n, a, b = er_graph(300, 5, seed=2)
    col = dc.greedy_color(n, a, b)
    ctx = gpu_ctx(dc.HI, n, a, b, col)
    before = ctx.colors().copy()
    nb = [ctx.neighbors(x) for x in range(10)]
    for ch in (po.as_changes([0, 1], [1, n], [1, 1]), po.as_changes([5], [5], [0]),
               po.as_changes([-1], [2], [0])):
        with pytest.raises(dc.DcError) as e:
            ctx.apply_batch(to_dc_changes(ch))
        assert e.value.status == dc.E_INVAL
    assert np.array_equal(ctx.colors(), before)
    assert all(np.array_equal(ctx.neighbors(x), nb[x]) for x in range(10))
    with pytest.raises(dc.DcError):
        ctx.set_colors(np.full(n, -1, np.int32))
    with pytest.raises(dc.DcError):
        ctx.load_edges(n, a, b)


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_iteration_cap_matches_oracle_partial_state(variant, ov):
    n, a, b = rmat_graph(12, 16, seed=4)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ch = es.sample_batch(2000, 2000, seed=4)
    for cap in (1, 2, 5):
        ctx = gpu_ctx(variant, n, a, b, col, iter_cap=cap)
        g = oracle_graph(n, a, b, col)
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT, iter_cap=cap)
        sg = ctx.apply_batch(to_dc_changes(ch), check=False)
        assert (rc == po.E_ITER_LIMIT) == (sg.status == dc.E_ITER_LIMIT)
        assert np.array_equal(ctx.colors(), g.colors())
        # the context stays usable after the cap fired
        ch2 = es.sample_batch(10, 10, seed=50 + cap)
        g2rc, so2 = g.apply_batch(ch2, ov, po.SNAPSHOT, iter_cap=cap)
        sg2 = ctx.apply_batch(to_dc_changes(ch2), check=False)
        assert np.array_equal(ctx.colors(), g.colors())
        ctx.close()


def test_pool_growth_and_relocation():
    """Tiny slack and many insertions into a few rows force relocations and
    pool growth with retry; the structure must still equal the oracle's."""
    n, a, b = er_graph(2000, 4, seed=6)
    col = dc.greedy_color(n, a, b)
    ctx = gpu_ctx(dc.HI, n, a, b, col, slack=1.01)
    g = oracle_graph(n, a, b, col)
    rng = np.random.default_rng(1)
    for i in range(4):
        x = rng.integers(0, 20, 20000)
        y = rng.integers(0, n, 20000)
        keep = x != y
        ch = po.as_changes(x[keep], y[keep], (rng.random(keep.sum()) < 0.8).astype(np.int32))
        rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so, scanned=False)
    info = ctx.info()
    assert info["slots_used"] <= info["slots_capacity"]
    for v in range(25):
        assert np.array_equal(ctx.neighbors(v), g.neighbors(v))
    ctx.compact()
    for v in range(25):
        assert np.array_equal(ctx.neighbors(v), g.neighbors(v))
    ch = po.as_changes([0, 1, 2], [100, 101, 102], [1, 1, 0])
    rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
    sg = ctx.apply_batch(to_dc_changes(ch))
    check_same(ctx, g, sg, so, scanned=False)


def test_device_resident_batch_entry_point():
    import torch

    n, a, b = rmat_graph(12, 8, seed=8)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ch = es.sample_batch(500, 500, seed=1)
    ctx = gpu_ctx(dc.HB, n, a, b, col)
    g = oracle_graph(n, a, b, col)
    rc, so = g.apply_batch(ch, po.HB, po.SNAPSHOT)
    d = torch.from_numpy(ch.view(np.int32).reshape(-1, 3).copy()).cuda()
    sg = ctx.apply_batch_device(d.data_ptr(), len(ch))
    check_same(ctx, g, sg, so)


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_cuda_graph_replay_matches_oracle(variant, ov):
    """Batches replayed from a captured CUDA graph: the line count changes
    every batch (read from device memory), the scratch grows (recapture) and
    a tiny slack forces pool growth (direct-path retry)."""
    n, a, b = rmat_graph(12, 8, seed=31)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ctx = gpu_ctx(variant, n, a, b, col, cuda_graph=True, slack=1.01)
    g = oracle_graph(n, a, b, col)
    for i, k in enumerate((50, 600, 10, 3000, 700, 1)):
        ch = es.sample_batch(k // 2, k - k // 2, seed=40 + i)
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so)
    ctx.close()


def test_greedy_initial_colouring_of_the_resident_graph():
    n, a, b = rmat_graph(12, seed=4)
    ctx = dc.Context(variant=dc.HI, unit_slots=256)
    ctx.load_edges(n, a, b)
    ctx.init_greedy_colors()
    want = dc.greedy_color(n, a, b)
    assert np.array_equal(ctx.colors(), want)
    assert ctx.validate() == 0
    # after a batch the colouring follows the current edge set
    es = dc.EdgeSet(n, a, b)
    ch = es.sample_batch(3000, 3000, seed=5)
    ctx.apply_batch(ch)
    rows = [ctx.neighbors(v) for v in range(n)]
    x = np.concatenate([np.full(len(r), v, np.int32) for v, r in enumerate(rows)])
    y = np.concatenate(rows).astype(np.int32)
    keep = x < y
    ctx.init_greedy_colors()
    assert np.array_equal(ctx.colors(), dc.greedy_color(n, x[keep], y[keep]))
    assert ctx.validate() == 0
    ctx.close()


@pytest.mark.parametrize("variant,ov", VARIANTS)
@pytest.mark.parametrize("min_live,unit_slots", [(64, 128), (256, 2048), (-1, 2048), (4, 128)])
def test_heavy_row_index_matches_oracle(variant, ov, min_live, unit_slots):
    """The per-batch index of heavy rows (HI: neighbours ordered by colour
    plus change lists; HB: prior neighbours first) with many rows indexed,
    rows split over many units, and the index off: colours, iterations,
    frontier sizes and covered entries stay those of the oracle, while the
    entries actually read drop when the index is on.  From 4 live slots the
    rows' copies outgrow the copy buffer (a quarter of the pool's slots for
    HI, half for HB), so the shortest rows lose their index and are
    scanned."""
    n, a, b = rmat_graph(14, 16, seed=5)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    ctx = gpu_ctx(variant, n, a, b, col, unit_slots=unit_slots, heavy_min_live=min_live)
    g = oracle_graph(n, a, b, col)
    read = scanned = 0
    for i in range(4):
        ch = es.sample_batch(4000, 4000, mode=dc.INS_RMAT, scale=14, seed=40 + i)
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        check_same(ctx, g, sg, so)
        read += sg.slots_read
        scanned += sg.slots_scanned
    assert ctx.validate() == 0
    if min_live > 0:
        assert read < scanned
    elif variant == dc.HI:
        assert read == scanned
    else:
        # HB pulls the marks of a dense frontier: it may read fewer entries
        # than the rule covers even without the index
        assert read <= scanned
    ctx.close()

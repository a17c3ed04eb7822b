"""Resident pool: graphs spilled to pinned host memory and reloaded, several
graphs' batches in one launch; every graph ends exactly as when its batches
are applied alone and in order (colours and loop iterations), checked
against the CPU oracle."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from dyncolor_b200.pool import ResidentPool
from helpers import oracle_graph, to_oracle_changes

pytestmark = pytest.mark.gpu


def make_workload(count, seed, rounds=4):
    rng = np.random.default_rng(seed)
    graphs, colors, seqs = [], [], []
    for i in range(count):
        n = int(rng.integers(300, 3000))
        m = int(n * float(rng.uniform(4, 16)) / 2)
        if i % 2 == 0:
            a, b = dc.rmat(int(np.ceil(np.log2(n))), m, seed=seed * 100 + i, n=n)
        else:
            a, b = dc.uniform_pairs(n, m, seed=seed * 100 + i)
        a, b = dc.dedup(n, a, b)
        graphs.append((n, a, b))
        colors.append(dc.greedy_color(n, a, b) if i % 3 else rng.integers(0, 6, n).astype(np.int32))
        es = dc.EdgeSet(n, a, b)
        seq = []
        for r in range(rounds):
            k = int(rng.integers(1, max(4, m // 3)))
            kd = min(k // 2, es.size())
            seq.append(es.sample_batch(kd, k - kd, seed=seed * 1000 + i * 10 + r))
        seqs.append(seq)
    return graphs, colors, seqs


def oracle_runs(graphs, colors, seqs, ov):
    """Per graph: the colours after all its batches and each batch's iterations."""
    out = []
    for (n, a, b), c, seq in zip(graphs, colors, seqs):
        o = oracle_graph(n, a, b, c)
        its = []
        for ch in seq:
            rc, so = o.apply_batch(to_oracle_changes(ch), ov, po.SNAPSHOT)
            assert rc == po.OK
            its.append(so.iterations)
        out.append((o.colors(), its))
    return out


@pytest.mark.parametrize("variant,ov", [(dc.HI, po.HI), (dc.HB, po.HB)])
@pytest.mark.parametrize("heavy_min_live", [-1, 64])
def test_pool_spill_reload_and_shared_launches_match_alone(variant, ov, heavy_min_live):
    """With the heavy-row index off, and on from 64 live slots (each launch
    then indexes the rows of its own graphs only, wherever the pool placed
    them, after other graphs used and left those vertex ids)."""
    graphs, colors, seqs = make_workload(10, seed=3)
    want = oracle_runs(graphs, colors, seqs, ov)
    nmax = max(n for n, _, _ in graphs)
    # room for about three graphs: every launch below forces evictions
    slots = int(3.2 * max(2 * len(a) for _, a, _ in graphs) * 1.25) + 64 * nmax
    pool = ResidentPool(variant=variant, vertex_capacity=3 * nmax, pool_slots=slots, max_graphs=16,
                        unit_slots=256, stage_slots=4096, heavy_min_live=heavy_min_live)
    ids = [pool.add_graph(n, a, b, c) for (n, a, b), c in zip(graphs, colors)]
    assert ids == list(range(len(graphs)))
    info = pool.info()
    assert info["spills"] > 0 and info["resident"] < len(graphs)
    rng = np.random.default_rng(11)
    nxt = [0] * len(graphs)
    its = [[] for _ in graphs]
    restored = 0
    while any(nxt[g] < len(seqs[g]) for g in range(len(graphs))):
        pending = [g for g in range(len(graphs)) if nxt[g] < len(seqs[g])]
        take = rng.choice(pending, size=min(len(pending), int(rng.integers(1, 3))), replace=False)
        st, it, rs = pool.apply([(int(g), seqs[g][nxt[g]]) for g in take])
        restored += int(rs.sum())
        for j, g in enumerate(take):
            its[g].append(int(it[j]))
            nxt[g] += 1
        if rng.random() < 0.3:
            pool.spill(int(rng.integers(0, len(graphs))))  # explicit spill, resident or not
    for g, (cw, iw) in enumerate(want):
        assert np.array_equal(pool.colors(g), cw), f"graph {g}: colours differ from the oracle"
        assert its[g] == iw, f"graph {g}: iterations {its[g]}, oracle {iw}"
    info = pool.info()
    assert info["restores"] > 0 and restored > 0
    assert info["pool_slots_used"] <= info["pool_slots"]
    pool.close()


def test_pool_rejects_bad_requests_without_changing_state():
    graphs, colors, seqs = make_workload(3, seed=4, rounds=1)
    pool = ResidentPool(vertex_capacity=10_000, pool_slots=1 << 20, max_graphs=4)
    for (n, a, b), c in zip(graphs, colors):
        pool.add_graph(n, a, b, c)
    before = [pool.colors(g) for g in range(3)]
    n0 = graphs[0][0]
    bad = dc.as_changes([0], [n0], [1])  # id outside graph 0
    with pytest.raises(dc.DcError) as e:
        pool.apply([(1, seqs[1][0]), (0, bad)])
    assert e.value.status == dc.E_INVAL
    with pytest.raises(dc.DcError) as e:
        pool.apply([(1, seqs[1][0]), (1, seqs[1][0])])  # two batches for one graph
    assert e.value.status == dc.E_INVAL
    with pytest.raises(dc.DcError) as e:
        pool.apply([(7, seqs[1][0])])
    assert e.value.status == dc.E_INVAL
    for g in range(3):
        assert np.array_equal(pool.colors(g), before[g])
    # an empty launch and an empty batch are no-ops
    st, it, _ = pool.apply([])
    st, it, _ = pool.apply([(2, np.empty(0, dtype=dc.CHANGE_DTYPE))])
    assert it[0] == 0 and np.array_equal(pool.colors(2), before[2])
    # a graph larger than the budget is refused
    n, a, b = graphs[0]
    small = ResidentPool(vertex_capacity=n - 1, pool_slots=1 << 16, max_graphs=2)
    with pytest.raises(dc.DcError) as e:
        small.add_graph(n, a, b, colors[0])
    assert e.value.status == dc.E_NOMEM
    small.close()
    pool.close()


def test_pool_cuda_graph_and_rows_growing_past_the_budget():
    # inserts grow rows after a reload; the pool compacts and evicts to fit
    graphs, colors, seqs = make_workload(6, seed=8, rounds=3)
    want = oracle_runs(graphs, colors, seqs, po.HI)
    nmax = max(n for n, _, _ in graphs)
    slots = int(2.5 * max(2 * len(a) for _, a, _ in graphs) * 1.25) + 32 * nmax
    pool = ResidentPool(vertex_capacity=2 * nmax + 16, pool_slots=slots, max_graphs=8, cuda_graph=True)
    for (n, a, b), c in zip(graphs, colors):
        pool.add_graph(n, a, b, c)
    its = [[] for _ in graphs]
    for r in range(3):
        for g in range(len(graphs)):
            st, it, _ = pool.apply([(g, seqs[g][r])])
            its[g].append(int(it[0]))
    for g, (cw, iw) in enumerate(want):
        assert np.array_equal(pool.colors(g), cw)
        assert its[g] == iw
    pool.close()


def test_pool_grows_past_budget_only_for_one_launch_and_shrinks_back():
    # one graph whose batch triples its edges cannot fit the budget: the pool
    # grows up to its hard limit for that launch, then returns to the budget
    n = 2000
    a, b = dc.uniform_pairs(n, 4000, seed=5)
    a, b = dc.dedup(n, a, b)
    col = dc.greedy_color(n, a, b)
    es = dc.EdgeSet(n, a, b)
    big = es.sample_batch(100, 12000, seed=9)
    small_n = 500
    sa, sb = dc.uniform_pairs(small_n, 1000, seed=6)
    sa, sb = dc.dedup(small_n, sa, sb)
    scol = dc.greedy_color(small_n, sa, sb)
    budget = int(2.5 * len(a)) + 8 * n + int(2.5 * len(sa)) + 8 * small_n
    o = oracle_graph(n, a, b, col)
    rc, so = o.apply_batch(to_oracle_changes(big), po.HI, po.SNAPSHOT)
    assert rc == po.OK
    # a hard limit equal to the budget: the launch fails and changes nothing
    tight = ResidentPool(vertex_capacity=4 * n, pool_slots=budget, pool_slots_max=budget, max_graphs=4)
    g0 = tight.add_graph(n, a, b, col)
    with pytest.raises(dc.DcError) as e:
        tight.apply([(g0, big)])
    assert e.value.status == dc.E_NOMEM
    assert np.array_equal(tight.colors(g0), col)
    tight.close()
    pool = ResidentPool(vertex_capacity=4 * n, pool_slots=budget, pool_slots_max=8 * budget, max_graphs=4)
    g0 = pool.add_graph(n, a, b, col)
    g1 = pool.add_graph(small_n, sa, sb, scol)
    st, it, _ = pool.apply([(g0, big)])
    assert np.array_equal(pool.colors(g0), o.colors()) and it[0] == so.iterations
    info = pool.info()
    assert info["overbudget"] > 0 and info["pool_slots"] > info["pool_slots_budget"]
    assert not pool.graph_size(g1)[2]  # evicted before the pool grew
    # the big graph spilled: the small one comes back and the pool shrinks to its budget
    pool.spill(g0)
    st, it, _ = pool.apply([(g1, np.empty(0, dtype=dc.CHANGE_DTYPE))])
    info = pool.info()
    assert info["pool_slots"] == info["pool_slots_budget"]
    assert np.array_equal(pool.colors(g1), scol)
    assert np.array_equal(pool.colors(g0), o.colors())
    pool.close()


@pytest.mark.parametrize("variant,ov", [(dc.HI, po.HI), (dc.HB, po.HB)])
def test_lanes_serve_overlapping_requests_like_each_graph_alone(variant, ov):
    """Requests that arrive while other lanes' launches run: three pools side
    by side (each with a third of the persistent CTAs, its own stream and a
    host thread), continuous batching in each.  Every graph ends with the
    colours, and every request with the iteration count, of applying the
    graph's batches alone and in order."""
    import torch

    from dyncolor_b200.serve import LanedServer, Request, assign_lanes

    graphs, colors, seqs = make_workload(12, seed=8, rounds=3)
    want = oracle_runs(graphs, colors, seqs, ov)
    sizes = [n for n, _, _ in graphs]
    which = assign_lanes(sizes, 3)
    ctas = max(1, 2 * torch.cuda.get_device_properties(0).multi_processor_count // 3)
    lanes = []
    for j in range(3):
        gl = [g for g in range(len(graphs)) if which[g] == j]
        nmax = max(sizes[g] for g in gl)
        slots = sum(int(2.5 * len(graphs[g][1])) + 8 * sizes[g] for g in gl) + 4096
        pool = ResidentPool(variant=variant, vertex_capacity=2 * sum(sizes[g] for g in gl) + nmax, pool_slots=slots,
                            max_graphs=len(gl) + 1, grid_ctas=ctas, cuda_graph=True)
        for g in gl:
            n, a, b = graphs[g]
            pool.add_graph(n, a, b, colors[g])
        lanes.append((pool, {g: i for i, g in enumerate(gl)}, 2 * sum(sizes[g] for g in gl) + nmax, slots))
    # all requests arrive at once, graph by graph round-robin, in batch order
    reqs, rid = [], 0
    for r in range(3):
        for g in range(len(graphs)):
            reqs.append(Request(rid, g, seqs[g][r], 1e-4 * rid))
            rid += 1
    st = LanedServer(lanes).run(reqs)
    assert st.lines == sum(len(x) for s_ in seqs for x in s_)
    for g in range(len(graphs)):
        pool, gmap, _, _ = lanes[which[g]]
        assert np.array_equal(pool.colors(gmap[g]), want[g][0]), f"graph {g}"
        its = [r.iterations for r in sorted((r for r in reqs if r.graph == g), key=lambda r: r.rid)]
        assert its == want[g][1], f"graph {g}"
    for pool, _, _, _ in lanes:
        pool.close()

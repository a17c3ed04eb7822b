"""Batched mode: every graph of a union ends exactly as when recoloured alone
(colours and loop iterations), checked against separate GPU runs and the
CPU oracle."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from dyncolor_b200.batched import BatchedContext
from helpers import oracle_graph, to_oracle_changes

pytestmark = pytest.mark.gpu


def make_graphs(count, seed, nmin=200, nmax=6000):
    rng = np.random.default_rng(seed)
    graphs, colors, batches = [], [], []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        deg = float(rng.uniform(4, 24))
        m = int(n * deg / 2)
        if i % 2 == 0:
            scale = max(1, int(np.ceil(np.log2(n))))
            a, b = dc.rmat(scale, m, seed=seed * 1000 + i, n=n)
        else:
            a, b = dc.uniform_pairs(n, m, seed=seed * 1000 + i)
        a, b = dc.dedup(n, a, b)
        graphs.append((n, a, b))
        if i % 3 == 0:
            colors.append(rng.integers(0, 8, n).astype(np.int32))  # arbitrary start
        else:
            colors.append(dc.greedy_color(n, a, b))
        k = int(np.exp(rng.uniform(np.log(4), np.log(max(8, m // 4)))))
        es = dc.EdgeSet(n, a, b)
        kd = min(k // 2, len(a))
        batches.append(es.sample_batch(kd, k - kd, seed=seed * 7 + i))
    return graphs, colors, batches


@pytest.mark.parametrize("variant,ov", [(dc.HI, po.HI), (dc.HB, po.HB)])
def test_batched_equals_separate_runs(variant, ov):
    graphs, colors, batches = make_graphs(40, seed=5)
    bc = BatchedContext(variant=variant, unit_slots=256)
    bc.load(graphs)
    bc.set_colors(colors)
    st = bc.apply(batches)
    got = bc.colors()
    its = bc.iterations()
    assert st.iterations == its.max()
    for g, ((n, a, b), col, ch) in enumerate(zip(graphs, colors, batches)):
        o = oracle_graph(n, a, b, col)
        rc, so = o.apply_batch(to_oracle_changes(ch), ov, po.SNAPSHOT)
        assert np.array_equal(got[g], o.colors()), f"graph {g}: colours differ from the oracle"
        assert its[g] == so.iterations, f"graph {g}: {its[g]} iterations, oracle {so.iterations}"
    # a few graphs alone on the GPU as well
    for g in (0, 1, 7):
        n, a, b = graphs[g]
        ctx = dc.Context(variant=variant)
        ctx.load_edges(n, a, b)
        ctx.set_colors(colors[g])
        s1 = ctx.apply_batch(batches[g])
        assert np.array_equal(ctx.colors(), got[g])
        assert s1.iterations == its[g]
        ctx.close()
    bc.close()


@pytest.mark.parametrize("variant,ov", [(dc.HI, po.HI), (dc.HB, po.HB)])
def test_batched_sequence_of_batches(variant, ov):
    graphs, colors, batches = make_graphs(12, seed=9)
    bc = BatchedContext(variant=variant)
    bc.load(graphs)
    bc.set_colors(colors)
    orc = [oracle_graph(n, a, b, c) for (n, a, b), c in zip(graphs, colors)]
    sets = [dc.EdgeSet(n, a, b) for n, a, b in graphs]
    for rnd in range(3):
        bat = []
        for g, ((n, a, b), es) in enumerate(zip(graphs, sets)):
            if (g + rnd) % 4 == 0:
                bat.append(np.empty(0, dtype=dc.CHANGE_DTYPE))  # graph without a batch this round
            else:
                bat.append(es.sample_batch(min(20, len(a) // 4), 20, seed=100 * rnd + g))
        bc.apply(bat)
        got = bc.colors()
        its = bc.iterations()
        for g, o in enumerate(orc):
            rc, so = o.apply_batch(to_oracle_changes(bat[g]), ov, po.SNAPSHOT)
            assert np.array_equal(got[g], o.colors())
            assert its[g] == so.iterations


def test_partition_rejects_cross_edges_and_lines():
    ctx = dc.Context()
    ctx.load_edges(6, np.array([0, 3, 2], np.int32), np.array([1, 4, 3], np.int32))
    with pytest.raises(dc.DcError):
        ctx.set_partition(np.array([0, 3, 6], np.int32))  # edge 2-3 joins the graphs
    ctx.close()
    ctx = dc.Context()
    ctx.load_edges(6, np.array([0, 3], np.int32), np.array([1, 4], np.int32))
    ctx.set_partition(np.array([0, 3, 6], np.int32))
    ctx.set_colors(np.zeros(6, np.int32))
    with pytest.raises(dc.DcError) as e:
        ctx.apply_batch(dc.as_changes([1], [5], [1]))
    assert e.value.status == dc.E_INVAL
    ctx.close()

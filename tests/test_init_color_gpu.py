"""Initial colouring on the device (dc_colors_init): the greedy lowest-free
colouring in vertex-id order or largest-degree-first order, computed as a
Jones-Plassmann schedule.  Colours must equal the sequential greedy pass in
the same order, computed on the host (dcg_greedy_color for the id order, the
oracle's greedy-in-order for LDF); the colourings are proper."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from helpers import oracle_graph, rmat_graph, to_dc_changes

pytestmark = pytest.mark.gpu


def _ldf_order(deg):
    n = len(deg)
    return np.lexsort((np.arange(n), -np.asarray(deg, np.int64))).astype(np.int32)


@pytest.mark.parametrize("unit_slots", [128, 2048])
def test_id_and_ldf_order_on_rmat(unit_slots):
    n, a, b = rmat_graph(18, 16, seed=2)
    ctx = dc.Context(unit_slots=unit_slots)
    ctx.load_edges(n, a, b)
    ctx.init_colors(dc.ORDER_ID)
    want = dc.greedy_color(n, a, b)
    assert np.array_equal(ctx.colors(), want)
    assert ctx.validate() == 0
    g = oracle_graph(n, a, b, np.zeros(n, np.int32))
    deg = np.array([g.live_degree(v) for v in range(n)])
    assert g.greedy_in_order(_ldf_order(deg)) == po.OK
    ctx.init_colors(dc.ORDER_LDF)
    got = ctx.colors()
    assert np.array_equal(got, g.colors())
    assert ctx.validate() == 0 and g.conflicts() == 0
    ctx.close()


def test_ldf_reseed_after_batches_and_on_hubs():
    """After update batches (rows with tombstones, relocated rows) and on a
    Chung-Lu graph whose hubs span many work units."""
    n = 1 << 18
    a, b = dc.chung_lu(n, 2.1, 24.0, n / 20.0, seed=5)
    a, b = dc.dedup(n, a, b)
    col = dc.greedy_color(n, a, b)
    ctx = dc.Context(variant=dc.HI, unit_slots=256)
    ctx.load_edges(n, a, b)
    ctx.set_colors(col)
    g = oracle_graph(n, a, b, col)
    es = dc.EdgeSet(n, a, b)
    for i in range(2):
        ch = es.sample_batch(10_000, 20_000, mode=dc.INS_DEGREE, seed=60 + i)
        rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
        ctx.apply_batch(to_dc_changes(ch))
    deg = np.array([g.live_degree(v) for v in range(n)])
    assert deg.max() > 5000
    ctx.init_colors(dc.ORDER_LDF)
    assert g.greedy_in_order(_ldf_order(deg)) == po.OK
    assert np.array_equal(ctx.colors(), g.colors())
    ctx.init_colors(dc.ORDER_ID)
    assert g.greedy_in_order(np.arange(n, dtype=np.int32)) == po.OK
    assert np.array_equal(ctx.colors(), g.colors())
    assert ctx.validate() == 0
    # the re-seeded colouring is a valid start for further batches
    ch = es.sample_batch(5_000, 5_000, mode=dc.INS_DEGREE, seed=99)
    rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
    sg = ctx.apply_batch(to_dc_changes(ch))
    assert np.array_equal(ctx.colors(), g.colors()) and sg.iterations == so.iterations
    ctx.close()


def test_empty_and_edgeless_graphs():
    ctx = dc.Context()
    ctx.load_edges(5, np.empty(0, np.int32), np.empty(0, np.int32))
    ctx.init_colors(dc.ORDER_LDF)
    assert np.array_equal(ctx.colors(), np.zeros(5, np.int32))
    ctx.close()
    with pytest.raises(dc.DcError) as e:
        c2 = dc.Context()
        c2.load_edges(3, np.array([0], np.int32), np.array([1], np.int32))
        c2.init_colors(7)
    assert e.value.status == dc.E_INVAL

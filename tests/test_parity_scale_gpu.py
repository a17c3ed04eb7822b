"""Bit-exact parity with the oracle at the sizes the benchmarks run.

The headline workload (R-MAT scale 24, 1 M-line batches) runs hundreds of
loop iterations over hundreds of colours with the heavy-row index on; the
skewed workload (Chung-Lu, exponent 2.1) has hub rows of tens of thousands
of neighbours whose masks span several 64-bit words.  These tests run the
same generators and batch rules at scales the oracle finishes in seconds,
three batches in sequence, and compare colours, iteration counts, seeding
targets, frontier sizes and covered adjacency entries with the oracle's
snapshot schedule after every batch.

Oracle rules followed: HI/gpuFunctions_undir.cuh:147-284 (HI seeding and
loop), HB/gpuFunctions_undir.cuh:222-314 (HB), HI/Color_main.cu:176-202."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from helpers import oracle_graph, rmat_graph, to_dc_changes

pytestmark = pytest.mark.gpu

VARIANTS = [(dc.HI, po.HI), (dc.HB, po.HB)]


def _run_sequence(variant, ov, n, a, b, batches, **kw):
    col = dc.greedy_color(n, a, b)
    ctx = dc.Context(variant=variant, **kw)
    ctx.load_edges(n, a, b)
    ctx.set_colors(col)
    g = oracle_graph(n, a, b, col)
    read = scanned = 0
    its = []
    for ch in batches:
        rc, so = g.apply_batch(ch, ov, po.SNAPSHOT)
        sg = ctx.apply_batch(to_dc_changes(ch))
        assert rc == po.OK
        gc, oc = ctx.colors(), g.colors()
        if not np.array_equal(gc, oc):
            bad = np.nonzero(gc != oc)[0]
            raise AssertionError(f"{len(bad)} colours differ, first {bad[:8]}")
        assert sg.iterations == so.iterations
        assert sg.seed_targets == so.seed_targets
        assert sg.frontier_total == so.frontier_total
        assert sg.slots_scanned == so.slots_scanned
        assert int(gc.max()) == so.max_color  # same colour count
        read += sg.slots_read
        scanned += sg.slots_scanned
        its.append(sg.iterations)
    assert ctx.validate() == 0 and g.conflicts() == 0
    ctx.close()
    return read, scanned, its, int(col.max()) + 1


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_rmat20_config2_mix_with_heavy_row_index(variant, ov):
    """R-MAT scale 20, edge factor 16, greedy colouring (208 colours), three
    batches of 100,000 lines (half deletions of existing edges, half
    insertions of absent R-MAT pairs): a batch of at least n/32 lines, so the
    heavy-row index is built and used at its default row threshold."""
    scale = 20
    n, a, b = rmat_graph(scale, 16, seed=1)
    es = dc.EdgeSet(n, a, b)
    batches = [es.sample_batch(50_000, 50_000, mode=dc.INS_RMAT, scale=scale, seed=100 + i) for i in range(3)]
    assert len(batches[0]) * 32 >= n
    read, scanned, its, colors0 = _run_sequence(variant, ov, n, a, b, batches)
    assert colors0 > 128  # masks of three or more 64-bit words
    assert min(its) > 100
    # rows were indexed: fewer entries read than the rules cover
    assert read < scanned


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_chung_lu_hubs_degree_preferential_batches(variant, ov):
    """Chung-Lu graph, exponent 2.1, 2^20 vertices, average degree 24, hub
    degrees above 20,000; three batches of 100,000 lines, 70% insertions
    with one endpoint drawn by degree (so hub rows take most of the
    conflicts), 30% deletions of existing edges."""
    n = 1 << 20
    a, b = dc.chung_lu(n, 2.1, 24.0, n / 20.0, seed=3)
    a, b = dc.dedup(n, a, b)
    deg = np.bincount(a, minlength=n) + np.bincount(b, minlength=n)
    assert deg.max() >= 20_000
    es = dc.EdgeSet(n, a, b)
    batches = [es.sample_batch(30_000, 70_000, mode=dc.INS_DEGREE, seed=200 + i) for i in range(3)]
    read, scanned, its, colors0 = _run_sequence(variant, ov, n, a, b, batches)
    assert colors0 > 128
    assert read <= scanned


@pytest.mark.parametrize("variant,ov", VARIANTS)
def test_rmat18_small_units_many_indexed_rows(variant, ov):
    """R-MAT scale 18 with 128-slot work units and rows indexed from 256
    live slots: hub rows split over hundreds of units, thousands of indexed
    rows, change lists appended every iteration."""
    scale = 18
    n, a, b = rmat_graph(scale, 16, seed=7)
    es = dc.EdgeSet(n, a, b)
    batches = [es.sample_batch(20_000, 20_000, mode=dc.INS_RMAT, scale=scale, seed=300 + i) for i in range(3)]
    read, scanned, its, _ = _run_sequence(variant, ov, n, a, b, batches, unit_slots=128, heavy_min_live=256)
    assert read < scanned

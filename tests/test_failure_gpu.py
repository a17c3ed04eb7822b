"""Failure detection on the device without a GPU fault.

Every grid-barrier wait of the persistent kernels is bounded
(dc_options.barrier_timeout_ms).  Here one warp is given a long serial job
(the mex of a 100,000-leaf star centre whose free colour lies 22 colour
windows up, tens of milliseconds of work), so every other CTA waits at the
next barrier far longer than a 1 ms limit.  The waits run out, the launch
ends with DC_E_TIMEOUT, the context refuses further work with DC_E_STATE,
and a fresh context on the same device recolours the same batch exactly as
the oracle does.  Nothing here faults, traps or hangs the GPU: the slow warp
finishes its bounded job and leaves at its next barrier like the others."""
import numpy as np
import pytest

import dyncolor_b200 as dc
import pyoracle as po
from helpers import oracle_graph, to_dc_changes

pytestmark = pytest.mark.gpu


def _star(leaves):
    n = leaves + 1
    a = np.zeros(leaves, np.int32)
    b = np.arange(1, n, dtype=np.int32)
    col = np.concatenate([[leaves], np.arange(leaves)]).astype(np.int32)
    return n, a, b, col


def test_barrier_wait_runs_out_and_context_refuses_work():
    n, a, b, col = _star(100_000)
    # deleting the edge to the leaf coloured 90,000 makes it the centre's mex
    leaf = 90_000 + 1
    ch = po.as_changes([0], [leaf], [0])
    ctx = dc.Context(variant=dc.HI, barrier_timeout_ms=1)
    ctx.load_edges(n, a, b)
    ctx.set_colors(col)
    st = ctx.apply_batch(to_dc_changes(ch), check=False)
    assert st.status == dc.E_TIMEOUT, ctx.last_error()
    for call in (lambda: ctx.apply_batch(to_dc_changes(ch)), ctx.colors, ctx.validate):
        with pytest.raises(dc.DcError) as e:
            call()
        assert e.value.status == dc.E_STATE
    ctx.close()
    # a fresh context on the same device works
    fresh = dc.Context(variant=dc.HI)
    fresh.load_edges(n, a, b)
    fresh.set_colors(col)
    sg = fresh.apply_batch(to_dc_changes(ch))
    g = oracle_graph(n, a, b, col)
    rc, so = g.apply_batch(ch, po.HI, po.SNAPSHOT)
    assert rc == po.OK
    got = fresh.colors()
    assert np.array_equal(got, g.colors())
    assert got[0] == 90_000 and sg.iterations == so.iterations
    assert fresh.validate() == 0
    fresh.close()

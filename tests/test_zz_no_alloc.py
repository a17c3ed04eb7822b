"""dc_validate_csr_noalloc: the colouring check for callers that cannot let
the library allocate device memory (its scratch is a fixed array inside
libdyncolor.so).  Checked against dc_validate on the same graph and
colouring, on two calls in a row, so a result left in the shared scratch by
the first call would show up in the second."""
import ctypes as C

import numpy as np
import pytest

import dyncolor_b200 as dc
from helpers import rmat_graph

pytestmark = pytest.mark.gpu


def _bind():
    L = dc.lib()
    f = L.dc_validate_csr_noalloc
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    return f


def _csr(n, a, b):
    """Plain CSR of the undirected edge list, in host arrays."""
    src = np.concatenate([a, b]).astype(np.int64)
    dst = np.concatenate([b, a]).astype(np.int32)
    order = np.argsort(src, kind="stable")
    adj = dst[order]
    deg = np.bincount(src, minlength=n).astype(np.int32)
    off = np.zeros(n, np.int64)
    off[1:] = np.cumsum(deg)[:-1]
    return off, deg, adj


def _noalloc(f, torch, n, off, deg, adj, colors):
    d_off = torch.from_numpy(off).cuda()
    d_deg = torch.from_numpy(deg).cuda()
    d_adj = torch.from_numpy(adj).cuda()
    d_col = torch.from_numpy(colors.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    conf, verts, cmax = C.c_int64(-1), C.c_int64(-1), C.c_int32(-1)
    rc = f(n, d_off.data_ptr(), d_deg.data_ptr(), d_adj.data_ptr(), d_col.data_ptr(), None,
           C.byref(conf), C.byref(verts), C.byref(cmax))
    return rc, conf.value, verts.value, cmax.value


def test_noalloc_validate_matches_dc_validate_twice():
    import torch

    f = _bind()
    n, a, b = rmat_graph(13, 8, seed=21)
    off, deg, adj = _csr(n, a, b)
    rng = np.random.default_rng(4)
    colorings = [rng.integers(0, 12, n).astype(np.int32), dc.greedy_color(n, a, b)]
    ctx = dc.Context(variant=dc.HI)
    ctx.load_edges(n, a, b)
    for colors in colorings:  # two calls in a row
        ctx.set_colors(colors)
        want = ctx.validate()
        rc, conf, verts, cmax = _noalloc(f, torch, n, off, deg, adj, colors)
        assert rc == dc.OK
        assert conf == want
        mono = colors[a] == colors[b]
        assert verts == len(np.unique(np.concatenate([a[mono], b[mono]])))
        assert cmax == int(colors.max())
    assert conf == 0  # the greedy colouring is proper
    ctx.close()


def test_noalloc_validate_rejects_bad_sizes():
    f = _bind()
    conf = C.c_int64()
    assert f((1 << 24) + 1, None, None, None, None, None, C.byref(conf), None, None) == dc.E_INVAL
    assert f(-1, None, None, None, None, None, C.byref(conf), None, None) == dc.E_INVAL


def test_noalloc_validate_skips_deleted_entries_and_flags_bad_input():
    """Deleted (-1) entries are skipped; a negative colour or a neighbour id
    outside [0, n) gives E_INVAL; the optional outputs may be NULL.  Every
    case stays inside the caller's arrays (the kernel checks an id before it
    reads that neighbour's colour)."""
    import torch

    f = _bind()
    n, a, b = rmat_graph(11, 8, seed=22)
    off, deg, adj = _csr(n, a, b)
    rng = np.random.default_rng(9)
    colors = rng.integers(0, 6, n).astype(np.int32)
    # delete about a third of the entries in place (both directions of an edge
    # need not go together: each live directed entry u > v counts once)
    adj_del = adj.copy()
    adj_del[rng.random(len(adj)) < 0.33] = -1
    src = np.repeat(np.arange(n), deg)
    live = adj_del >= 0
    u, v = adj_del[live], src[live]
    want = int(np.count_nonzero((u > v) & (colors[u] == colors[v])))
    rc, conf, verts, cmax = _noalloc(f, torch, n, off, deg, adj_del, colors)
    assert rc == dc.OK and conf == want and cmax == int(colors.max())
    mono = (u > v) & (colors[u] == colors[v])
    assert verts == len(np.unique(np.concatenate([u[mono], v[mono]])))
    # NULL optional outputs
    d = [torch.from_numpy(x).cuda() for x in (off, deg, adj_del, colors)]
    torch.cuda.synchronize()
    conf2 = C.c_int64(-1)
    assert f(n, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), None,
             C.byref(conf2), None, None) == dc.OK
    assert conf2.value == want
    # a negative colour
    bad_col = colors.copy()
    bad_col[7] = -1
    assert _noalloc(f, torch, n, off, deg, adj, bad_col)[0] == dc.E_INVAL
    # a neighbour id equal to n
    bad_adj = adj.copy()
    bad_adj[3] = n
    assert _noalloc(f, torch, n, off, deg, bad_adj, colors)[0] == dc.E_INVAL
    # and the next clean call is unaffected by the flags the bad ones left
    rc, conf, _, _ = _noalloc(f, torch, n, off, deg, adj_del, colors)
    assert rc == dc.OK and conf == want

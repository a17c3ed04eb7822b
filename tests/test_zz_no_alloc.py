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

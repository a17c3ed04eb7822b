"""Resident multi-graph pool (include/dyncolor_pool.h) through ctypes.

Many graphs stay resident in one device context under a fixed budget of
adjacency slots; the update batches of several graphs are recoloured in the
same launches, each graph ending as a separate run of its batch would.
Graphs that do not fit are held in pinned host memory and reloaded on use.
The reference recolours one graph per process run (HI/Color_main.cu:21-216)
and has no counterpart.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import CHANGE_DTYPE, HI, OK, DcError, Stats, _ptr, lib, status_str


class PoolOptions(C.Structure):
    _fields_ = [
        ("variant", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
        ("max_graphs", C.c_int32),
        ("vertex_capacity", C.c_int32),
        ("pool_slots", C.c_int64),
        ("iter_cap", C.c_int64),
        ("slack", C.c_float),
        ("blocks_per_sm", C.c_int32),
        ("unit_slots", C.c_int32),
        ("cuda_graph", C.c_int32),
        ("stage_slots", C.c_int64),
        ("pool_slots_max", C.c_int64),
        ("grid_ctas", C.c_int32),
        ("heavy_min_live", C.c_int32),
        ("reserved", C.c_int32 * 6),
    ]


class PoolRequest(C.Structure):
    _fields_ = [("graph", C.c_int32), ("pad", C.c_int32), ("lines", C.c_void_p), ("k", C.c_int64)]


class PoolResult(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("restored", C.c_int32), ("pad", C.c_int32)]


class PoolInfo(C.Structure):
    _fields_ = [
        ("graphs", C.c_int32),
        ("resident", C.c_int32),
        ("resident_vertices", C.c_int64),
        ("vertex_capacity", C.c_int64),
        ("pool_slots_used", C.c_int64),
        ("pool_slots", C.c_int64),
        ("pool_slots_budget", C.c_int64),
        ("pool_slots_max", C.c_int64),
        ("overbudget", C.c_int64),
        ("spills", C.c_int64),
        ("restores", C.c_int64),
        ("spill_bytes", C.c_int64),
        ("restore_bytes", C.c_int64),
        ("spill_ms", C.c_double),
        ("restore_ms", C.c_double),
        ("launches", C.c_int64),
        ("compactions", C.c_int64),
        ("device_bytes", C.c_int64),
        ("host_bytes", C.c_int64),
        ("compact_ms", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        P = C.c_void_p
        L.dc_pool_options_default.argtypes = [C.POINTER(PoolOptions)]
        L.dc_pool_create.argtypes = [C.POINTER(P), C.POINTER(PoolOptions)]
        L.dc_pool_destroy.argtypes = [P]
        L.dc_pool_destroy.restype = None
        L.dc_pool_add_graph.argtypes = [P, C.c_int32, P, P, C.c_int64, P, C.POINTER(C.c_int32)]
        L.dc_pool_apply.argtypes = [P, C.POINTER(PoolRequest), C.c_int32, C.POINTER(PoolResult),
                                    C.POINTER(Stats)]
        L.dc_pool_colors_read.argtypes = [P, C.c_int32, P, C.c_int32]
        L.dc_pool_spill.argtypes = [P, C.c_int32]
        L.dc_pool_graph_size.argtypes = [P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int32)]
        L.dc_pool_info_get.argtypes = [P, C.POINTER(PoolInfo)]
        L.dc_pool_last_error.argtypes = [P]
        L.dc_pool_last_error.restype = C.c_char_p
        _bound = True
    return L


class ResidentPool:
    """Graphs registered with add_graph get ids 0, 1, ...; apply() takes
    [(graph, lines), ...] with at most one batch per graph."""

    def __init__(self, variant: int = HI, vertex_capacity: int = 1 << 22, pool_slots: int = 1 << 28,
                 max_graphs: int = 1024, device: int = 0, iter_cap: int = 0, slack: float = 0.0,
                 blocks_per_sm: int = 0, unit_slots: int = 0, cuda_graph: bool = False,
                 stage_slots: int = 0, pool_slots_max: int = 0, stream: int = 0, grid_ctas: int = 0,
                 heavy_min_live: int = 0):
        L = _lib()
        o = PoolOptions()
        L.dc_pool_options_default(C.byref(o))
        o.variant = variant
        o.device = device
        o.stream = stream or None
        o.max_graphs = max_graphs
        o.vertex_capacity = vertex_capacity
        o.pool_slots = pool_slots
        if iter_cap:
            o.iter_cap = iter_cap
        if slack:
            o.slack = slack
        o.blocks_per_sm = blocks_per_sm
        if unit_slots:
            o.unit_slots = unit_slots
        o.cuda_graph = 1 if cuda_graph else 0
        if stage_slots:
            o.stage_slots = stage_slots
        o.pool_slots_max = pool_slots_max
        o.grid_ctas = grid_ctas
        o.heavy_min_live = heavy_min_live
        h = C.c_void_p()
        rc = L.dc_pool_create(C.byref(h), C.byref(o))
        if rc != OK:
            raise DcError(rc, f"dc_pool_create: {status_str(rc)}")
        self._h = h
        self.sizes: list[int] = []

    def close(self):
        if getattr(self, "_h", None):
            _lib().dc_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != OK:
            msg = _lib().dc_pool_last_error(self._h).decode(errors="replace")
            raise DcError(rc, f"{what}: {status_str(rc)}: {msg}")

    def add_graph(self, n: int, a, b, colors) -> int:
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        c = np.ascontiguousarray(colors, dtype=np.int32)
        if len(c) != n:
            raise ValueError("colour array size differs from n")
        g = C.c_int32(-1)
        self._check(_lib().dc_pool_add_graph(self._h, n, _ptr(a), _ptr(b), len(a), _ptr(c), C.byref(g)),
                    "dc_pool_add_graph")
        self.sizes.append(n)
        return g.value

    def apply(self, batches, check: bool = True):
        """batches: [(graph, lines structured array), ...]. Returns
        (launch Stats, per-request iterations array, per-request restored flags)."""
        cnt = len(batches)
        reqs = (PoolRequest * max(cnt, 1))()
        keep = []
        for i, (g, lines) in enumerate(batches):
            x = np.ascontiguousarray(lines, dtype=CHANGE_DTYPE)
            keep.append(x)
            reqs[i].graph = int(g)
            reqs[i].lines = x.ctypes.data if len(x) else None
            reqs[i].k = len(x)
        res = (PoolResult * max(cnt, 1))()
        st = Stats()
        rc = _lib().dc_pool_apply(self._h, reqs, cnt, res, C.byref(st))
        if check:
            self._check(rc, "dc_pool_apply")
        its = np.array([res[i].iterations for i in range(cnt)], dtype=np.int64)
        restored = np.array([res[i].restored for i in range(cnt)], dtype=np.int32)
        st.status = rc
        return st, its, restored

    def colors(self, graph: int) -> np.ndarray:
        out = np.empty(self.sizes[graph], dtype=np.int32)
        self._check(_lib().dc_pool_colors_read(self._h, graph, _ptr(out), len(out)), "dc_pool_colors_read")
        return out

    def spill(self, graph: int):
        self._check(_lib().dc_pool_spill(self._h, graph), "dc_pool_spill")

    def graph_size(self, graph: int):
        n, slots, res = C.c_int32(), C.c_int64(), C.c_int32()
        self._check(_lib().dc_pool_graph_size(self._h, graph, C.byref(n), C.byref(slots), C.byref(res)),
                    "dc_pool_graph_size")
        return n.value, slots.value, bool(res.value)

    def info(self) -> dict:
        i = PoolInfo()
        self._check(_lib().dc_pool_info_get(self._h, C.byref(i)), "dc_pool_info_get")
        return i.as_dict()

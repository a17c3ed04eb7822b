"""dyncolor_b200 -- incremental graph recolouring on B200 (sm_100a).

Thin ctypes mirror of the C ABI in ``include/dyncolor.h`` (libdyncolor.so,
built in-tree by ``make -C dyncolor_b200/csrc``).  The call surface follows
the reference drivers' host phases:

=====================  ==============================================
reference phase         here
=====================  ==============================================
read_graphEdges +       ``Context.load_edges(n, a, b)``
transfer_data_to_GPU
read_Input_Color        ``Context.set_colors(colors)``
readin_changes +        ``Context.apply_batch(changes)``
kernels + loop
vertexcolor readback    ``Context.colors()``
validate kernel         ``Context.validate()``
=====================  ==============================================

There is no CPU path: if the shared library is missing or no CUDA device is
usable, constructing a :class:`Context` raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import io  # noqa: F401  (reference text formats)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdyncolor.so")

HI, HB = 0, 1
OK, E_INVAL, E_NOMEM, E_CUDA, E_ITER_LIMIT, E_STATE, E_TIMEOUT, E_INTERNAL = range(8)
INS_UNIFORM, INS_RMAT, INS_DEGREE = 0, 1, 2
ORDER_ID, ORDER_LDF = 0, 1

CHANGE_DTYPE = np.dtype([("node1", "<i4"), ("node2", "<i4"), ("inst", "<i4")])


class Options(C.Structure):
    _fields_ = [
        ("variant", C.c_int32),
        ("device", C.c_int32),
        ("stream", C.c_void_p),
        ("iter_cap", C.c_int64),
        ("slack", C.c_float),
        ("blocks_per_sm", C.c_int32),
        ("reserve_slots", C.c_int64),
        ("unit_slots", C.c_int32),
        ("cuda_graph", C.c_int32),
        ("heavy_min_live", C.c_int32),
        ("barrier_timeout_ms", C.c_int32),
        ("grid_ctas", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("seed_targets", C.c_int64),
        ("frontier_total", C.c_int64),
        ("slots_scanned", C.c_int64),
        ("edges_inserted", C.c_int64),
        ("edges_deleted", C.c_int64),
        ("rows_relocated", C.c_int64),
        ("status", C.c_int32),
        ("max_color", C.c_int32),
        ("device_ms", C.c_double),
        ("struct_ms", C.c_double),
        ("recolor_ms", C.c_double),
        ("phase_ms", C.c_double * 6),
        ("slots_read", C.c_int64),
        ("pairs", C.c_int64),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["phase_ms"] = list(self.phase_ms)
        return d


class GraphInfo(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("edges", C.c_int64),
        ("slots_used", C.c_int64),
        ("slots_capacity", C.c_int64),
        ("device_bytes", C.c_int64),
    ]


class DcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status
        self.message = message


_lib = None


def lib() -> C.CDLL:
    """Loads libdyncolor.so; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C dyncolor_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    L.dc_options_default.argtypes = [C.POINTER(Options)]
    L.dc_create.argtypes = [C.POINTER(P), C.POINTER(Options)]
    L.dc_destroy.argtypes = [P]
    L.dc_destroy.restype = None
    L.dc_graph_load_edges.argtypes = [P, C.c_int32, P, P, C.c_int64]
    L.dc_colors_set.argtypes = [P, P, C.c_int32]
    L.dc_colors_init_greedy.argtypes = [P]
    L.dc_colors_init.argtypes = [P, C.c_int32]
    L.dc_apply_batch.argtypes = [P, P, C.c_int64, C.POINTER(Stats)]
    L.dc_apply_batch_device.argtypes = [P, P, C.c_int64, C.POINTER(Stats)]
    L.dc_colors_read.argtypes = [P, P, C.c_int32]
    L.dc_colors_device.argtypes = [P, C.POINTER(P)]
    L.dc_prop_read.argtypes = [P, P, C.c_int32]
    L.dc_validate.argtypes = [P, C.POINTER(C.c_int64)]
    L.dc_neighbors.argtypes = [P, C.c_int32, P, C.c_int32, C.POINTER(C.c_int32)]
    L.dc_graph_info_get.argtypes = [P, C.POINTER(GraphInfo)]
    L.dc_compact.argtypes = [P]
    L.dc_partition_set.argtypes = [P, C.c_int32, P]
    L.dc_graph_iterations.argtypes = [P, P, C.c_int32]
    L.dc_last_error.argtypes = [P]
    L.dc_last_error.restype = C.c_char_p
    L.dc_status_str.argtypes = [C.c_int]
    L.dc_status_str.restype = C.c_char_p
    L.dcg_rmat.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_double, C.c_double, C.c_double,
                           C.c_uint64, P, P]
    L.dcg_uniform_pairs.argtypes = [C.c_int32, C.c_int64, C.c_uint64, P, P]
    L.dcg_chung_lu.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, P, P,
                               C.c_int64]
    L.dcg_chung_lu.restype = C.c_int64
    L.dcg_dedup.argtypes = [C.c_int32, P, P, C.c_int64]
    L.dcg_dedup.restype = C.c_int64
    L.dcg_greedy_color.argtypes = [C.c_int32, P, P, C.c_int64, P]
    L.dcg_edgeset_create.argtypes = [C.c_int32, P, P, C.c_int64]
    L.dcg_edgeset_create.restype = P
    L.dcg_edgeset_destroy.argtypes = [P]
    L.dcg_edgeset_destroy.restype = None
    L.dcg_edgeset_size.argtypes = [P]
    L.dcg_edgeset_size.restype = C.c_int64
    L.dcg_edgeset_sample_batch.argtypes = [P, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                           C.c_double, C.c_double, C.c_double, C.c_uint64, P]
    L.dcg_edgeset_sample_batch.restype = C.c_int64
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def as_changes(node1, node2, inst) -> np.ndarray:
    ch = np.empty(len(node1), dtype=CHANGE_DTYPE)
    ch["node1"] = node1
    ch["node2"] = node2
    ch["inst"] = inst
    return ch


def status_str(s: int) -> str:
    return lib().dc_status_str(s).decode()


class Context:
    """One graph + colouring on one GPU (dc_ctx)."""

    def __init__(self, variant: int = HI, device: int = 0, iter_cap: int = 0, slack: float = 0.0,
                 blocks_per_sm: int = 0, unit_slots: int = 0, stream: int | None = None,
                 reserve_slots: int = 0, cuda_graph: bool = False, heavy_min_live: int = 0,
                 barrier_timeout_ms: int = 0, grid_ctas: int = 0):
        L = lib()
        opt = Options()
        L.dc_options_default(C.byref(opt))
        opt.variant = int(variant)
        opt.device = int(device)
        if iter_cap:
            opt.iter_cap = int(iter_cap)
        if slack:
            opt.slack = float(slack)
        opt.blocks_per_sm = int(blocks_per_sm)
        if unit_slots:
            opt.unit_slots = int(unit_slots)
        opt.reserve_slots = int(reserve_slots)
        opt.cuda_graph = 1 if cuda_graph else 0
        opt.heavy_min_live = int(heavy_min_live)
        if barrier_timeout_ms:
            opt.barrier_timeout_ms = int(barrier_timeout_ms)
        opt.grid_ctas = int(grid_ctas)
        opt.stream = stream
        h = C.c_void_p()
        rc = L.dc_create(C.byref(h), C.byref(opt))
        if rc != OK:
            raise DcError(rc, f"dc_create failed: {status_str(rc)}")
        self._h = h
        self.variant = int(variant)
        self.n = None

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().dc_destroy(h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != OK:
            msg = lib().dc_last_error(self._h).decode()
            raise DcError(rc, f"{what}: {status_str(rc)}: {msg}")

    def last_error(self) -> str:
        return lib().dc_last_error(self._h).decode()

    def load_edges(self, n: int, a, b):
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        if a.shape != b.shape:
            raise ValueError("a and b differ in length")
        self._check(lib().dc_graph_load_edges(self._h, int(n), _ptr(a), _ptr(b), len(a)),
                    "dc_graph_load_edges")
        self.n = int(n)

    def set_colors(self, colors):
        c = np.ascontiguousarray(colors, dtype=np.int32)
        self._check(lib().dc_colors_set(self._h, _ptr(c), len(c)), "dc_colors_set")

    def init_greedy_colors(self):
        """Greedy lowest-free colouring in vertex-id order of the current graph."""
        self._check(lib().dc_colors_init_greedy(self._h), "dc_colors_init_greedy")

    def init_colors(self, order: int = ORDER_ID):
        """Greedy lowest-free colouring of the current graph in the given
        order (ORDER_ID: vertex ids; ORDER_LDF: largest live degree first),
        computed on the device."""
        self._check(lib().dc_colors_init(self._h, int(order)), "dc_colors_init")

    def apply_batch(self, changes, check: bool = True) -> Stats:
        ch = np.ascontiguousarray(changes, dtype=CHANGE_DTYPE)
        st = Stats()
        rc = lib().dc_apply_batch(self._h, _ptr(ch), len(ch), C.byref(st))
        if check:
            self._check(rc, "dc_apply_batch")
        st.status = rc
        return st

    def apply_batch_device(self, d_changes: int, k: int, check: bool = True) -> Stats:
        st = Stats()
        rc = lib().dc_apply_batch_device(self._h, C.c_void_p(d_changes), int(k), C.byref(st))
        if check:
            self._check(rc, "dc_apply_batch_device")
        st.status = rc
        return st

    def colors(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n, dtype=np.int32)
        self._check(lib().dc_colors_read(self._h, _ptr(out), self.n), "dc_colors_read")
        return out

    def colors_device_ptr(self) -> int:
        p = C.c_void_p()
        self._check(lib().dc_colors_device(self._h, C.byref(p)), "dc_colors_device")
        return int(p.value or 0)

    def prop(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        self._check(lib().dc_prop_read(self._h, _ptr(out), self.n), "dc_prop_read")
        return out

    def validate(self) -> int:
        c = C.c_int64()
        self._check(lib().dc_validate(self._h, C.byref(c)), "dc_validate")
        return int(c.value)

    def neighbors(self, v: int) -> np.ndarray:
        deg = C.c_int32()
        self._check(lib().dc_neighbors(self._h, int(v), None, 0, C.byref(deg)), "dc_neighbors")
        out = np.empty(max(deg.value, 1), dtype=np.int32)
        self._check(lib().dc_neighbors(self._h, int(v), _ptr(out), len(out), C.byref(deg)),
                    "dc_neighbors")
        return np.sort(out[: deg.value])

    def info(self) -> dict:
        gi = GraphInfo()
        self._check(lib().dc_graph_info_get(self._h, C.byref(gi)), "dc_graph_info_get")
        return {f: getattr(gi, f) for f, _ in gi._fields_}

    def compact(self):
        self._check(lib().dc_compact(self._h), "dc_compact")

    def set_partition(self, first):
        """Batched mode: graph g owns vertices [first[g], first[g+1])."""
        f = np.ascontiguousarray(first, dtype=np.int32)
        self._check(lib().dc_partition_set(self._h, len(f) - 1, _ptr(f)), "dc_partition_set")
        self.ngraphs = len(f) - 1

    def graph_iterations(self) -> np.ndarray:
        out = np.empty(self.ngraphs, dtype=np.int64)
        self._check(lib().dc_graph_iterations(self._h, _ptr(out), self.ngraphs), "dc_graph_iterations")
        return out


# ---------------------------------------------------------------------------
# generators (include/dyncolor_gen.h)
# ---------------------------------------------------------------------------

def rmat(scale: int, m: int, a=0.57, b=0.19, c=0.19, seed=1, n: int | None = None):
    n = (1 << scale) if n is None else int(n)
    xa = np.empty(m, dtype=np.int32)
    xb = np.empty(m, dtype=np.int32)
    rc = lib().dcg_rmat(scale, n, m, a, b, c, seed, _ptr(xa), _ptr(xb))
    if rc != OK:
        raise DcError(rc, "dcg_rmat")
    return xa, xb


def uniform_pairs(n: int, m: int, seed=1):
    xa = np.empty(m, dtype=np.int32)
    xb = np.empty(m, dtype=np.int32)
    rc = lib().dcg_uniform_pairs(n, m, seed, _ptr(xa), _ptr(xb))
    if rc != OK:
        raise DcError(rc, "dcg_uniform_pairs")
    return xa, xb


def chung_lu(n: int, gamma: float, avg_deg: float, max_deg: float, seed=1):
    cap = int(round(n * avg_deg / 2)) + 1
    xa = np.empty(cap, dtype=np.int32)
    xb = np.empty(cap, dtype=np.int32)
    m = lib().dcg_chung_lu(n, gamma, avg_deg, max_deg, seed, _ptr(xa), _ptr(xb), cap)
    if m < 0:
        raise DcError(-m, "dcg_chung_lu")
    return xa[:m].copy(), xb[:m].copy()


def dedup(n: int, a, b):
    a = np.array(a, dtype=np.int32, copy=True)
    b = np.array(b, dtype=np.int32, copy=True)
    m = lib().dcg_dedup(n, _ptr(a), _ptr(b), len(a))
    if m < 0:
        raise DcError(-m, "dcg_dedup")
    return a[:m].copy(), b[:m].copy()


def greedy_color(n: int, a, b) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    out = np.zeros(n, dtype=np.int32)
    rc = lib().dcg_greedy_color(n, _ptr(a), _ptr(b), len(a), _ptr(out))
    if rc != OK:
        raise DcError(rc, "dcg_greedy_color")
    return out


class EdgeSet:
    """Current edge set used to draw update batches (dcg_edgeset)."""

    def __init__(self, n: int, a, b):
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        self._h = lib().dcg_edgeset_create(n, _ptr(a), _ptr(b), len(a))
        if not self._h:
            raise MemoryError("dcg_edgeset_create")
        self.n = n

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().dcg_edgeset_destroy(h)
            self._h = None

    def size(self) -> int:
        return int(lib().dcg_edgeset_size(self._h))

    def sample_batch(self, k_del: int, k_ins: int, mode: int = INS_UNIFORM, scale: int = 0,
                     a=0.57, b=0.19, c=0.19, seed=1) -> np.ndarray:
        out = np.empty(k_del + k_ins, dtype=CHANGE_DTYPE)
        w = lib().dcg_edgeset_sample_batch(self._h, k_del, k_ins, mode, scale, a, b, c, seed,
                                           _ptr(out))
        if w < 0:
            raise DcError(-w, "dcg_edgeset_sample_batch")
        return out[:w]

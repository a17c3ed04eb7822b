"""ctypes wrapper of liboracle.so -- the CPU checker for the parity tests.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py``.  The product package never
imports it.

Also parses the reference's text formats (graph ``a b w`` lines, colour
``node color`` lines, change ``a b w inst`` lines; see
HI/all_structure_undir.cuh:78-183) and runs the reference harness binaries in
``oracle/_ref`` when they exist.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

HI, HB = 0, 1
SNAPSHOT, SERIAL = 0, 1
OK, E_INVAL, E_NOMEM, E_ITER_LIMIT = 0, 1, 2, 4


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int64),
        ("seed_targets", C.c_int64),
        ("frontier_total", C.c_int64),
        ("slots_scanned", C.c_int64),
        ("changed_vertices", C.c_int64),
        ("status", C.c_int32),
        ("max_color", C.c_int32),
        ("internal_pairs", C.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


CHANGE_DTYPE = np.dtype([("node1", "<i4"), ("node2", "<i4"), ("inst", "<i4")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("liboracle.so not built: run `make -C oracle`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int32]
        L.orc_destroy.argtypes = [P]
        L.orc_load_edges.argtypes = [P, P, P, C.c_int64]
        L.orc_set_colors.argtypes = [P, P]
        L.orc_get_colors.argtypes = [P, P]
        L.orc_get_prop.argtypes = [P, P]
        L.orc_apply_batch.argtypes = [P, C.c_int, C.c_int, P, C.c_int64, C.c_int64, C.POINTER(Stats)]
        L.orc_conflicts.restype = C.c_int64
        L.orc_conflicts.argtypes = [P]
        L.orc_live_degree.restype = C.c_int32
        L.orc_live_degree.argtypes = [P, C.c_int32]
        L.orc_neighbors.restype = C.c_int32
        L.orc_neighbors.argtypes = [P, C.c_int32, P, C.c_int32]
        L.orc_is_greedy_id_order.argtypes = [P]
        L.orc_greedy_id_order.argtypes = [P]
        L.orc_greedy_in_order.argtypes = [P, P]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_instrument.argtypes = [C.c_int]
        # seeded workload generators (dc_gen.cpp compiled into this library)
        L.dcg_rmat.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, P, P]
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
        L.dcg_edgeset_sample_batch.argtypes = [P, C.c_int64, C.c_int64, C.c_int32, C.c_int32,
                                               C.c_double, C.c_double, C.c_double, C.c_uint64, P]
        L.dcg_edgeset_sample_batch.restype = C.c_int64
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def as_changes(node1, node2, inst) -> np.ndarray:
    ch = np.empty(len(node1), dtype=CHANGE_DTYPE)
    ch["node1"] = node1
    ch["node2"] = node2
    ch["inst"] = inst
    return ch


class Graph:
    """One graph + colouring held by the C oracle."""

    def __init__(self, n: int):
        self.n = int(n)
        self._g = lib().orc_create(self.n)
        if not self._g:
            raise MemoryError("orc_create failed")

    def __del__(self):
        g = getattr(self, "_g", None)
        if g:
            lib().orc_destroy(g)
            self._g = None

    def load_edges(self, a, b) -> int:
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        return lib().orc_load_edges(self._g, _ptr(a), _ptr(b), len(a))

    def set_colors(self, colors) -> int:
        c = np.ascontiguousarray(colors, dtype=np.int32)
        assert len(c) == self.n
        return lib().orc_set_colors(self._g, _ptr(c))

    def colors(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        lib().orc_get_colors(self._g, _ptr(out))
        return out

    def prop(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.int32)
        lib().orc_get_prop(self._g, _ptr(out))
        return out

    def apply_batch(self, changes: np.ndarray, variant: int, schedule: int = SNAPSHOT,
                    iter_cap: int = 1 << 40):
        ch = np.ascontiguousarray(changes, dtype=CHANGE_DTYPE)
        st = Stats()
        rc = lib().orc_apply_batch(self._g, variant, schedule, _ptr(ch), len(ch), iter_cap, C.byref(st))
        return rc, st

    def conflicts(self) -> int:
        return int(lib().orc_conflicts(self._g))

    def live_degree(self, v: int) -> int:
        return int(lib().orc_live_degree(self._g, v))

    def neighbors(self, v: int) -> np.ndarray:
        d = lib().orc_neighbors(self._g, int(v), None, 0)
        out = np.empty(max(d, 1), dtype=np.int32)
        lib().orc_neighbors(self._g, int(v), _ptr(out), len(out))
        return out[:d]

    def is_greedy_id_order(self) -> bool:
        return lib().orc_is_greedy_id_order(self._g) == 1

    def greedy_in_order(self, order) -> int:
        o = np.ascontiguousarray(order, dtype=np.int32)
        return lib().orc_greedy_in_order(self._g, _ptr(o))

    def greedy_id_order(self) -> int:
        return lib().orc_greedy_id_order(self._g)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


# ---------------------------------------------------------------------------
# workload generators (the product's dc_gen.cpp, compiled into liboracle.so,
# so a checker-side process can build the benchmark inputs without loading
# libdyncolor.so; same seeds give the same graphs and batches)
# ---------------------------------------------------------------------------

INS_UNIFORM, INS_RMAT, INS_DEGREE = 0, 1, 2


def gen_rmat(scale: int, m: int, seed: int = 1, a=0.57, b=0.19, c=0.19):
    n = 1 << scale
    xa = np.empty(m, dtype=np.int32)
    xb = np.empty(m, dtype=np.int32)
    if lib().dcg_rmat(scale, n, m, a, b, c, seed, _ptr(xa), _ptr(xb)) != OK:
        raise RuntimeError("dcg_rmat")
    return xa, xb


def gen_chung_lu(n: int, gamma: float, avg_deg: float, max_deg: float, seed: int = 1):
    cap = int(round(n * avg_deg / 2)) + 1
    xa = np.empty(cap, dtype=np.int32)
    xb = np.empty(cap, dtype=np.int32)
    m = lib().dcg_chung_lu(n, gamma, avg_deg, max_deg, seed, _ptr(xa), _ptr(xb), cap)
    if m < 0:
        raise RuntimeError("dcg_chung_lu")
    return xa[:m].copy(), xb[:m].copy()


def gen_dedup(n: int, a, b):
    a = np.array(a, dtype=np.int32, copy=True)
    b = np.array(b, dtype=np.int32, copy=True)
    m = lib().dcg_dedup(n, _ptr(a), _ptr(b), len(a))
    if m < 0:
        raise RuntimeError("dcg_dedup")
    return a[:m].copy(), b[:m].copy()


def gen_greedy_color(n: int, a, b) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    out = np.zeros(n, dtype=np.int32)
    if lib().dcg_greedy_color(n, _ptr(a), _ptr(b), len(a), _ptr(out)) != OK:
        raise RuntimeError("dcg_greedy_color")
    return out


class GenEdgeSet:
    """Edge set that draws update batches (dcg_edgeset)."""

    def __init__(self, n: int, a, b):
        a = np.ascontiguousarray(a, dtype=np.int32)
        b = np.ascontiguousarray(b, dtype=np.int32)
        self._h = lib().dcg_edgeset_create(n, _ptr(a), _ptr(b), len(a))
        if not self._h:
            raise MemoryError("dcg_edgeset_create")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().dcg_edgeset_destroy(h)
            self._h = None

    def sample_batch(self, k_del: int, k_ins: int, mode: int = INS_UNIFORM, scale: int = 0, seed: int = 1,
                     a=0.57, b=0.19, c=0.19) -> np.ndarray:
        out = np.empty(k_del + k_ins, dtype=CHANGE_DTYPE)
        w = lib().dcg_edgeset_sample_batch(self._h, k_del, k_ins, mode, scale, a, b, c, seed, _ptr(out))
        if w < 0:
            raise RuntimeError("dcg_edgeset_sample_batch")
        return out[:w]


# ---------------------------------------------------------------------------
# reference text formats
# ---------------------------------------------------------------------------

def parse_graph_file(path):
    """``a b w`` per line (read_graphEdges)."""
    a, b = [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) >= 2:
                a.append(int(p[0]))
                b.append(int(p[1]))
    return np.array(a, dtype=np.int32), np.array(b, dtype=np.int32)


def parse_color_file(path, n):
    """``node color`` per line (read_Input_Color)."""
    c = np.zeros(n, dtype=np.int32)
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) >= 2:
                c[int(p[0])] = int(p[1])
    return c


def parse_change_file(path):
    """``a b w inst`` per line (readin_changes)."""
    rows = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) >= 4:
                rows.append((int(p[0]), int(p[1]), int(p[3])))
    ch = np.empty(len(rows), dtype=CHANGE_DTYPE)
    for i, (x, y, t) in enumerate(rows):
        ch[i] = (x, y, t)
    return ch


def write_graph_file(path, a, b):
    with open(path, "w") as f:
        for x, y in zip(a.tolist(), b.tolist()):
            f.write(f"{x} {y} 1\n")


def write_color_file(path, colors):
    with open(path, "w") as f:
        for v, c in enumerate(colors.tolist()):
            f.write(f"{v} {c}\n")


def write_change_file(path, changes):
    with open(path, "w") as f:
        for x, y, t in zip(changes["node1"].tolist(), changes["node2"].tolist(),
                           changes["inst"].tolist()):
            f.write(f"{x} {y} 1 {t}\n")


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, b)) for b in ("ref_hi", "ref_hb"))


def run_ref(variant: int, schedule: int, a, b, colors, changes, iter_cap: int = 100000):
    """Runs the reference's own kernel bodies (oracle/_ref) on one batch.

    Returns (iterations, status, colors)."""
    exe = os.path.join(REF_DIR, "ref_hi" if variant == HI else "ref_hb")
    mode = "snapshot" if schedule == SNAPSHOT else "serial"
    n = len(colors)
    with tempfile.TemporaryDirectory() as d:
        gp, cp, xp, op = (os.path.join(d, x) for x in ("g.txt", "c.txt", "x.txt", "o.txt"))
        write_graph_file(gp, a, b)
        write_color_file(cp, colors)
        write_change_file(xp, changes)
        subprocess.run([exe, mode, gp, str(n), str(len(a)), cp, xp, op, str(iter_cap)],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)
        with open(op) as f:
            head = f.readline().split()
            cols = np.array([int(x) for x in f.read().split()], dtype=np.int32)
    return int(head[1]), int(head[3]), cols

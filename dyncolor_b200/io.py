"""Reference text formats (host side).

* graph file: one ``a b w`` line per undirected edge, weight ignored
  (read_graphEdges, HI/all_structure_undir.cuh:156-183);
* colour file: ``node color`` lines (read_Input_Color,
  HI/all_structure_undir.cuh:130-150);
* change file: ``a b w inst`` lines, inst 1 insert / 0 delete, other values
  ignored (readin_changes, HI/all_structure_undir.cuh:78-128).

Lines with fewer fields than the format needs are skipped, like the
reference's ``sscanf`` leaves them unused.
"""
from __future__ import annotations

import numpy as np

CHANGE_DTYPE = np.dtype([("node1", "<i4"), ("node2", "<i4"), ("inst", "<i4")])


def _rows(path, width):
    out = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if len(p) >= width:
                out.append([int(x) for x in p[:width]])
    return out


def read_graph(path):
    """Returns (a, b) int32 arrays of the edge lines."""
    r = _rows(path, 2)
    arr = np.array(r, dtype=np.int32).reshape(-1, 2)
    return arr[:, 0].copy(), arr[:, 1].copy()


def read_colors(path, n: int) -> np.ndarray:
    """Colour per vertex; vertices without a line keep colour 0."""
    c = np.zeros(n, dtype=np.int32)
    for v, col in _rows(path, 2):
        c[v] = col
    return c


def read_changes(path) -> np.ndarray:
    r = _rows(path, 4)
    ch = np.empty(len(r), dtype=CHANGE_DTYPE)
    for i, (a, b, _w, inst) in enumerate(r):
        ch[i] = (a, b, inst)
    return ch


def write_graph(path, a, b):
    with open(path, "w") as f:
        for x, y in zip(np.asarray(a).tolist(), np.asarray(b).tolist()):
            f.write(f"{x} {y} 1\n")


def write_colors(path, colors):
    with open(path, "w") as f:
        for v, c in enumerate(np.asarray(colors).tolist()):
            f.write(f"{v} {c}\n")


def write_changes(path, changes):
    with open(path, "w") as f:
        for x, y, t in zip(changes["node1"].tolist(), changes["node2"].tolist(),
                           changes["inst"].tolist()):
            f.write(f"{x} {y} 1 {t}\n")

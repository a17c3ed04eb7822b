"""Shared helpers of the test-suite: workload builders and the oracle runner."""
import numpy as np

import dyncolor_b200 as dc
import pyoracle as po


def changes_from_golden(c):
    arr = c["changes"]
    return po.as_changes(arr[:, 0], arr[:, 1], arr[:, 2]) if len(arr) else np.empty(0, po.CHANGE_DTYPE)


def rmat_graph(scale, ef=16, seed=1):
    n = 1 << scale
    a, b = dc.rmat(scale, ef * n, seed=seed)
    a, b = dc.dedup(n, a, b)
    return n, a, b


def er_graph(n, avg_deg, seed=1):
    m = int(n * avg_deg / 2)
    a, b = dc.uniform_pairs(n, m, seed=seed)
    a, b = dc.dedup(n, a, b)
    return n, a, b


def oracle_graph(n, a, b, colors):
    g = po.Graph(n)
    assert g.load_edges(a, b) == po.OK
    assert g.set_colors(colors) == po.OK
    return g


def to_oracle_changes(ch):
    out = np.empty(len(ch), dtype=po.CHANGE_DTYPE)
    out["node1"] = ch["node1"]
    out["node2"] = ch["node2"]
    out["inst"] = ch["inst"]
    return out


def to_dc_changes(ch):
    out = np.empty(len(ch), dtype=dc.CHANGE_DTYPE)
    out["node1"] = ch["node1"]
    out["node2"] = ch["node2"]
    out["inst"] = ch["inst"]
    return out

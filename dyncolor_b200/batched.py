"""Batched mode: many independent graphs recoloured in the same launches.

The graphs are loaded as one disjoint union (graph g owns a contiguous
vertex range) and declared with ``dc_partition_set``; every update batch is
the concatenation of the graphs' own batches.  Each graph ends exactly as a
separate run of it would (colours and loop iterations); the reference has
no counterpart (it recolours one graph per process).
"""
from __future__ import annotations

import numpy as np

from . import CHANGE_DTYPE, HI, Context


class BatchedContext:
    def __init__(self, variant: int = HI, **ctx_kw):
        self.ctx = Context(variant=variant, **ctx_kw)
        self.first = None

    def close(self):
        self.ctx.close()

    def load(self, graphs):
        """graphs: sequence of (n, a, b) with local vertex ids."""
        sizes = np.array([int(n) for n, _, _ in graphs], dtype=np.int64)
        first = np.zeros(len(graphs) + 1, dtype=np.int64)
        first[1:] = np.cumsum(sizes)
        if first[-1] >= 2**31:
            raise ValueError("the union exceeds 2^31 vertices")
        m = sum(len(x) for _, x, _ in graphs)
        a = np.empty(m, dtype=np.int32)
        b = np.empty(m, dtype=np.int32)
        at = 0
        for i, (_, x, y) in enumerate(graphs):
            np.add(x, np.int32(first[i]), out=a[at:at + len(x)], casting="unsafe")
            np.add(y, np.int32(first[i]), out=b[at:at + len(y)], casting="unsafe")
            at += len(x)
        self.ctx.load_edges(int(first[-1]), a, b)
        del a, b
        self.first = first.astype(np.int32)
        self.ctx.set_partition(self.first)

    @property
    def n(self) -> int:
        return int(self.first[-1])

    def set_colors(self, colors_per_graph):
        self.ctx.set_colors(np.concatenate([np.asarray(c, np.int32) for c in colors_per_graph]))

    def union_batch(self, batches) -> np.ndarray:
        """Concatenates per-graph change lines, shifting ids to union ids."""
        parts = []
        for g, ch in enumerate(batches):
            if len(ch) == 0:
                continue
            x = np.empty(len(ch), dtype=CHANGE_DTYPE)
            x["node1"] = ch["node1"] + self.first[g]
            x["node2"] = ch["node2"] + self.first[g]
            x["inst"] = ch["inst"]
            parts.append(x)
        return np.concatenate(parts) if parts else np.empty(0, dtype=CHANGE_DTYPE)

    def apply(self, batches, check: bool = True):
        return self.ctx.apply_batch(self.union_batch(batches), check=check)

    def colors(self):
        c = self.ctx.colors()
        return [c[self.first[g]:self.first[g + 1]] for g in range(len(self.first) - 1)]

    def iterations(self) -> np.ndarray:
        return self.ctx.graph_iterations()

"""Generates tests/golden/ref_vectors.npz from the reference's own code.

Run in a container where the reference sources exist (they are compiled into
oracle/_ref by `make -C oracle ref`):

    python tests/golden/make_golden.py

Cases:
  * the reference's sample fixture (graph.txt, prevColor.txt, cE.txt of the
    HI and HB projects), read from the reference tree;
  * seeded random small graphs whose colours stay far below 31, the range in
    which the reference's 32-bit mask arithmetic is exact
    (HI/gpuFunctions_undir.cuh:36-69, HB/gpuFunctions_undir.cuh:36-54).

Each case is run through oracle/_ref/ref_{hi,hb} in both schedules (serial =
the reference's kernels with one thread; snapshot = every kernel item
against the state at the start of its launch) and the resulting colours and
iteration counts are stored.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

REF = "/root/reference"
SAMPLES = {
    "sample_hi": (po.HI, REF + "/DynColorHeuristicIndependent/DynColorHeuristicIndependent"),
    "sample_hb": (po.HB, REF + "/DynColorHeuristicBased/DynColorHeuristicBased"),
}
N_RANDOM = 120
ITER_CAP = 2000


def random_case(rng):
    n = int(rng.integers(2, 64))
    m = int(rng.integers(0, 3 * n))
    a = rng.integers(0, n, m).astype(np.int32)
    b = rng.integers(0, n, m).astype(np.int32)
    keep = a != b
    a, b = a[keep], b[keep]
    ncol = int(rng.integers(1, 9))
    col = rng.integers(0, ncol, n).astype(np.int32)
    k = int(rng.integers(0, 3 * n))
    x = rng.integers(0, n, k)
    y = rng.integers(0, n, k)
    inst = rng.integers(0, 2, k)
    keep = x != y
    ch = po.as_changes(x[keep], y[keep], inst[keep])
    return n, a, b, col, ch


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref not built (make -C oracle ref)")
    out = {}
    names = []

    def put(name, variant, n, a, b, col, ch):
        names.append(name)
        out[f"{name}/variant"] = np.array([variant], dtype=np.int32)
        out[f"{name}/n"] = np.array([n], dtype=np.int32)
        out[f"{name}/a"] = a
        out[f"{name}/b"] = b
        out[f"{name}/colors"] = col
        out[f"{name}/changes"] = np.stack([ch["node1"], ch["node2"], ch["inst"]], axis=1).astype(np.int32)
        for sch, tag in ((po.SERIAL, "serial"), (po.SNAPSHOT, "snapshot")):
            it, status, rc = po.run_ref(variant, sch, a, b, col, ch, iter_cap=ITER_CAP)
            assert rc.max(initial=0) <= 30, "outside the reference's exact colour range"
            out[f"{name}/{tag}_colors"] = rc
            out[f"{name}/{tag}_iters"] = np.array([it, status], dtype=np.int64)

    for name, (variant, d) in SAMPLES.items():
        a, b = po.parse_graph_file(d + "/graph.txt")
        col = po.parse_color_file(d + "/prevColor.txt", 10)
        ch = po.parse_change_file(d + "/cE.txt")
        put(name, variant, 10, a, b, col, ch)
        # the other variant on the same fixture as well
        put(name + "_other", 1 - variant, 10, a, b, col, ch)

    rng = np.random.default_rng(20261203)
    for i in range(N_RANDOM):
        n, a, b, col, ch = random_case(rng)
        put(f"rand{i:03d}", i % 2, n, a, b, col, ch)

    out["_names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "ref_vectors.npz"), **out)
    print(f"wrote {len(names)} cases")


if __name__ == "__main__":
    main()

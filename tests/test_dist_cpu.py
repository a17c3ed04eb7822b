"""The bench's multi-process host logic (one rank per GPU under torchrun) on
CPU: world size 2 over gloo, max/sum over ranks, and the workload that rank 0
builds and the other ranks load from shared memory."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    try:
        d = bench.Dist(world, backend="gloo")
        mx = d.max(float(rank))
        sm = d.sum(float(rank + 1))
        sys.argv = ["bench.py", "--scale", "8", "--batch", "64"]
        args = bench.parse_args()
        w = bench.get_workload(args, d, 2)
        digest = float(np.int64(w["a"]).sum() + 7 * np.int64(w["colors"]).sum()
                       + sum(int(b["node1"].sum()) for b in w["batches"]))
        same = d.max(digest) == digest and d.max(-digest) == -digest
        d.barrier()
        d.close()
        q.put((rank, mx, sm, same, len(w["batches"]), int(w["n"])))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert r[1] != "error", r
        rank, mx, sm, same, nb, n = r
        assert mx == 1.0 and sm == 3.0
        assert same, "ranks loaded different workloads"
        assert nb == 2 and n == 256

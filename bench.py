#!/usr/bin/env python
"""Benchmark: edge-updates/s of incremental recolouring on one or more B200s.

Workload (default): undirected R-MAT graph, scale 24 (16.7 M vertices),
edge factor 16 (a=0.57, b=c=0.19, d=0.05; self-loops and duplicates
removed, no vertex permutation), greedy lowest-free colouring in vertex-id
order, then a sequence of update batches of 1,000,000 lines each, 50%
deletions of existing edges (uniform over edges, so their endpoints follow
the R-MAT distribution) and 50% insertions of absent pairs with R-MAT
endpoints.  One step = one batch through apply-update-batch
(structural update + seeding + recolouring loop).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--variant hi|hb]
    python bench.py --impl reference ...   # the reference's own code on the CPU

N > 1 runs N independent replicas (the path does not shard a single graph),
one process per GPU under torch.distributed; value is the sum over replicas
divided by the slowest replica's device time.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-updates/sec"
UNIT = "edge-updates/s"
HBM_FALLBACK_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--variant", choices=["hi", "hb"], default="hi")
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edgefactor", type=int, default=16)
    ap.add_argument("--batch", type=int, default=1_000_000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle replay of the first batch (the parity check and the CPU baseline)")
    ap.add_argument("--no-further-configs", action="store_true",
                    help="skip the other single-graph configurations reported under detail.configs")
    ap.add_argument("--cl-vertices", type=int, default=4_000_000, help="skewed-degree configuration: vertices")
    ap.add_argument("--cl-max-deg", type=float, default=360_000.0,
                    help="skewed-degree configuration: Chung-Lu weight of the largest vertex")
    ap.add_argument("--ref-iter-cap", type=int, default=2000)
    ap.add_argument("--ref-sample", type=int, default=1_000,
                    help="reference arm: change lines of each step's bounded sample")
    ap.add_argument("--ref-step-budget-ms", type=float, default=20_000.0,
                    help="reference arm: a step's loop stops once its timed work passes this budget")
    ap.add_argument("--ref-max-fail", type=int, default=3,
                    help="reference arm: stop after this many unconverged steps in a row")
    ap.add_argument("--unit-slots", type=int, default=0, help="adjacency slots per warp work unit (0: library default)")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="persistent CTAs per SM (0: from occupancy)")
    ap.add_argument("--heavy-min-live", type=int, default=0,
                    help="HI: live slots from which a row is indexed by colour (0: library default, <0: off)")
    ap.add_argument("--mode", choices=["plain", "batched", "served"], default="plain",
                    help="plain: one large graph (headline); batched: many graphs in one launch; "
                         "served: request stream over resident graphs")
    ap.add_argument("--graphs", type=int, default=4096, help="batched mode: number of graphs")
    ap.add_argument("--default-batched-graphs", type=int, default=512,
                    help="plain mode: graphs of the short batched comparison under detail.batched (0: none)")
    ap.add_argument("--served-graphs", type=int, default=256, help="served mode: resident graphs")
    ap.add_argument("--served-smin", type=int, default=14, help="served mode: smallest graph scale")
    ap.add_argument("--served-smax", type=int, default=20, help="served mode: largest graph scale")
    ap.add_argument("--requests", type=int, default=1000, help="served mode: requests per run")
    ap.add_argument("--loads", default="1000,10000,50000", help="served mode: offered loads, requests/s")
    ap.add_argument("--budget-frac", type=float, default=0.5,
                    help="served mode: device row and vertex budget as a fraction of the total graph state")
    ap.add_argument("--max-lines", type=int, default=1 << 22, help="served mode: lines per shared launch")
    ap.add_argument("--policies", default="plain,batched,lanes",
                    help="served mode: plain (one batch per launch), batched (continuous batching in one pool), "
                         "lanes (continuous batching in --lanes pools side by side)")
    ap.add_argument("--lanes", type=int, default=4, help="served mode: pools that run side by side")
    ap.add_argument("--pool-heavy-min-live", type=int, default=0,
                    help="served mode: the pools' heavy-row index threshold (<= 0: off, the library default)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only; no collective on the data path)
# ---------------------------------------------------------------------------

class Dist:
    """One process per GPU (torchrun env).  NCCL on GPUs; gloo with CPU
    tensors where no GPU is visible (the multi-process host logic)."""

    def __init__(self, want_gpus: int, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False
        self.dev = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as tdist

            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            timeout = datetime.timedelta(minutes=10)
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.dev = torch.device("cuda", self.local)
                tdist.init_process_group("nccl", timeout=timeout, device_id=self.dev)
            else:
                self.dev = torch.device("cpu")
                tdist.init_process_group("gloo", timeout=timeout)
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as tdist

            tdist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch
        import torch.distributed as tdist

        t = torch.tensor([x], dtype=torch.float64, device=self.dev)
        tdist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch.distributed as tdist

        return self._reduce(x, tdist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch.distributed as tdist

        return self._reduce(x, tdist.ReduceOp.SUM)

    def close(self):
        if self.pg:
            import torch.distributed as tdist

            tdist.destroy_process_group()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def workload_dir(args, dist: Dist) -> str:
    port = os.environ.get("MASTER_PORT", "0")
    return os.path.join("/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir(),
                        f"dcbench_{args.scale}_{args.edgefactor}_{args.batch}_{args.seed}_{port}_{os.getppid() if dist.world > 1 else os.getpid()}")


class _ProductGen:
    """Workload generators of the product library (libdyncolor.so)."""

    def __init__(self):
        import dyncolor_b200 as dc

        self.rmat = lambda scale, m, seed: dc.rmat(scale, m, seed=seed)
        self.chung_lu = lambda n, g, avg, mx, seed: dc.chung_lu(n, g, avg, mx, seed=seed)
        self.dedup = dc.dedup
        self.greedy_color = dc.greedy_color
        self.EdgeSet = dc.EdgeSet
        self.INS_RMAT, self.INS_DEGREE = dc.INS_RMAT, dc.INS_DEGREE


class _CheckerGen:
    """The same generators compiled into the checker library (liboracle.so),
    for the reference arm, which must not load libdyncolor.so."""

    def __init__(self):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po

        self.rmat = lambda scale, m, seed: po.gen_rmat(scale, m, seed=seed)
        self.chung_lu = lambda n, g, avg, mx, seed: po.gen_chung_lu(n, g, avg, mx, seed=seed)
        self.dedup = po.gen_dedup
        self.greedy_color = po.gen_greedy_color
        self.EdgeSet = po.GenEdgeSet
        self.INS_RMAT, self.INS_DEGREE = po.INS_RMAT, po.INS_DEGREE


def build_workload(args, nbatches: int, gen=None):
    gen = gen or _ProductGen()
    n = 1 << args.scale
    t0 = time.time()
    a, b = gen.rmat(args.scale, args.edgefactor * n, args.seed)
    a, b = gen.dedup(n, a, b)
    colors = gen.greedy_color(n, a, b)
    es = gen.EdgeSet(n, a, b)
    half = args.batch // 2
    batches = [es.sample_batch(half, args.batch - half, mode=gen.INS_RMAT, scale=args.scale,
                               seed=args.seed * 1000 + i) for i in range(nbatches)]
    return {"n": n, "a": a, "b": b, "colors": colors, "batches": batches,
            "gen_s": time.time() - t0}


def get_workload(args, dist: Dist, nbatches: int):
    """Rank 0 builds the workload; other ranks load it from shared memory."""
    if dist.world == 1:
        return build_workload(args, nbatches)
    d = workload_dir(args, dist)
    if dist.rank == 0:
        w = build_workload(args, nbatches)
        os.makedirs(d, exist_ok=True)
        np.save(os.path.join(d, "a.npy"), w["a"])
        np.save(os.path.join(d, "b.npy"), w["b"])
        np.save(os.path.join(d, "colors.npy"), w["colors"])
        np.save(os.path.join(d, "batches.npy"), np.stack(w["batches"]))
    dist.barrier()
    if dist.rank != 0:
        w = {"n": 1 << args.scale, "a": np.load(os.path.join(d, "a.npy")),
             "b": np.load(os.path.join(d, "b.npy")), "colors": np.load(os.path.join(d, "colors.npy")),
             "gen_s": 0.0}
        w["batches"] = list(np.load(os.path.join(d, "batches.npy")))
    dist.barrier()
    if dist.rank == 0:
        shutil.rmtree(d, ignore_errors=True)
    return w


def config(args, w) -> dict:
    return {
        "workload": (f"rmat{args.scale}-ef{args.edgefactor} update batches of {args.batch} lines "
                     f"(50% deletions of existing edges / 50% insertions of absent R-MAT pairs), "
                     f"variant {args.variant.upper()}"),
        "graph": {"vertices": int(w["n"]), "edges": int(len(w["a"])), "generator": "R-MAT a=0.57 b=c=0.19",
                  "initial_colors": int(w["colors"].max()) + 1, "seed": args.seed},
        "batch_lines": args.batch,
        "variant": args.variant.upper(),
        "l2": "inputs larger than L2 (adjacency >= 2 GB per replica); no flush",
        "parallelism": "replicas",
    }


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(
            ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
             "-lms", "200", "-i", str(self.device)],
            stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# DRAM bytes (read + write) per covered adjacency entry of the recolour
# launch, from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum,
# one pass) of this bench's workloads; keyed by (variant, scale, edge factor,
# lines).  The summary that each figure comes from is in profiles/.
MEASURED_DRAM_BYTES_PER_ENTRY = {("hi", 24, 16, 1_000_000): 1.285, ("hi", 22, 16, 250_000): 1.127}


def load_traffic(variant: str, scale: int, ef: int, lines: int):
    """Measured DRAM bytes per covered entry for this workload, or None."""
    return MEASURED_DRAM_BYTES_PER_ENTRY.get((variant, scale, ef, lines))


def roofline_of(stats, K, hi: bool, k_lines: int, traffic_per_entry=None) -> dict:
    """Roofline of the dominant kernel over K batches (SURVEY-style
    algorithmic bytes: 8 B per covered adjacency entry for HI, 12 B for HB;
    16 B per line for the structural kernel)."""
    rec_ms = sum(s.recolor_ms for s in stats)
    str_ms = sum(s.struct_ms for s in stats)
    scanned = sum(s.slots_scanned for s in stats)
    per_slot = 8 if hi else 12  # adjacency id + neighbour colour (+ priority)
    peak, peak_kind = hbm_peak()
    if rec_ms >= str_ms:
        dom, dom_ms, alg = "recolor_kernel", rec_ms, per_slot * scanned
    else:
        dom, dom_ms, alg = "struct_kernel", str_ms, 16 * 2 * k_lines * K
    achieved = alg / (dom_ms / 1e3) / 1e9
    traffic = traffic_per_entry * scanned / K if traffic_per_entry and dom == "recolor_kernel" else None
    out = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
           "algorithmic_bytes_per_launch": alg / K,
           "entries_covered_per_launch": scanned / K,
           "entries_read_per_launch": sum(s.slots_read for s in stats) / K,
           "note": f"{per_slot} B per covered adjacency entry (id + neighbour colour"
                   + ("" if hi else " + priority") + "), covered entries counted on the device"}
    if traffic is not None:
        # measured DRAM bytes of a launch over its duration, against the peak
        out["dram_gbs"] = traffic / (dom_ms / K / 1e3) / 1e9
        out["dram_frac"] = out["dram_gbs"] / peak
    return out


def measure_batches(ctx, dbat, k, W, K, stream):
    """W untimed batches, then K timed ones (CUDA events on the library's
    stream); returns (ms, per-batch stats)."""
    import torch

    for i in range(W):
        ctx.apply_batch_device(dbat[i].data_ptr(), k)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [ctx.apply_batch_device(dbat[W + i].data_ptr(), k) for i in range(K)]
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), stats


# ---------------------------------------------------------------------------
# CPU baseline and oracle check (checker code under oracle/, used only here)
# ---------------------------------------------------------------------------

def oracle_first_batch(args, w, gpu_colors, gpu_stats) -> tuple[dict, dict]:
    """Replays the first batch of the headline sequence (applied to the
    initial graph) on the C oracle with every host thread, compares its
    colours and step counts with the GPU's, and reports the same run as the
    CPU baseline."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    threads = os.cpu_count() or 1
    po.set_threads(threads)
    t0 = time.perf_counter()
    g = po.Graph(w["n"])
    g.load_edges(w["a"], w["b"])
    g.set_colors(w["colors"])
    load_s = time.perf_counter() - t0
    ch = w["batches"][0]
    och = np.empty(len(ch), dtype=po.CHANGE_DTYPE)
    for f in ("node1", "node2", "inst"):
        och[f] = ch[f]
    t0 = time.perf_counter()
    rc, st = g.apply_batch(och, po.HI if args.variant == "hi" else po.HB, po.SNAPSHOT)
    dt = time.perf_counter() - t0
    oc = g.colors()
    diff = int(np.count_nonzero(oc != gpu_colors))
    check = {
        "batch": "first batch of the sequence, applied to the initial graph",
        "lines": int(len(och)), "oracle_status": int(rc),
        "colors_identical": diff == 0, "colors_differing": diff,
        "iterations_gpu": int(gpu_stats.iterations), "iterations_oracle": int(st.iterations),
        "frontier_total_equal": int(gpu_stats.frontier_total) == int(st.frontier_total),
        "entries_covered_equal": int(gpu_stats.slots_scanned) == int(st.slots_scanned),
        "max_color_gpu": int(gpu_colors.max()), "max_color_oracle": int(st.max_color),
        "oracle_conflicts": int(g.conflicts()),
    }
    check["bit_exact"] = (diff == 0 and check["iterations_gpu"] == check["iterations_oracle"]
                          and check["frontier_total_equal"] and check["entries_covered_equal"])
    base = {"value": len(och) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"one full batch ({len(och)} lines, the first of the sequence) applied to the "
                       f"initial graph by the C oracle (snapshot schedule, {threads} OpenMP threads): "
                       f"{dt:.1f} s, {st.iterations} iterations; graph load {load_s:.1f} s not timed")}
    return check, base


def run_reference(args, dist) -> dict:
    """The reference's own kernel bodies on the host cores (oracle/_ref),
    every kernel launched on all host threads.  The inputs come from the
    generators compiled into the checker library, so this arm never loads
    libdyncolor.so.  Only steps whose recolouring converged count."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_hi" if args.variant == "hi" else "ref_hb")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "oracle/_ref harness not built (reference sources absent at build time)"}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    threads = os.cpu_count() or 1
    nb = args.warmup + args.steps
    w = build_workload(args, nb, gen=_CheckerGen())
    d = tempfile.mkdtemp()
    try:
        np.stack([w["a"], w["b"]], 1).astype(np.int32).tofile(os.path.join(d, "g.bin"))
        w["colors"].astype(np.int32).tofile(os.path.join(d, "c.bin"))
        files = []
        for i in range(nb):
            f = os.path.join(d, f"x{i}.txt")
            po.write_change_file(f, w["batches"][i][: args.ref_sample])
            files.append(f)
        out = os.path.join(d, "o.txt")
        subprocess.run([exe, "bench", os.path.join(d, "g.bin"), str(w["n"]), str(len(w["a"])),
                        os.path.join(d, "c.bin"), ",".join(files), out, str(args.ref_iter_cap),
                        str(args.ref_step_budget_ms), str(args.ref_max_fail), str(threads)],
                       check=True, stdout=subprocess.DEVNULL)
        rows = [line.split() for line in open(out)]
    finally:
        shutil.rmtree(d, ignore_errors=True)
    its = [int(r[1]) for r in rows]
    conv = [r for r in rows[args.warmup:] if r[3] == "0"]
    how = (f"first {args.ref_sample} lines of each batch, each applied to the initial graph by the "
           f"reference's own kernel bodies, every kernel launched on {threads} host threads; step budget "
           f"{args.ref_step_budget_ms / 1e3:.0f} s or {args.ref_iter_cap} iterations")
    if not conv:
        return {"impl": "reference", "unavailable": (
            f"the reference's recolouring converged on none of the {len(rows)} steps run ({how}; loop "
            f"iterations {its}; stopped after {args.ref_max_fail} unconverged steps in a row): its 32-bit "
            f"saturation masks are exact only for colours <= 30 and this graph starts with "
            f"{int(w['colors'].max()) + 1} colours")}
    ms = sum(float(r[5]) for r in conv)
    lines = args.ref_sample * len(conv)
    value = lines / (ms / 1e3)
    sample = f"{how}; {len(conv)} timed steps converged and count (loop iterations of all steps {its})"
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / len(conv),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic", "config": config(args, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def sub_result(name, desc, ctx_args, n, a, b, colors, batches, W, K, hi, dev, stream, graph_desc,
               traffic=None) -> dict:
    """One further configuration: fresh context, W untimed and K timed
    batches, device time, roofline, and a properness check."""
    import torch

    import dyncolor_b200 as dc

    ctx = dc.Context(variant=dc.HI if hi else dc.HB, device=dev, stream=stream.cuda_stream, **ctx_args)
    ctx.load_edges(n, a, b)
    ctx.set_colors(colors)
    k = len(batches[0])
    dbat = [torch.from_numpy(np.ascontiguousarray(x).view(np.int32).reshape(-1, 3)).to(f"cuda:{dev}")
            for x in batches[: W + K]]
    ms, stats = measure_batches(ctx, dbat, k, W, K, stream)
    conflicts = ctx.validate()
    ctx.close()
    del dbat
    return {
        "name": name, "workload": desc, "graph": graph_desc, "variant": "HI" if hi else "HB",
        "batch_lines": k, "warmup": W, "steps": K,
        "value": K * k / (ms / 1e3), "unit": UNIT, "ms_per_batch": ms / K,
        "iterations_per_batch": [int(s.iterations) for s in stats],
        "recolor_ms_per_batch": sum(s.recolor_ms for s in stats) / K,
        "struct_ms_per_batch": sum(s.struct_ms for s in stats) / K,
        "roofline": roofline_of(stats, K, hi, k, traffic),
        "max_color": int(max(s.max_color for s in stats)),
        "conflicts_after": int(conflicts),
    }


def run_further_configs(args, w, dev, stream) -> list:
    """The other single-graph configurations: the headline graph with 100 k
    and 10 M-line batches and with the HB variant, and the skewed-degree
    Chung-Lu graph (both variants)."""
    import dyncolor_b200 as dc

    out = []
    n, a, b, col = w["n"], w["a"], w["b"], w["colors"]
    gd = {"vertices": int(n), "edges": int(len(a)), "generator": "R-MAT a=0.57 b=c=0.19",
          "initial_colors": int(col.max()) + 1}
    ctx_args = dict(unit_slots=args.unit_slots, blocks_per_sm=args.blocks_per_sm,
                    heavy_min_live=args.heavy_min_live)
    for lines, W, K in ((100_000, 2, 5), (10_000_000, 1, 2)):
        es = dc.EdgeSet(n, a, b)
        bs = [es.sample_batch(lines // 2, lines - lines // 2, mode=dc.INS_RMAT, scale=args.scale,
                              seed=args.seed * 7000 + lines // 1000 + i) for i in range(W + K)]
        del es
        out.append(sub_result(f"rmat{args.scale}_b{lines}_hi",
                              f"rmat{args.scale}-ef{args.edgefactor}, batches of {lines} lines in sequence "
                              f"(50/50, R-MAT endpoints)", ctx_args, n, a, b, col, bs, W, K, True, dev, stream,
                              gd, load_traffic("hi", args.scale, args.edgefactor, lines)))
    out.append(sub_result(f"rmat{args.scale}_b{args.batch}_hb",
                          f"rmat{args.scale}-ef{args.edgefactor}, batches of {args.batch} lines in sequence "
                          f"(the headline batches), variant HB", ctx_args, n, a, b, col, w["batches"], 1, 2, False,
                          dev, stream, gd, load_traffic("hb", args.scale, args.edgefactor, args.batch)))
    # skewed degrees: Chung-Lu, exponent 2.1, 4 M vertices, average degree 24
    cn = args.cl_vertices
    t0 = time.time()
    ca, cb = dc.chung_lu(cn, 2.1, 24.0, args.cl_max_deg, seed=args.seed + 3)
    ca, cb = dc.dedup(cn, ca, cb)
    ccol = dc.greedy_color(cn, ca, cb)
    deg = np.bincount(ca, minlength=cn) + np.bincount(cb, minlength=cn)
    es = dc.EdgeSet(cn, ca, cb)
    kd = int(0.3 * args.batch)
    cbs = [es.sample_batch(kd, args.batch - kd, mode=dc.INS_DEGREE, seed=args.seed * 9000 + i) for i in range(4)]
    del es
    cgd = {"vertices": int(cn), "edges": int(len(ca)), "generator": "Chung-Lu gamma=2.1 avg degree 24",
           "max_degree": int(deg.max()), "initial_colors": int(ccol.max()) + 1,
           "gen_s": round(time.time() - t0, 1)}
    for hi, W, K in ((True, 1, 3), (False, 1, 2)):
        out.append(sub_result(f"chunglu_{cn}_b{args.batch}_{'hi' if hi else 'hb'}",
                              f"Chung-Lu (gamma 2.1) {cn} vertices, batches of {args.batch} lines in sequence "
                              f"(70% insertions with one endpoint drawn by degree, 30% deletions)",
                              ctx_args, cn, ca, cb, ccol, cbs, W, K, hi, dev, stream, cgd))
    return out


def run_ours(args, dist: Dist):
    import torch

    import dyncolor_b200 as dc

    dev = dist.local
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup
    w = get_workload(args, dist, W + 2 * K)
    variant = dc.HI if args.variant == "hi" else dc.HB
    stream = torch.cuda.Stream(device=dev)
    ctx = dc.Context(variant=variant, device=dev, stream=stream.cuda_stream, unit_slots=args.unit_slots,
                     blocks_per_sm=args.blocks_per_sm, heavy_min_live=args.heavy_min_live)
    t0 = time.time()
    ctx.load_edges(w["n"], w["a"], w["b"])
    ctx.set_colors(w["colors"])
    load_s = time.time() - t0
    k = args.batch
    # device-resident inputs for the kernel-time measurement
    dbat = [torch.from_numpy(np.ascontiguousarray(x).view(np.int32).reshape(-1, 3)).to(f"cuda:{dev}")
            for x in w["batches"][: W + K]]
    torch.cuda.synchronize()
    # the first warm-up batch's colours are kept for the oracle check
    first_stats = ctx.apply_batch_device(dbat[0].data_ptr(), k)
    first_colors = ctx.colors().copy() if dist.rank == 0 else None
    for i in range(1, W):
        ctx.apply_batch_device(dbat[i].data_ptr(), k)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = []
    for i in range(K):
        stats.append(ctx.apply_batch_device(dbat[W + i].data_ptr(), k))
    e1.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    ms = dist.max(ms_local)
    total_updates = dist.sum(float(K * k))
    value = total_updates / (ms / 1e3)
    # end to end: pinned host lines in, full colour array out, every step
    host = [torch.from_numpy(np.ascontiguousarray(x).view(np.int32).reshape(-1)).pin_memory()
            for x in w["batches"][W + K: W + 2 * K]]
    colors_out = torch.empty(w["n"], dtype=torch.int32).pin_memory()
    cnp = colors_out.numpy()
    torch.cuda.synchronize()
    dist.barrier()
    t0 = time.perf_counter()
    for i in range(K):
        ctx.apply_batch(host[i].numpy().view(dc.CHANGE_DTYPE))
        ctx.colors(out=cnp)
    torch.cuda.synchronize()
    e2e_s = dist.max(time.perf_counter() - t0)
    conflicts = ctx.validate()
    ctx.close()
    del dbat
    torch.cuda.empty_cache()
    roof = roofline_of(stats, K, variant == dc.HI, k, load_traffic(args.variant, args.scale, args.edgefactor, k))
    out = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": dist.world,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic",
        "config": config(args, w),
        "e2e": {"value": total_updates / e2e_s if e2e_s > 0 else None, "unit": UNIT,
                "h2d_bytes_per_step": 12 * k, "d2h_bytes_per_step": 4 * int(w["n"])},
        # per batch: structural + recolour launches, and the four heavy-row
        # index kernels when the batch uses the index (lines * 256 >= n)
        "gpu_launches": (6 if args.heavy_min_live >= 0 and k * 256 >= int(w["n"]) else 2) * K,
        "roofline": roof,
        "clocks": clk,
        "detail": {
            "iterations_per_batch": [int(s.iterations) for s in stats],
            "struct_ms_per_batch": sum(s.struct_ms for s in stats) / K,
            "recolor_ms_per_batch": sum(s.recolor_ms for s in stats) / K,
            "phase_ms_per_batch": {nm: round(sum(s.phase_ms[i] for s in stats) / K, 3)
                                   for i, nm in enumerate(("seeding", "find_eligible", "mex", "commit"))},
            "slots_scanned_per_batch": sum(s.slots_scanned for s in stats) / K,
            "slots_read_per_batch": sum(s.slots_read for s in stats) / K,
            "max_color": int(max(s.max_color for s in stats)),
            "conflicts_after": int(conflicts),
            "workload_gen_s": round(w["gen_s"], 1),
            "load_s": round(load_s, 2),
        },
    }
    if dist.world == 1 and not args.no_further_configs:
        t0 = time.time()
        out["detail"]["configs"] = run_further_configs(args, w, dev, stream)
        out["detail"]["configs_s"] = round(time.time() - t0, 1)
        if args.default_batched_graphs > 0:
            # the batched configuration, shortened: graphs in one launch
            # against each graph alone, every graph's colours compared
            t0 = time.time()
            b = run_batched(args, dist, count=args.default_batched_graphs, tune=False)
            out["detail"]["batched"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "e2e",
                                                           "plain_each_graph_alone", "speedup_vs_plain",
                                                           "bit_exact_vs_alone", "graphs_differing", "config")}
            out["detail"]["batched_s"] = round(time.time() - t0, 1)
    return out, w, first_colors, first_stats


# ---------------------------------------------------------------------------
# batched mode: thousands of independent graphs, one launch per update round
# ---------------------------------------------------------------------------

def build_batched_workload(count, seed, nmin=1_000, nmax=200_000, kmin=100, kmax=50_000, rank=0, world=1):
    """Graphs with vertex counts log-uniform in [nmin, nmax], average degree
    uniform in [8, 32], R-MAT or Erdos-Renyi (alternating), greedy colouring;
    one batch per graph of log-uniform size in [kmin, kmax], half deletions of
    existing edges, half insertions of absent pairs.  With world > 1 only the
    graphs i with i % world == rank are built (whole graphs per GPU)."""
    import dyncolor_b200 as dc

    from concurrent.futures import ThreadPoolExecutor

    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(np.int64)
    degs = rng.uniform(8, 32, count)
    ks = np.exp(rng.uniform(np.log(kmin), np.log(kmax), count)).astype(np.int64)

    def one(i):
        n, m, k = int(ns[i]), int(ns[i] * degs[i] / 2), int(ks[i])
        if i % 2 == 0:
            a, b = dc.rmat(int(np.ceil(np.log2(n))), m, seed=seed * 100_003 + i, n=n)
        else:
            a, b = dc.uniform_pairs(n, m, seed=seed * 100_003 + i)
        a, b = dc.dedup(n, a, b)
        c = dc.greedy_color(n, a, b)
        es = dc.EdgeSet(n, a, b)
        kd = min(k // 2, len(a))
        x = es.sample_batch(kd, k - kd, seed=seed * 7 + i)
        return (n, a, b), c, x

    # the generators release the GIL (ctypes), so host threads overlap them
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        out = list(ex.map(one, range(rank, count, world)))
    return [o[0] for o in out], [o[1] for o in out], [o[2] for o in out]


def run_batched(args, dist, count=None, tune=True):
    """Batched mode: `count` graphs (default --graphs) in one launch sequence
    against each graph alone.  tune=False keeps the library's tile defaults
    (the short comparison the default run reports under detail.batched)."""
    import dyncolor_b200 as dc
    from dyncolor_b200.batched import BatchedContext
    from dyncolor_b200.tune import autotune

    count = args.graphs if count is None else count
    variant = dc.HI if args.variant == "hi" else dc.HB
    t0 = time.time()
    import torch

    torch.cuda.set_device(dist.local)
    dev = dist.local
    # whole graphs per GPU: rank r takes graphs r, r + N, ...
    graphs, colors, batches = build_batched_workload(count, args.seed, rank=dist.rank, world=dist.world)
    gen_s = time.time() - t0
    lines = int(sum(len(x) for x in batches))
    best, table = {}, {}
    if tune:
        # autotune the tile parameters on a sample of the graphs
        rng = np.random.default_rng(args.seed + 1)
        idx = sorted(rng.choice(len(graphs), min(256, len(graphs)), replace=False).tolist())
        sg, sc, sb = [graphs[i] for i in idx], [colors[i] for i in idx], [batches[i] for i in idx]

        def make(opts):
            bc = BatchedContext(variant=variant, device=dev, **opts)
            bc.load(sg)
            bc.set_colors(sc)
            return bc

        best, table = autotune(make, lambda bc: bc.apply(sb).device_ms)
    # all graphs, one launch (replayed from a captured CUDA graph)
    bc = BatchedContext(variant=variant, device=dev, cuda_graph=True, **best)
    bc.load(graphs)
    bc.set_colors(colors)
    ub = bc.union_batch(batches)
    dist.barrier()
    t0 = time.perf_counter()
    st = bc.ctx.apply_batch(ub)
    got = bc.ctx.colors()
    e2e_b = dist.max(time.perf_counter() - t0)
    dev_b = dist.max(st.device_ms)
    its_b = bc.iterations()
    first = bc.first.copy()
    bc.close()
    # plain: each graph recoloured alone (its own context), one launch per batch
    dev_plain, e2e_p, its_p = 0.0, 0.0, []
    mismatched = 0
    for g, ((n, a, b), c0, x) in enumerate(zip(graphs, colors, batches)):
        pc = dc.Context(variant=variant, device=dev, **best)
        pc.load_edges(n, a, b)
        pc.set_colors(c0)
        t0 = time.perf_counter()
        s1 = pc.apply_batch(x)
        alone = pc.colors()
        e2e_p += time.perf_counter() - t0
        pc.close()
        dev_plain += s1.device_ms
        its_p.append(s1.iterations)
        if not np.array_equal(alone, got[first[g]:first[g + 1]]):
            mismatched += 1
    same_local = mismatched == 0 and bool(np.array_equal(its_b, np.array(its_p)))
    # every rank ran its own graphs at the same time: max of the times, sum of the work
    lines_all = int(dist.sum(float(lines)))
    mismatched = int(dist.sum(float(mismatched)))
    same = dist.sum(0.0 if same_local else 1.0) == 0.0
    dev_plain = dist.max(dev_plain)
    e2e_p = dist.max(e2e_p)
    nverts = int(dist.sum(float(first[-1])))
    nedges = int(dist.sum(float(sum(len(x) for _, x, _ in graphs))))
    value = lines_all / (dev_b / 1e3)
    plain = lines_all / (dev_plain / 1e3)
    lines = lines_all
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": 1, "warmup": 0,
        "ms_per_step": dev_b, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "int32", "data": "synthetic", "mode": "batched",
        "config": {"workload": (f"{count} independent graphs (vertices log-uniform in [1k, 200k], "
                                f"average degree uniform in [8, 32], R-MAT / Erdos-Renyi alternating), one "
                                f"batch per graph (log-uniform in [100, 50k] lines, 50/50), variant "
                                f"{args.variant.upper()}"),
                   "vertices": nverts, "edges": nedges, "lines": lines, "tuned": best, "cuda_graph": True,
                   "parallelism": f"whole graphs per GPU over {dist.world} GPU(s)"},
        "e2e": {"value": lines / e2e_b, "unit": UNIT, "h2d_bytes_per_step": 12 * lines,
                "d2h_bytes_per_step": 4 * nverts},
        "plain_each_graph_alone": {"value": plain, "e2e": lines / e2e_p, "launches": 2 * count,
                                   "device_ms": dev_plain},
        "speedup_vs_plain": value / plain,
        "bit_exact_vs_alone": same, "graphs_differing": mismatched,
        "detail": {"iterations_max": int(its_b.max()), "iterations_median": float(np.median(its_b)),
                   "tuning_ms": {f"unit_slots={k[1]},blocks_per_sm={k[0]}": round(v, 3)
                                 for k, v in table.items()},
                   "workload_gen_s": round(gen_s, 1)},
    }


# ---------------------------------------------------------------------------
# served mode: a request stream over resident graphs
# ---------------------------------------------------------------------------

def build_served_workload(args):
    """Graphs: two of every three from the R-MAT generator of the single-graph
    workloads (a=0.57, b=c=0.19, edgefactor 16), the third from the skewed
    Chung-Lu generator (exponent 2.1, average degree 24, maximum degree n/20),
    each with 2^s vertices, s uniform in [smin, smax], greedy initial colours.
    Requests: Poisson arrivals (unit rate here, scaled per offered load),
    targets Zipf(1.1), sizes log-uniform in [10, 1M] lines; each graph's
    requests are drawn in order from its evolving edge set with the batch
    rule of its generator's workload (R-MAT: half deletions, R-MAT endpoints;
    Chung-Lu: 30% deletions, one inserted endpoint by degree)."""
    from concurrent.futures import ThreadPoolExecutor

    import dyncolor_b200 as dc
    from dyncolor_b200.serve import make_trace

    G = args.served_graphs
    rng = np.random.default_rng(args.seed + 17)
    scales = rng.integers(args.served_smin, args.served_smax + 1, G)
    arrivals, targets, sizes = make_trace(args.requests, G, 1.0, args.seed)
    mine = [[] for _ in range(G)]
    for j, g in enumerate(targets):
        mine[int(g)].append(j)

    def one(i):
        s = int(scales[i])
        n = 1 << s
        seed = args.seed * 1_000_003 + i
        if i % 3 == 2:
            a, b = dc.chung_lu(n, 2.1, 24.0, n / 20.0, seed=seed)
        else:
            a, b = dc.rmat(s, 16 * n, seed=seed)
        a, b = dc.dedup(n, a, b)
        c = dc.greedy_color(n, a, b)
        lines = {}
        if mine[i]:
            es = dc.EdgeSet(n, a, b)
            alive = len(a)  # deletions are drawn from the original edges still present
            for r, j in enumerate(mine[i]):
                k = int(sizes[j])
                if i % 3 == 2:
                    kd = min(int(0.3 * k), alive)
                    x = es.sample_batch(kd, k - kd, mode=dc.INS_DEGREE, seed=seed * 31 + r)
                else:
                    kd = min(k // 2, alive)
                    x = es.sample_batch(kd, k - kd, mode=dc.INS_RMAT, scale=s, seed=seed * 31 + r)
                alive -= kd
                lines[j] = x
        return (n, a, b), c, lines

    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        out = list(ex.map(one, range(G)))
    graphs = [o[0] for o in out]
    colors = [o[1] for o in out]
    req_lines = [None] * len(targets)
    for o in out:
        for j, x in o[2].items():
            req_lines[j] = x
    return graphs, colors, arrivals, targets, req_lines, scales


def run_served(args):
    import dyncolor_b200 as dc
    from dyncolor_b200.pool import ResidentPool
    from dyncolor_b200.serve import LanedServer, Request, Server, assign_lanes

    variant = dc.HI if args.variant == "hi" else dc.HB
    t0 = time.time()
    graphs, colors, arrivals, targets, req_lines, scales = build_served_workload(args)
    gen_s = time.time() - t0
    nsum = sum(n for n, _, _ in graphs)
    nmax = max(n for n, _, _ in graphs)
    est_slots = sum(int(2.5 * len(a)) + 4 * n for n, a, _ in graphs)
    state_bytes = 4 * est_slots + 36 * nsum
    vcap = max(int(args.budget_frac * nsum), 2 * nmax)
    slots = max(int(args.budget_frac * est_slots), 4 * max(int(2.5 * len(a)) + 4 * n for n, a, _ in graphs))
    lines_total = int(sum(len(x) for x in req_lines))
    loads = [float(x) for x in args.loads.split(",") if x]
    runs, first_colors, first_its, exact = [], None, None, True
    policies = [x for x in args.policies.split(",") if x]
    sizes = [n for n, _, _ in graphs]

    def make_pools(policy):
        """[(pool, {graph: local id}, vertex capacity, slots)]: one pool with
        every graph, or one per lane with a share of the SMs and of the
        budget."""
        if policy != "lanes":
            pool = ResidentPool(variant=variant, vertex_capacity=vcap, pool_slots=slots, pool_slots_max=4 * slots,
                                max_graphs=len(graphs) + 1, cuda_graph=True,
                                heavy_min_live=args.pool_heavy_min_live)
            return [(pool, {g: g for g in range(len(graphs))}, vcap, slots)]
        nl = args.lanes
        which = assign_lanes(sizes, nl)
        import torch

        props = torch.cuda.get_device_properties(0)
        out = []
        for j in range(nl):
            gl = [g for g in range(len(graphs)) if which[g] == j]
            share = sum(sizes[g] for g in gl) / max(nsum, 1)
            # vertex ids are cheap next to rows: every graph of the lane keeps
            # its ids, and the row budget alone decides what spills
            lv = sum(sizes[g] for g in gl) + 2 * max(sizes[g] for g in gl)
            ls = max(int(slots * share * 1.2), 4 * max(int(2.5 * len(graphs[g][1])) + 4 * sizes[g] for g in gl))
            pool = ResidentPool(variant=variant, vertex_capacity=lv, pool_slots=ls, pool_slots_max=4 * ls,
                                max_graphs=len(gl) + 1, cuda_graph=True,
                                grid_ctas=max(1, 2 * props.multi_processor_count // nl),
                                heavy_min_live=args.pool_heavy_min_live)
            out.append((pool, {g: i for i, g in enumerate(gl)}, lv, ls))
        return out

    for rate in loads:
        for policy in policies:
            lanes = make_pools(policy)
            tb = time.time()
            for pool, gmap, _, _ in lanes:
                for g in sorted(gmap, key=lambda x: gmap[x]):
                    (n, a, b), c = graphs[g], colors[g]
                    pool.add_graph(n, a, b, c)
            build_s = time.time() - tb
            info0 = [pool.info() for pool, _, _, _ in lanes]
            reqs = [Request(j, int(targets[j]), req_lines[j], float(arrivals[j]) / rate)
                    for j in range(len(targets))]
            if policy == "lanes":
                st = LanedServer(lanes, max_lines=args.max_lines).run(reqs)
            else:
                st = Server(lanes[0][0], policy, vcap, slots, max_lines=args.max_lines).run(reqs)
            info1 = [pool.info() for pool, _, _, _ in lanes]
            fin = [None] * len(graphs)
            for pool, gmap, _, _ in lanes:
                for g, i in gmap.items():
                    fin[g] = pool.colors(i)
            its = np.array([r.iterations for r in sorted(reqs, key=lambda r: r.rid)])
            if first_colors is None:
                first_colors, first_its = fin, its
            else:
                exact = exact and all(np.array_equal(x, y) for x, y in zip(fin, first_colors)) \
                    and bool(np.array_equal(its, first_its))
            d = {k: sum(i1[k] - i0[k] for i0, i1 in zip(info0, info1))
                 for k in ("restores", "spills", "restore_ms", "spill_ms", "compact_ms", "compactions")}
            summ = st.summary(reqs)
            summ.update({
                "offered_req_per_s": rate, "policy": policy, "lanes": len(lanes), "pool_build_s": round(build_s, 2),
                "restores": d["restores"], "spills": d["spills"], "restore_ms": round(d["restore_ms"], 1),
                "spill_ms": round(d["spill_ms"], 1), "compact_ms": round(d["compact_ms"], 1),
                "compactions": d["compactions"],
                "device_gb": round(sum(i["device_bytes"] for i in info1) / 1e9, 2),
                "pinned_host_gb": round(sum(i["host_bytes"] for i in info1) / 1e9, 2),
            })
            runs.append(summ)
            for pool, _, _, _ in lanes:
                pool.close()
    top = [r for r in runs if r["offered_req_per_s"] == max(loads)]
    best = max(top, key=lambda r: (r["policy"] != "plain", r["updates_per_s"]))
    plain = next((r for r in top if r["policy"] == "plain"), best)
    return {
        "metric": METRIC, "value": best["updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": len(runs),
        "warmup": 0, "ms_per_step": best["makespan_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic", "mode": "served",
        "config": {"workload": (f"{len(graphs)} resident graphs (R-MAT ef16 and Chung-Lu 2.1, 2^s vertices, "
                                f"s in [{args.served_smin}, {args.served_smax}]), {len(targets)} requests, "
                                f"Poisson arrivals, Zipf(1.1) targets, log-uniform [10, 1M] lines, variant "
                                f"{args.variant.upper()}"),
                   "vertices": nsum, "edges": int(sum(len(a) for _, a, _ in graphs)), "lines": lines_total,
                   "graph_state_gb": round(state_bytes / 1e9, 2), "budget_frac": args.budget_frac,
                   "vertex_capacity": vcap, "pool_slots": slots, "max_lines_per_launch": args.max_lines},
        "e2e": {"value": best["updates_per_s"], "unit": UNIT,
                "h2d_bytes_per_step": 12 * lines_total, "d2h_bytes_per_step": 0},
        "plain_one_batch_per_launch": {"value": plain["updates_per_s"], "p50_ms": plain["p50_ms"],
                                       "p99_ms": plain["p99_ms"]},
        "best_policy": best["policy"],
        "p99_vs_plain": best["p99_ms"] / plain["p99_ms"] if plain["p99_ms"] else None,
        "speedup_vs_plain": best["updates_per_s"] / plain["updates_per_s"] if plain["updates_per_s"] else None,
        "bit_exact_across_policies": exact,
        "runs": runs,
        "detail": {"workload_gen_s": round(gen_s, 1), "scales": np.bincount(scales).tolist()},
    }


def main():
    args = parse_args()
    if args.mode == "batched":
        dist = Dist(args.gpus)
        try:
            out = run_batched(args, dist)
            if dist.rank == 0:
                print(json.dumps(out), flush=True)
        finally:
            dist.close()
        return
    if args.mode == "served":
        print(json.dumps(run_served(args)), flush=True)
        return
    if args.impl == "reference":
        # the reference has no GPU path here: rank 0 times it, other ranks exit
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(run_reference(args, _Solo(args.gpus))),
                  flush=True)
        return
    dist = Dist(args.gpus)
    try:
        out, w, first_colors, first_stats = run_ours(args, dist)
        if dist.rank == 0:
            if dist.world == 1 and not args.no_cpu_baseline:
                check, base = oracle_first_batch(args, w, first_colors, first_stats)
                out["detail"]["oracle_checked"] = check
                out["cpu_baseline"] = base
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


class _Solo:
    """World description for the reference arm (no process group)."""

    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", str(max(gpus, 1))))
        self.rank = 0


if __name__ == "__main__":
    main()

"""Command line with the reference drivers' argv (HI/Color_main.cu:21-37):

    python -m dyncolor_b200 <graph> <nodes> <edges> <prevColor> <changes>
        [--variant hi|hb] [--out colors.txt] [--device N]

``edges`` is advisory, as in the reference (it only sized an allocation).
Prints the phase times, the highest colour id used and the number of
monochromatic edges (the reference's validate kernel prints one line per
such edge).
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

from . import HB, HI, Context, io


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="dyncolor_b200")
    ap.add_argument("graph")
    ap.add_argument("nodes", type=int)
    ap.add_argument("edges", type=int)
    ap.add_argument("prev_color")
    ap.add_argument("changes")
    ap.add_argument("--variant", choices=["hi", "hb"], default="hi")
    ap.add_argument("--out", default=None)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)

    t0 = time.perf_counter()
    a, b = io.read_graph(args.graph)
    t1 = time.perf_counter()
    print(f"Time taken to read input graph: {int((t1 - t0) * 1e6)} microseconds")
    colors = io.read_colors(args.prev_color, args.nodes)
    print(f"Max color id in input graph: {int(colors.max(initial=-1))}")
    t2 = time.perf_counter()
    ch = io.read_changes(args.changes)
    t3 = time.perf_counter()
    print(f"Reading input changed edges data completed. totalInsertion:{int((ch['inst'] == 1).sum())}")
    print(f"Time taken to read input changed edges: {int((t3 - t2) * 1e6)} microseconds")

    ctx = Context(variant=HB if args.variant == "hb" else HI, device=args.device)
    t4 = time.perf_counter()
    ctx.load_edges(args.nodes, a, b)
    ctx.set_colors(colors)
    t5 = time.perf_counter()
    print(f"**Time taken to transfer graph data from CPU to GPU: {(t5 - t4) * 1e3:.3f} milliseconds**")
    st = ctx.apply_batch(ch)
    print(f"****Total Time for Vertex Color Update: {st.device_ms:.3f} milliseconds****"
          f" (iterations {st.iterations})")
    out = ctx.colors()
    print(f"highest color id used: {int(out.max(initial=-1))}")
    bad = ctx.validate()
    if bad:
        print(f"##Error found: {bad} monochromatic edges")
    if args.out:
        io.write_colors(args.out, out)
    return 0 if bad == 0 else 1


if __name__ == "__main__":
    sys.exit(main())

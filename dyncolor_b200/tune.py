"""Autotuner for the recolouring launches.

Picks the runtime tile parameters (slots per warp work unit, persistent CTAs
per SM) for a workload by timing each candidate on a tuning sample: the
caller provides ``make`` (options -> a ready context) and ``run`` (context ->
device milliseconds of one representative batch).  A fresh context per
candidate keeps the sample's starting state identical.
"""
from __future__ import annotations

import itertools
import math

DEFAULT_SPACE = {
    "unit_slots": (512, 1024, 2048, 4096),
    "blocks_per_sm": (1, 2),
}


def autotune(make, run, space=None, repeats: int = 1):
    """Returns (best options, {options tuple: best ms}) over the grid `space`."""
    space = space or DEFAULT_SPACE
    keys = sorted(space)
    results = {}
    best, best_ms = None, math.inf
    for combo in itertools.product(*(space[k] for k in keys)):
        opts = dict(zip(keys, combo))
        ms = math.inf
        for _ in range(repeats):
            ctx = make(opts)
            try:
                ms = min(ms, float(run(ctx)))
            finally:
                ctx.close()
        results[combo] = ms
        if ms < best_ms:
            best, best_ms = opts, ms
    return best, results

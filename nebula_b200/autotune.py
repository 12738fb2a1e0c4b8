"""Autotuner for the batched persistent kernel.

Picks the pool capacity, block size, refill threshold and walk cell budget
(leaf cells an octree walk takes per wavefront iteration) of ``nb.Batch`` for
a given set of jobs by timing runs on a bounded sample of the batch (every
job cut to ``sample_scale`` of its primaries, so the energy and geometry mix
is kept).  Search: coordinate descent from a start point -- capacity first
(it sets the population and the spill traffic), then block size, then the
refill threshold, then the walk budget -- and optionally a second pass; each point is timed as the
best of ``repeats`` runs after one warm-up run, with CUDA events on the
launch (``Batch.kernel_ms``).

Defaults sweep the ranges of the mixed-batch workload: capacity 2^18..2^24,
block 128..512, refill threshold 10..50 % (and 100 %, the plain refill rule),
walk budget 1, 2 or 4 cells.
"""
from __future__ import annotations

import json
import math

import numpy as np

from .api import Batch

CAPACITIES = tuple(1 << k for k in range(18, 25))
BLOCKS = (128, 256, 512)
THRESHOLDS = (0.1, 0.2, 0.3, 0.5, 1.0)
WALK_CELLS = (1, 2, 4)


def sample_jobs(jobs, scale):
    """Each job cut to ceil(scale * n) primaries (at least one)."""
    out = []
    for gi, seed, pri in jobs:
        n = max(1, int(math.ceil(len(pri) * scale)))
        out.append((gi, seed, pri[:n]))
    return out


def time_config(geoms, mats, jobs, capacity, block, threshold, walk_cells=1, repeats=2, queue_factor=4, device=0):
    """Best kernel time (ms) of ``repeats`` runs after a warm-up run."""
    b = Batch(geoms, mats, capacity=capacity, block_size=block, refill_threshold=threshold,
              queue_factor=queue_factor, device=device, walk_cells=walk_cells)
    try:
        b.set_jobs(jobs)
        b.run()
        best = math.inf
        for _ in range(repeats):
            b.run()
            best = min(best, b.kernel_ms())
        return best
    finally:
        b.close()


def tune_batch(geoms, mats, jobs, capacities=CAPACITIES, blocks=BLOCKS, thresholds=THRESHOLDS,
               walk_cells=WALK_CELLS, sample_scale=0.1, repeats=2, passes=1, start=(1 << 20, 256, 1.0, 1),
               device=0, log=None, timer=None):
    """Coordinate descent over (capacity, block, threshold, walk cells).
    Returns (best dict, list of every timed point).  ``timer(cap, blk, thr,
    cells) -> ms`` replaces the GPU timing (used to test the search)."""
    sample = sample_jobs(jobs, sample_scale)
    n_pri = sum(len(p) for _, _, p in sample)
    cache = {}
    table = []

    def measure(cap, blk, thr, cells):
        key = (cap, blk, thr, cells)
        if key not in cache:
            ms = (timer(cap, blk, thr, cells) if timer else
                  time_config(geoms, mats, sample, cap, blk, thr, cells, repeats=repeats, device=device))
            cache[key] = ms
            row = dict(capacity=cap, block=blk, threshold=thr, walk_cells=cells, ms=ms,
                       primaries_per_s=n_pri / (ms / 1e3))
            table.append(row)
            if log:
                log(row)
        return cache[key]

    cap, blk, thr, cells = start
    for _ in range(passes):
        cap = min(capacities, key=lambda c: measure(c, blk, thr, cells))
        blk = min(blocks, key=lambda b: measure(cap, b, thr, cells))
        thr = min(thresholds, key=lambda t: measure(cap, blk, t, cells))
        cells = min(walk_cells, key=lambda w: measure(cap, blk, thr, w))
    best = dict(capacity=cap, block=blk, threshold=thr, walk_cells=cells, ms=cache[(cap, blk, thr, cells)],
                sample_scale=sample_scale, sample_primaries=n_pri)
    return best, table


def save(path, best, table):
    with open(path, "w") as f:
        json.dump({"best": best, "points": table}, f, indent=1)


def load(path):
    with open(path) as f:
        return json.load(f)["best"]

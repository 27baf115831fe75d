"""Launch-shape tuning of multi-grid batches (mt3d_fwdsolve_multi).

The FP32 stencil kernels give each block a tile of 32 x 8 node columns and a
chunk of the node planes; how many chunks a grid's columns are split into
trades the blocks' start-up (three planes staged before the first is
computed) against filling the GPU's resident slots in few, full waves.  The
library picks the count from an occupancy model of one grid alone; in a
multi-grid batch the grids share every launch, so the best split of each
grid depends on the others.  tune() times the batch's FP32 iterations with
candidate counts, one grid at a time (coordinate descent from the
library's choice), and caches the result in a JSON file keyed by the grids'
sizes and right-hand-side counts.  The tile shape itself is fixed by the
kernels' tensor-copy boxes and shared-memory budget and is not tuned.
"""
from __future__ import annotations

import json
import os
import time

from mt3d import capi

CANDIDATES = (1, 2, 3, 4, 6, 8, 12, 16)


def key_of(solvers, omegas) -> str:
    return ";".join(f"{s.grid.nx}x{s.grid.ny}x{s.grid.nz}:{len(o)}" for s, o in zip(solvers, omegas))


def candidates(nz: int):
    """Chunk counts with at least 4 node planes per chunk; 0 is the library's
    own choice."""
    return [0] + [c for c in CANDIDATES if (nz + 1) // c >= 4]


def _time(solvers, omegas, e_ptrs, bc_ptrs, src_ptrs, trans, zch, sync, reset, reps: int) -> float:
    best = float("inf")
    for _ in range(reps):
        if reset is not None:
            reset()
        sync()
        t0 = time.perf_counter()
        capi.fwdsolve_multi(solvers, omegas, e_ptrs, trans=trans, bc=bc_ptrs, src=src_ptrs, zchunks=zch, device=True)
        sync()
        best = min(best, time.perf_counter() - t0)
    return best


def tune(solvers, omegas, e_ptrs, bc_ptrs, src_ptrs, trans, sync, cache_path: str | None = None, iters: int = 60,
         reps: int = 2, reset=None):
    """Per-grid chunk counts for a multi-grid batch (list of ints, 0 = the
    library's choice).  The timed runs are mt3d_fwdsolve_multi calls on the
    caller's device buffers (e_ptrs are overwritten) with one FP32 cycle of
    `iters` iterations per grid; sync() must wait for the device, and
    reset() (if given) must zero the e buffers, which every run then starts
    from.  Without it a run starts from the previous run's output, and a
    transposed solve returns its interior field multiplied by the edge
    volumes (as FWDsolve3D does), which is no first guess: repeated runs
    then grow without bound.  The handles' control is restored afterwards."""
    key = key_of(solvers, omegas)
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as fh:
            cache = json.load(fh)
        if key in cache:
            return list(cache[key]["zchunks"])
    keep = [dict(s.control) for s in solvers]
    try:
        for s, c in zip(solvers, keep):
            s.set_control(**dict(c, IterPerDivCor=iters, MaxDivCor=1))
        zch = [0] * len(solvers)
        t_best = _time(solvers, omegas, e_ptrs, bc_ptrs, src_ptrs, trans, zch, sync, reset, reps)
        t_default = t_best
        for g, s in enumerate(solvers):
            for c in candidates(s.grid.nz)[1:]:
                trial = list(zch)
                trial[g] = c
                t = _time(solvers, omegas, e_ptrs, bc_ptrs, src_ptrs, trans, trial, sync, reset, reps)
                if t < 0.98 * t_best:
                    t_best, zch = t, trial
    finally:
        for s, c in zip(solvers, keep):
            s.set_control(**c)
    if cache_path:
        cache[key] = {"zchunks": zch, "seconds": t_best, "default_seconds": t_default, "iters": iters}
        with open(cache_path, "w") as fh:
            json.dump(cache, fh, indent=1)
    return zch

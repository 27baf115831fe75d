"""Converged iteration counts of the CPU oracle on the 200x200x100 benchmark
workload, for the CPU baseline of bench.py.

TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline): nothing in the
product path imports it.

The CPU baseline times a bounded sample of the reference solver's Krylov
iterations (QMR with the D-ILU preconditioner and a divergence correction
every 40 iterations, the defaults of f90/3D_MT/FWD/EMsolve3D.f90:58-70) on the
benchmark grid on the GPU box's host cores, and scales the time per iteration
by the iterations a solve needs.  This script measures those iterations: it
runs the oracle to the benchmark's relative residual of 1e-7 on right-hand
sides of the benchmark's own workload -- the lowest, a middle and the highest
of the 16 frequencies, each as a forward solve (plane-wave boundary data of
polarisation 1) and as an adjoint solve (the receiver sources of polarisation
1) -- one process per solve, and writes cpu_iterations_200x200x100.json next
to this file.

    python oracle/cpu_iterations.py [--procs 6] [--freqs 0,8,15]

It takes hours of CPU time (about 1.5 s per QMR iteration per core on the
200x200x100 grid); run it once on the build host and commit the JSON.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this file's own directory heads sys.path, where a module
# would shadow the oracle package: import from the repository root instead
sys.path[:] = [p for p in sys.path if os.path.abspath(p or os.getcwd()) != HERE]
for _p in (os.path.join(ROOT, "modem-gpu_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)
OUT = os.path.join(HERE, "cpu_iterations_200x200x100.json")
TOL = 1e-7
ITER_PER_DIVCOR = 40  # the reference's default IterPerDivCor
MAX_DIVCOR = 300      # 12000 iterations at most


def _solve(job):
    fidx, kind = job
    sys.path.insert(0, os.path.join(ROOT, "modem-gpu_b200"))
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    from mt3d import bc as mbc
    from mt3d import models
    from oracle.oracle import PC_DILU, QMR, Oracle

    m, f = models.config_combined()
    omega = 2 * np.pi * float(f[fidx])
    o = Oracle(m.grid)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=QMR, precond=PC_DILU, IterPerDivCor=ITER_PER_DIVCOR, MaxDivCor=MAX_DIVCOR, tolEMfwd=TOL,
                  tolEMadj=TOL)
    t0 = time.perf_counter()
    if kind == "fwd":
        _, rc = o.fwdsolve(bc=mbc.boundary_1d(m, omega, 1))
    else:
        src = bench.receiver_sources(m, 20, seed=100)[0]
        _, rc = o.fwdsolve(trans=True, src=src)
    dt = time.perf_counter() - t0
    d = o.diagnostics()
    return {"freq_index": fidx, "freq_hz": float(f[fidx]), "kind": kind, "iterations": int(d["nIterTotal"]),
            "div_corrections": int(d["nDivCor"]), "converged": rc == 0,
            "final_relres": float(d["EMrelErr"][-1]) if len(d["EMrelErr"]) else None, "seconds": dt,
            "seconds_per_iteration": dt / max(1, d["nIterTotal"])}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=6)
    ap.add_argument("--freqs", default="0,8,15")
    args = ap.parse_args()
    jobs = [(int(i), k) for i in args.freqs.split(",") for k in ("fwd", "adj")]
    t0 = time.time()
    with mp.get_context("spawn").Pool(args.procs) as pool:
        res = pool.map(_solve, jobs, chunksize=1)
    its = [r["iterations"] for r in res]
    out = {"workload": "200x200x100 (12 air + 88 earth) random field (config_combined), 16 freq 1e-4..1e2 Hz",
           "solver": f"oracle QMR + D-ILU, divergence correction every {ITER_PER_DIVCOR} iterations, tol {TOL}",
           "mean_iterations": sum(its) / len(its), "solves": res, "host": platform.processor() or platform.machine(),
           "wall_seconds": time.time() - t0, "script": "oracle/cpu_iterations.py"}
    with open(OUT, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()

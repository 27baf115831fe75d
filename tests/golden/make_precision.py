"""Generate tests/golden/precision_100x100x60.npz: the FP64 oracle's converged
solution of the 100x100x60 random-field model at 1 Hz.

The model is models.config_precision() (10 air + 50 earth layers, seeded
Gaussian random field of log10 resistivity, mean 2, std 0.5, exponential
correlation length 5 cells, clipped to [0, 4]); the boundary data are the
1-D layered plane-wave fields of mt3d/bc.py for both polarisations.  The
oracle solves both forward problems with the reference's solver, QMR with
the D-ILU preconditioner and a divergence correction every 40 iterations
(f90/3D_MT/FWD/EMsolve3D.f90, f90/3D_MT/FWD/solver.f90), asked for a
relative residual of 1e-10 within 24000 iterations.  QMR levels off just
above that: the fixture records the residuals reached (2.2e-10 and 1.7e-10
for the two polarisations, status 1 = iteration limit) -- still three
orders below the 1e-7 of a production solve, so the iteration error of a
1e-7 solve dominates any comparison against it.

Stored: the Full_Impedance tensors (dataResp, f90/3D_MT/DataFunc.f90:143-189,
through oracle/datafunc.py) at a 10 x 10 array of surface sites on the core
cells, and both polarisations' fields on 4096 seeded earth edges.

    python tests/golden/make_precision.py

About two hours on two cores.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
# run as a script, this file's own directory heads sys.path, where a module
# would shadow the oracle package: import from the repository root instead
sys.path[:] = [p for p in sys.path if os.path.abspath(p or os.getcwd()) != HERE]
for _p in (os.path.join(ROOT, "modem-gpu_b200"), ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)
OUT = os.path.join(HERE, "precision_100x100x60.npz")
TOL = 1e-10
N_EDGES = 4096


def setup():
    """Model, omega, sites (x, y, z from the grid origin) and sampled edges."""
    sys.path.insert(0, os.path.join(ROOT, "modem-gpu_b200"))
    sys.path.insert(0, ROOT)
    from mt3d import bc as mbc
    from mt3d import models

    m, f = models.config_precision()
    g = m.grid
    omega = 2 * np.pi * float(f[0])
    xe = np.concatenate([[0.0], np.cumsum(g.dx)])
    ye = np.concatenate([[0.0], np.cumsum(g.dy)])
    ix = np.linspace(10, g.nx - 11, 10).round().astype(int)
    iy = np.linspace(10, g.ny - 11, 10).round().astype(int)
    sites = np.array([[0.5 * (xe[i] + xe[i + 1]), 0.5 * (ye[j] + ye[j + 1]), 0.0] for j in iy for i in ix])
    sig = mbc.edge_conductivity(m)
    earth = np.flatnonzero(sig > 1e-6)
    edges = np.sort(np.random.default_rng(7).choice(earth, N_EDGES, replace=False))
    return m, omega, sites, edges


def _solve(mode):
    sys.path.insert(0, os.path.join(ROOT, "modem-gpu_b200"))
    sys.path.insert(0, ROOT)
    from mt3d import bc as mbc
    from oracle.oracle import PC_DILU, QMR, Oracle

    m, omega, _, _ = setup()
    o = Oracle(m.grid)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=QMR, precond=PC_DILU, IterPerDivCor=40, MaxDivCor=600, tolEMfwd=TOL, tolEMadj=TOL)
    t0 = time.perf_counter()
    e, rc = o.fwdsolve(bc=mbc.boundary_1d(m, omega, mode))
    d = o.diagnostics()
    return e, rc, int(d["nIterTotal"]), float(d["EMrelErr"][-1]), time.perf_counter() - t0


def main():
    sys.path.insert(0, ROOT)
    from oracle import datafunc

    m, omega, sites, edges = setup()
    g = m.grid
    with mp.get_context("spawn").Pool(2) as pool:
        (e1, rc1, n1, r1, t1), (e2, rc2, n2, r2, t2) = pool.map(_solve, [1, 2])
    print(f"mode 1: rc {rc1}, {n1} iterations, relres {r1:.3e}, {t1:.0f} s")
    print(f"mode 2: rc {rc2}, {n2} iterations, relres {r2:.3e}, {t2:.0f} s")
    c = datafunc.coords(g.dx, g.dy, g.dz, g.nzAir)
    Z = datafunc.impedance(c, omega, sites, e1, e2)
    np.savez_compressed(OUT, sites=sites, omega=omega, Z=Z, edges=edges, E1=e1[edges], E2=e2[edges],
                        relres=np.array([r1, r2]), iterations=np.array([n1, n2]), tol=TOL,
                        status=np.array([rc1, rc2]))
    print("wrote", OUT)


if __name__ == "__main__":
    main()

"""Generate tests/golden/cylinder_tight.npz: the oracle's impedances for the
reference's cylinder fixture (tests/golden/cylinder_1per.npz, the set-up of
tests/test_golden.py) with the solves converged far beyond the fixture's own.

The fixture holds the reference's forward run at its production tolerance
1e-7, so it carries that run's iteration error (up to about 3e-5 of |Zxy|
at a few sites).  This file holds the same chain -- BC_x0_WS boundary
conditions and first guess (oracle/bc2d.py), QMR + D-ILU with a divergence
correction every 40 iterations (the reference's solver, oracle/mt3d_oracle.c),
dataResp (oracle/datafunc.py) -- run to a relative residual of 1e-10 or
where QMR levels off, so a tight GPU solve can be compared with the
converged discrete solution of the reference's own discretisation.

    python tests/golden/make_cylinder_tight.py
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path[:] = [p for p in sys.path if os.path.abspath(p or os.getcwd()) != HERE]
for _p in (os.path.join(ROOT, "modem-gpu_b200"), ROOT, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)
OUT = os.path.join(HERE, "cylinder_tight.npz")
TOL = 1e-10


def _solve(imode):
    from oracle import bc2d
    from oracle.oracle import PC_DILU, QMR, Oracle
    from test_golden import cylinder
    g, m, omega, sites, origin, G = cylinder()
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=QMR, precond=PC_DILU, MaxDivCor=500, tolEMfwd=TOL, tolEMadj=TOL, tolDivCor=1e-8)
    s = bc2d.sigma_cells(g, m.m_earth, m.air_cond)
    e0 = bc2d.compute_bc(g, s, omega, imode)
    t0 = time.perf_counter()
    e, rc = o.fwdsolve(bc=e0, e0=e0)
    d = o.diagnostics()
    return e, rc, int(d["nIterTotal"]), float(d["EMrelErr"][-1]), time.perf_counter() - t0


def main():
    from oracle import datafunc
    from test_golden import cylinder
    g, m, omega, sites, origin, G = cylinder()
    with mp.get_context("spawn").Pool(2) as pool:
        (e1, rc1, n1, r1, t1), (e2, rc2, n2, r2, t2) = pool.map(_solve, [1, 2])
    print(f"mode 1: rc {rc1}, {n1} iterations, relres {r1:.3e}, {t1:.0f} s")
    print(f"mode 2: rc {rc2}, {n2} iterations, relres {r2:.3e}, {t2:.0f} s")
    c = datafunc.coords(g.dx, g.dy, g.dz, g.nzAir, origin)
    Z = datafunc.impedance(c, omega, sites, e1, e2)
    np.savez_compressed(OUT, Z=Z, relres=np.array([r1, r2]), iterations=np.array([n1, n2]),
                        status=np.array([rc1, rc2]), tol=TOL)
    print("wrote", OUT)


if __name__ == "__main__":
    main()

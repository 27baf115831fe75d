"""The precision statement on the 100x100x60 random-field model at 1 Hz
(models.config_precision): the GPU's mixed-precision and FP64 solves against
the oracle's FP64 solution converged to a relative residual of 2e-10
(tests/golden/precision_100x100x60.npz, made by tests/golden/make_precision.py
with the reference's solver, QMR + D-ILU, which levels off there).

For each GPU path and tolerance the test records the relative error of the
fields on 4096 seeded earth edges (2-norm) and of the Full_Impedance tensors
at 100 surface sites (per site, max_ij |dZ_ij| / max_ij |Z_ij|, the largest
over the sites).  Bounds, about five times the measured errors:
  * grad-div formulation (the benchmark's), FP64 and mixed precision with
    FP64 refinement (with the diagonal and with the benchmark's polynomial
    preconditioner): at residual 1e-7 impedances within 1e-5 and fields
    within 2e-5 (measured 1.7e-6 / 2.5e-6); at 1e-8 within 1e-6 and 2e-6
    (1.3e-7 / 1.7e-7); at 1e-9 within 1e-7 and 2e-7 (1.5e-8 / 2.0e-8);
  * the reference's formulation (curl-curl + divergence correction), FP64
    and mixed, at the production tolerance 1e-7: impedances within 1e-6 and
    fields within 5e-6 (measured 8.0e-7 / 1.3e-6).
"""
import os

import numpy as np
import pytest

from mt3d import bc as mbc
from mt3d import capi, models

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def z_error(Z, Zref):
    Z, Zref = np.asarray(Z).reshape(-1, 4), np.asarray(Zref).reshape(-1, 4)
    return float(np.max(np.max(np.abs(Z - Zref), axis=1) / np.max(np.abs(Zref), axis=1)))


@pytest.fixture(scope="module")
def precision_case(cuda):
    f = np.load(os.path.join(HERE, "golden", "precision_100x100x60.npz"))
    assert np.all(f["relres"] <= 3e-10)
    m, freqs = models.config_precision()
    omega = 2 * np.pi * float(freqs[0])
    assert abs(omega - float(f["omega"])) < 1e-12 * omega
    bcs = [mbc.boundary_1d(m, omega, mode) for mode in (1, 2)]
    return f, m, omega, bcs


BOUNDS = {  # (formulation, tol): (impedance, field)
    (capi.FORM_CCGD, 1e-7): (1e-5, 2e-5),
    (capi.FORM_CCGD, 1e-8): (1e-6, 2e-6),
    (capi.FORM_CCGD, 1e-9): (1e-7, 2e-7),
    (capi.FORM_CCDC, 1e-7): (1e-6, 5e-6),
}


# (precision, polynomial preconditioner coefficient): FP64, mixed with the
# diagonal preconditioner, and mixed with the benchmark's polynomial one
# (grad-div formulation only, the one the benchmark runs)
PATHS = {"fp64": (capi.PREC_FP64, 0.0), "mixed": (capi.PREC_MIXED, 0.0), "mixed-poly": (capi.PREC_MIXED, 0.9)}
CASES = [(f, t, p) for f, t in BOUNDS for p in PATHS if not (p == "mixed-poly" and f == capi.FORM_CCDC)]


@pytest.mark.parametrize("formulation,tol,path", CASES, ids=[f"{'ccgd' if f else 'ccdc'}-{t:g}-{p}" for f, t, p in CASES])
def test_precision_against_converged_oracle(precision_case, formulation, tol, path):
    f, m, omega, bcs = precision_case
    precision, poly = PATHS[path]
    s = capi.Solver(m.grid)
    s.set_formulation(formulation)
    s.set_restart(0)
    s.set_poly(poly)
    s.update_cond(m.m_earth, m.air_cond)
    if formulation == capi.FORM_CCGD:
        s.set_control(IterPerDivCor=300, MaxDivCor=60, tolEMfwd=tol, tolEMadj=tol, precision=precision)
    else:
        s.set_control(IterPerDivCor=100, MaxDivCor=300, tolEMfwd=tol, tolEMadj=tol, tolDivCor=1e-9,
                      precision=precision)
    e, st, rc = s.fwdsolve_batch(np.array([omega, omega]), bc=np.stack(bcs))
    it, rr = s.batch_diagnostics(2)
    assert rc == 0
    Z = s.impedance(omega, f["sites"], e[0], e[1])
    zerr = z_error(Z, f["Z"])
    idx = f["edges"]
    eerr = max(np.linalg.norm(e[0][idx] - f["E1"]) / np.linalg.norm(f["E1"]),
               np.linalg.norm(e[1][idx] - f["E2"]) / np.linalg.norm(f["E2"]))
    print(f"formulation {formulation} path {path} tol {tol:g}: iterations {it.tolist()}, "
          f"relres {rr.tolist()}, Z error {zerr:.3e}, E error {eerr:.3e}")
    zb, eb = BOUNDS[(formulation, tol)]
    assert zerr <= zb and eerr <= eb

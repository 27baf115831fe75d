"""The precision statement on the 100x100x60 random-field model at 1 Hz
(models.config_precision): the GPU's mixed-precision and FP64 solves against
the oracle's FP64 solution converged to a relative residual of 2e-10
(tests/golden/precision_100x100x60.npz, made by tests/golden/make_precision.py
with the reference's solver, QMR + D-ILU, which levels off there).

For each GPU path and tolerance the test records the relative error of the
fields on 4096 seeded earth edges (2-norm) and of the Full_Impedance tensors
at 100 surface sites (per site, max_ij |dZ_ij| / max_ij |Z_ij|, the largest
over the sites).  Bounds:
  * at relative residual 1e-9 (FP64, and mixed with FP64 refinement), every
    impedance within 1e-6 and the sampled fields within 1e-5;
  * at the production tolerance 1e-7, impedances within 1e-4 and fields
    within 1e-3 (the iteration error of a 1e-7 solve; the printed values are
    the measured ones).
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


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("tol", [1e-7, 1e-9])
def test_precision_against_converged_oracle(precision_case, precision, tol):
    f, m, omega, bcs = precision_case
    s = capi.Solver(m.grid)
    s.set_formulation(capi.FORM_CCGD)
    s.set_restart(0)
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=300, MaxDivCor=60, tolEMfwd=tol, tolEMadj=tol, precision=precision)
    e, st, rc = s.fwdsolve_batch(np.array([omega, omega]), bc=np.stack(bcs))
    it, rr = s.batch_diagnostics(2)
    assert rc == 0 and np.all(rr <= tol)
    Z = s.impedance(omega, f["sites"], e[0], e[1])
    zerr = z_error(Z, f["Z"])
    idx = f["edges"]
    eerr = max(np.linalg.norm(e[0][idx] - f["E1"]) / np.linalg.norm(f["E1"]),
               np.linalg.norm(e[1][idx] - f["E2"]) / np.linalg.norm(f["E2"]))
    print(f"precision {precision} tol {tol:g}: iterations {it.tolist()}, relres {rr.tolist()}, "
          f"Z error {zerr:.3e}, E error {eerr:.3e}")
    if tol <= 1e-9:
        assert zerr <= 1e-6 and eerr <= 1e-5
    else:
        assert zerr <= 1e-4 and eerr <= 1e-3

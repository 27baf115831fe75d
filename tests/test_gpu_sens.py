"""The misfit gradient on the GPU (mt3d_jmult_t through mt3d/sens.py) against
the oracle's restatement of the reference's JmultT_TX chain and against
central finite differences, and the transpose-solve identity of the
reference's symmetry test, on the device.

Problem: tests/test_oracle.py::gradient_problem (10 x 12 x 12 grid, two
frequencies, four sites, 5 % noise).  The oracle's chain is itself checked
against finite differences there.

Tolerances:
  * FP64 GPU gradient vs the oracle's: relative 2-norm <= 1e-6 (solves to
    relative residual 1e-10 on both sides);
  * mixed-precision GPU gradient vs the oracle's: <= 1e-5 (1e-10 FP64
    residual reached by FP32 cycles under FP64 refinement);
  * GPU finite differences (step 1e-4, six earth cells) vs the GPU
    gradient: <= 1e-4 of the largest gradient entry (each misfit from solves
    to 1e-10, whose iteration error no longer cancels between m + h and
    m - h as the oracle's does);
  * the symmetry identity b2^T S b1 = b1^T S^T b2: <= 1e-6 relative.
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, relerr, small_grid
from mt3d import bc as mbc
from mt3d import capi, models
from mt3d import sens as gsens
from oracle.oracle import Oracle, interior_edge_mask
from test_oracle import gradient_problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gprob(cuda):
    from oracle import sens
    g, start, freqs, bcs, sites, d_obs, err, ctl, cells = gradient_problem()
    phi, grad = sens.misfit_gradient(g, start, freqs, bcs, sites, d_obs, err, ctl)
    return g, start, freqs, bcs, sites, d_obs, err, cells, phi, grad


def _solver(g, m, formulation, precision, tol=1e-10):
    s = capi.Solver(g)
    s.set_formulation(formulation)
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=200, MaxDivCor=100, tolEMfwd=tol, tolEMadj=tol, tolDivCor=1e-10,
                  precision=precision)
    return s


@pytest.mark.parametrize("formulation", [capi.FORM_CCDC, capi.FORM_CCGD], ids=["ccdc", "ccgd"])
@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_MIXED], ids=["fp64", "mixed"])
def test_gradient_matches_oracle_chain(gprob, formulation, precision):
    g, start, freqs, bcs, sites, d_obs, err, cells, phi_o, grad_o = gprob
    s = _solver(g, start, formulation, precision)
    phi, grad = gsens.misfit_gradient(s, start.m_earth, freqs, bcs, sites, d_obs, err)
    assert abs(phi - phi_o) <= 1e-8 * phi_o
    assert relerr(grad, grad_o) <= (1e-6 if precision == capi.PREC_FP64 else 1e-5)


def test_gradient_matches_finite_differences(gprob):
    g, start, freqs, bcs, sites, d_obs, err, cells, _, _ = gprob
    s = _solver(g, start, capi.FORM_CCGD, capi.PREC_FP64)
    phi, grad = gsens.misfit_gradient(s, start.m_earth, freqs, bcs, sites, d_obs, err)
    h = 1e-4
    for c in cells:
        f = []
        for sign in (1, -1):
            m = start.m_earth.copy()
            m[c] += sign * h
            s.update_cond(m, start.air_cond)
            Z, _ = gsens.predict(s, freqs, bcs, sites)
            f.append(gsens.misfit(Z, d_obs, err)[0])
        fd = (f[0] - f[1]) / (2 * h)
        assert abs(fd - grad[c]) <= 1e-4 * np.abs(grad).max(), (c, fd, grad[c])


def test_jmult_t_device_entry_matches_host(gprob):
    import torch
    g, start, freqs, bcs, sites, d_obs, err, cells, _, _ = gprob
    s = _solver(g, start, capi.FORM_CCGD, capi.PREC_MIXED)
    Z, E = gsens.predict(s, freqs, bcs, sites)
    _, w, _ = gsens.misfit(Z, d_obs, err)
    om = 2 * np.pi * freqs[0]
    dm, ea, rc = s.jmult_t(om, sites, E[0, 0], E[0, 1], w[0], start.m_earth, want_eadj=True)
    assert rc == 0
    e0 = torch.from_numpy(np.ascontiguousarray(E[0])).to("cuda")
    dmd = torch.zeros(dm.size, dtype=torch.float64, device="cuda")
    ead = torch.zeros((2, s.nE), dtype=torch.complex128, device="cuda")
    assert s.jmult_t_device(om, sites, e0.data_ptr(), w[0], start.m_earth, dmd.data_ptr(), ead.data_ptr()) == 0
    torch.cuda.synchronize()
    assert np.array_equal(dmd.cpu().numpy(), dm)
    assert np.array_equal(ead.cpu().numpy(), ea)


@pytest.mark.parametrize("formulation", [capi.FORM_CCDC, capi.FORM_CCGD], ids=["ccdc", "ccgd"])
def test_transpose_solve_identity_on_device(cuda, formulation):
    """Stest-style identity (f90/SENS/SymmetryTest.f90:205-272) with the GPU
    solves: for S = A_II^-1, b2^T S b1 = b1^T S^T b2, S^T from the
    transposed solve (whose output is V_E-weighted, EMsolve3D.f90:356-359)."""
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    VE = o.VE
    mask = interior_edge_mask(g)
    em = mask & earth_mask(g, m)
    rng = np.random.default_rng(11)
    s1 = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    s2 = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    s = _solver(g, m, formulation, capi.PREC_FP64, tol=1e-9)
    s.update_freq(omega)
    e1, rc1 = s.fwdsolve(trans=False, src=s1)
    e2, rc2 = s.fwdsolve(trans=True, src=VE * s2)
    assert rc1 == 0 and rc2 == 0
    lhs = (VE * s2)[mask] @ e1[mask]
    rhs = (VE * s1)[mask] @ (e2[mask] / VE[mask])
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs)


def test_config_gradient_against_central_differences(cuda):
    """The gradient workload: 80 x 80 x 50 grid, data of the true model
    (random field with a 0.3 and a 1000 ohm-m block) at 10 x 10 surface
    sites and 6 frequencies (1e-3..1e1 Hz) with 5 % noise, gradient at the
    100 ohm-m halfspace.  The gradient with respect to log10 sigma is ln(10)
    times the ln sigma gradient (the model parameter of the library).
    Central differences with step 1e-4 in log10 sigma on 32 seeded earth
    cells of the top 20 layers under the core agree with it to 1e-4 of the
    largest gradient entry, and the reference's Taylor test (TEST_GRAD,
    f90/Mod3DMT.f90:297-333) with a random step of 1e-3 agrees to 2 % (its
    second-order term).  The gradient comes from mixed-precision solves to
    1e-10; the differences of the misfit need FP64 solves to 1e-12 (at 1e-10
    their iteration error left a median deviation of 3.5e-4)."""
    true, start, freqs = models.config_gradient()
    g = true.grid
    xe = np.concatenate([[0.0], np.cumsum(g.dx)])
    ye = np.concatenate([[0.0], np.cumsum(g.dy)])
    ii = np.arange(g.nx // 2 - 20, g.nx // 2 + 20, 4)
    jj = np.arange(g.ny // 2 - 20, g.ny // 2 + 20, 4)
    sites = np.array([[0.5 * (xe[i] + xe[i + 1]), 0.5 * (ye[j] + ye[j + 1]), 0.0] for j in jj for i in ii])
    assert len(sites) == 100
    bcs = [[mbc.boundary_1d(start, 2 * np.pi * f, p) for p in (1, 2)] for f in freqs]
    s = _solver(g, true, capi.FORM_CCGD, capi.PREC_MIXED)
    Zt, _ = gsens.predict(s, freqs, bcs, sites)
    rng = np.random.default_rng(7)
    err = 0.05 * np.abs(Zt).max(axis=(2, 3))[..., None, None] * np.ones(Zt.shape)
    d_obs = Zt + err * (rng.standard_normal(Zt.shape) + 1j * rng.standard_normal(Zt.shape)) / np.sqrt(2)
    s.update_cond(start.m_earth, start.air_cond)
    phi, grad = gsens.misfit_gradient(s, start.m_earth, freqs, bcs, sites, d_obs, err)
    grad10 = np.log(10.0) * grad
    ci = rng.integers(g.nx // 2 - 20, g.nx // 2 + 20, 32)
    cj = rng.integers(g.ny // 2 - 20, g.ny // 2 + 20, 32)
    ck = rng.integers(0, 20, 32)
    cells = [int(i + g.nx * (j + g.ny * k)) for i, j, k in zip(ci, cj, ck)]
    sf = _solver(g, start, capi.FORM_CCGD, capi.PREC_FP64, tol=1e-12)
    h10 = 1e-4
    fd = gsens.central_differences(sf, start.m_earth, start.air_cond, cells, freqs, bcs, sites, d_obs, err,
                                   h=h10 * np.log(10.0)) * np.log(10.0)
    dev = np.abs(fd - grad10[cells]) / np.abs(grad10).max()
    dm = 1e-3 * rng.standard_normal(start.m_earth.size)
    f0, df, lin = gsens.taylor_test(s, start.m_earth, start.air_cond, dm, freqs, bcs, sites, d_obs, err)
    print(f"config_gradient: phi {phi:.6e}, max|grad log10| {np.abs(grad10).max():.3e}, FD deviation max "
          f"{dev.max():.2e} median {np.median(dev):.2e}, Taylor f(m0+dm)-f(m0) {df:.6e} vs grad.dm {lin:.6e}")
    assert dev.max() <= 1e-4
    assert abs(df - lin) <= 0.02 * abs(lin)

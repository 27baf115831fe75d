"""GPU parity: the CUDA path (through the C ABI, libmt3d.so) against the oracle.

Tolerances (FP64 unless stated):
  * operator apply: relative 2-norm difference <= 1e-13 (summation order only);
  * BiCGStab residual history: <= 1e-8 relative over the first iterations;
  * solutions of the full divergence-corrected solve: <= 1e-5 relative on the
    edges where the field is unique (sigma > 0), both solves at tol 1e-7 or
    tighter; the air edges carry a gauge (gradient) part that only the
    divergence correction pins;
  * mixed precision (FP32 inner iterations, FP64 refinement) against FP64:
    the same 1e-5 bound, and a true FP64 relative residual <= the tolerance.
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, relerr, small_grid
from mt3d import bc as mbc
from mt3d import capi, models
from oracle.oracle import BICG, COCG, PC_JACOBI, PC_ZLINE, Oracle, interior_edge_mask

pytestmark = pytest.mark.gpu


def make_pair(g, m, omega, **ctl):
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=BICG, precond=PC_JACOBI, **ctl)
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(**ctl)
    return o, s


@pytest.fixture(scope="module")
def prob(cuda):
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    o, s = make_pair(g, m, omega)
    return g, m, omega, o, s


def test_interior_index(prob):
    g, m, omega, o, s = prob
    idx = s.interior_index() - 1
    assert np.array_equal(np.flatnonzero(interior_edge_mask(g)), idx)


def test_mult_aii_matches_oracle(prob):
    g, m, omega, o, s = prob
    mask = interior_edge_mask(g)
    rng = np.random.default_rng(0)
    xi = rng.standard_normal(s.nEi) + 1j * rng.standard_normal(s.nEi)
    x = np.zeros(g.n_edges, complex)
    x[mask] = xi
    for adjt in (False, True):
        y = s.mult_aii(xi, adjt=adjt)
        yref = o.multA(x, adjt=adjt)[mask]
        assert relerr(y, yref) < 1e-13


def test_operator_setup_matches_oracle(prob):
    """Sigma_E and the DivCorrSetUp coefficients that update_cond builds on the
    device against the oracle's UpdateCond (relative 1e-14: the cell
    exponentials may differ in the last bit)."""
    g, m, omega, o, s = prob
    sig, coef, _ = s.get_cond()
    assert np.max(np.abs(sig - o.sigE) / np.maximum(np.abs(o.sigE), 1e-300)) < 1e-14
    db1, db2, c = o.divcorr_coef()
    nx, ny, nz = g.nx, g.ny, g.nz
    nX, nY = nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    i, j, k = (a.ravel(order="F") for a in (i, j, k))
    inner = (i >= 1) & (i < nx) & (j >= 1) & (j < ny) & (k >= 1) & (k < nz)
    ii, jj, kk = i[inner], j[inner], k[inner]
    ex = ii + nx * (jj + (ny + 1) * kk)
    ey = nX + ii + (nx + 1) * (jj + ny * kk)
    ez = nX + nY + ii + (nx + 1) * (jj + (ny + 1) * kk)
    want = np.zeros((7, s.nN))
    for q, (arr, e) in enumerate(((db1, ex), (db2, ex), (db1, ey), (db2, ey), (db1, ez), (db2, ez))):
        want[q, inner] = arr[e]
    want[6] = c
    scale = np.max(np.abs(want), axis=1, keepdims=True)
    assert np.max(np.abs(coef - want) / scale) < 1e-14
    assert np.all(coef[:, ~inner] == 0)


@pytest.mark.parametrize("imode", [1, 2])
def test_compute_bc_matches_oracle(prob, imode):
    """E0 of the 2-D TE boundary solver on the device (band elimination in
    shared memory) against the oracle's sparse direct solves: relative 1e-10."""
    from oracle import bc2d
    g, m, omega, o, s = prob
    e = s.compute_bc(imode)
    want = bc2d.compute_bc(g, bc2d.sigma_cells(g, m.m_earth, m.air_cond), omega, imode)
    assert np.max(np.abs(e - want)) < 1e-10 * np.max(np.abs(want))


def test_compute_bc_window_in_global_memory(cuda):
    """130 vertical cells: the elimination window (130 x 130 complex, 270 KB)
    no longer fits in shared memory and lives in global memory, and the rows
    exceed four per thread (the generic update loop)."""
    from oracle import bc2d
    g = models.make_grid(6, 7, 30, 100, core=500.0, n_pad=1, pad_growth=1.6, air_first=60.0, air_growth=1.12,
                         earth_first=40.0, earth_growth=1.03)
    m = random_model(g, seed=7)
    omega = 2 * np.pi * 0.3
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    sig = bc2d.sigma_cells(g, m.m_earth, m.air_cond)
    for imode in (1, 2):
        e = s.compute_bc(imode)
        want = bc2d.compute_bc(g, sig, omega, imode)
        assert np.max(np.abs(e - want)) < 1e-10 * np.max(np.abs(want))


def test_compute_bc_device_matches_host(prob):
    """mt3d_compute_bc_device (explicit omega, device output) gives the same E0
    as the host entry point at the handle's frequency."""
    import torch
    g, m, omega, o, s = prob
    for imode in (1, 2):
        out = torch.zeros(2 * s.nE, dtype=torch.float64, device="cuda")
        s._check(s.L.mt3d_compute_bc_device(s.h, imode, float(omega), capi.C.c_void_p(out.data_ptr())))
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.complex128), s.compute_bc(imode))
    with pytest.raises(capi.MT3DError):
        s._check(s.L.mt3d_compute_bc_device(s.h, 3, float(omega), capi.C.c_void_p(out.data_ptr())))


def test_compute_bc_tall_slices(cuda):
    """72 vertical cells: the elimination window (72 x 72 complex, 81 KB) takes
    the opted-in shared memory and 32 x 32 threads."""
    from oracle import bc2d
    g = models.make_grid(8, 9, 20, 52, core=500.0, n_pad=2, pad_growth=1.6, air_first=60.0, air_growth=1.3,
                         earth_first=40.0, earth_growth=1.08)
    m = random_model(g, seed=5)
    omega = 2 * np.pi * 3.0
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    sig = bc2d.sigma_cells(g, m.m_earth, m.air_cond)
    for imode in (1, 2):
        e = s.compute_bc(imode)
        want = bc2d.compute_bc(g, sig, omega, imode)
        assert np.max(np.abs(e - want)) < 1e-10 * np.max(np.abs(want))


def test_bicg_history_matches_oracle(prob):
    g, m, omega, o, s = prob
    mask = interior_edge_mask(g)
    bcv = mbc.boundary_1d(m, omega, 2)
    b = -o.multA(np.where(mask, 0, bcv))
    x0 = np.zeros(g.n_edges, complex)
    xo, no, ro, fo = o.krylov(b, x0, 40, 1e-7)
    xg, ng, rg, fg, rc = s.bicg(b[mask], np.zeros(s.nEi, complex), 40, 1e-7)
    assert fo == fg == 0
    k = min(12, ng, no)
    assert np.max(np.abs(rg[:k] - ro[:k]) / ro[:k]) < 1e-8
    if no == ng:
        assert relerr(xg, xo[mask]) < 1e-6


@pytest.mark.parametrize("mode", [1, 2])
def test_fwdsolve_fp64_matches_oracle(prob, mode):
    g, m, omega, o, s = prob
    bcv = mbc.boundary_1d(m, omega, mode)
    s.set_control(precision=capi.PREC_FP64)
    eg, rc = s.fwdsolve(bc=bcv)
    eo, rco = o.fwdsolve(bc=bcv)
    assert rc == 0 and rco == 0
    em = earth_mask(g, m)
    assert relerr(eg[em], eo[em]) < 1e-5
    bmask = ~interior_edge_mask(g)
    assert np.array_equal(eg[bmask], bcv[bmask])
    dg, do = s.diagnostics(), o.diagnostics()
    assert dg["nDivCor"] >= 1
    assert abs(dg["nIterTotal"] - do["nIterTotal"]) <= max(3, 0.1 * do["nIterTotal"])
    assert dg["final_relres"] < 5e-7


@pytest.mark.parametrize("mode", [1, 2])
def test_qmr_matches_oracle(prob, mode):
    """GPU QMR (the reference's default solver, f90/3D_MT/FWD/solver.f90:
    122-343) with the diagonal preconditioner against the oracle's QMR with
    the same preconditioner: the residual history of the first Krylov call
    to 1e-8, the divergence-corrected solution to 1e-5 on the edges where it
    is unique, and the iteration counts within 10 %."""
    from oracle.oracle import QMR
    g, m, omega, o, s = prob
    bcv = mbc.boundary_1d(m, omega, mode)
    o.set_control(solver=QMR, precond=PC_JACOBI)
    s.set_control(solver=capi.SOLVER_QMR, precision=capi.PREC_FP64)
    try:
        eg, rc = s.fwdsolve(bc=bcv)
        eo, rco = o.fwdsolve(bc=bcv)
        dg, do = s.diagnostics(), o.diagnostics()
    finally:
        o.set_control(solver=BICG, precond=PC_JACOBI)
        s.set_control(precision=capi.PREC_FP64)
    assert rc == 0 and rco == 0
    k = min(12, len(dg["EMrelErr"]), len(do["EMrelErr"]))
    assert np.max(np.abs(dg["EMrelErr"][:k] - do["EMrelErr"][:k]) / do["EMrelErr"][:k]) < 1e-8
    em = earth_mask(g, m)
    assert relerr(eg[em], eo[em]) < 1e-5
    assert abs(dg["nIterTotal"] - do["nIterTotal"]) <= max(3, 0.1 * do["nIterTotal"])


def test_qmr_rejects_mixed_precision(prob):
    g, m, omega, o, s = prob
    with pytest.raises(capi.MT3DError) as ei:
        s.set_control(solver=capi.SOLVER_QMR, precision=capi.PREC_MIXED)
    assert ei.value.code == 5
    s.set_control(precision=capi.PREC_FP64)


def test_fwdsolve_mixed_matches_fp64(prob):
    g, m, omega, o, s = prob
    bcv = mbc.boundary_1d(m, omega, 1)
    s.set_control(precision=capi.PREC_FP64)
    e64, rc64 = s.fwdsolve(bc=bcv)
    s.set_control(precision=capi.PREC_MIXED)
    emx, rcm = s.fwdsolve(bc=bcv)
    d = s.diagnostics()
    s.set_control(precision=capi.PREC_FP64)
    assert rc64 == 0 and rcm == 0
    assert d["final_relres"] <= 1e-7
    em = earth_mask(g, m)
    assert relerr(emx[em], e64[em]) < 1e-5


def test_layered_closed_form_gpu(cuda):
    g = small_grid()
    m = models.halfspace_model(g, 30.0)
    omega = 2 * np.pi * 0.1
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        s.set_control(tolEMfwd=1e-9, precision=prec)
        for mode in (1, 2):
            e, rc = s.fwdsolve(bc=mbc.boundary_1d(m, omega, mode))
            assert rc == 0
            assert relerr(e, mbc.layered_solution(m, omega, mode)) < 1e-6


def test_batch_matches_single(prob):
    g, m, omega, o, s = prob
    oms = np.array([omega, omega, 2 * np.pi * 0.05, 2 * np.pi * 0.05])
    modes = [1, 2, 1, 2]
    bcs = np.stack([mbc.boundary_1d(m, w, md) for w, md in zip(oms, modes)])
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        s.set_control(precision=prec, MaxDivCor=100)
        eb, st, rc = s.fwdsolve_batch(oms, bc=bcs)
        assert rc == 0 and np.all(st == 0)
        for r in range(4):
            s.update_freq(oms[r])
            e1, rc1 = s.fwdsolve(bc=bcs[r])
            assert rc1 == 0
            assert relerr(eb[r], e1) < 1e-12
    s.update_freq(omega)
    s.set_control(precision=capi.PREC_FP64)


def test_transposed_solve_matches_oracle(prob):
    g, m, omega, o, s = prob
    mask = interior_edge_mask(g)
    em = mask & earth_mask(g, m)
    rng = np.random.default_rng(4)
    src = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    src = src * o.VE
    eg, rc = s.fwdsolve(trans=True, src=src)
    eo, rco = o.fwdsolve(trans=True, src=src)
    assert rc == 0 and rco == 0
    emask = earth_mask(g, m)
    assert relerr(eg[emask], eo[emask]) < 1e-5
    # boundary values from AdjtBC of the V_E-weighted interior solution
    bm = ~mask
    assert relerr(eg[bm], o.adjt_bc(np.where(mask, eg, 0))[bm] * -1) < 1e-10


def test_forward_source_matches_oracle(prob):
    g, m, omega, o, s = prob
    mask = interior_edge_mask(g)
    em = mask & earth_mask(g, m)
    rng = np.random.default_rng(9)
    src = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    eg, rc = s.fwdsolve(trans=False, src=src)
    eo, rco = o.fwdsolve(trans=False, src=src)
    assert rc == 0 and rco == 0
    emask = earth_mask(g, m)
    assert relerr(eg[emask], eo[emask]) < 1e-5


def test_pmult_t_matches_oracle(prob):
    g, m, omega, o, s = prob
    rng = np.random.default_rng(2)
    e0 = rng.standard_normal((2, g.n_edges)) + 1j * rng.standard_normal((2, g.n_edges))
    ea = rng.standard_normal((2, g.n_edges)) + 1j * rng.standard_normal((2, g.n_edges))
    assert relerr(s.pmult_t(e0, ea, m.m_earth), o.pmult_t(e0, ea, m.m_earth)) < 1e-13


def test_config_small_forward_matches_oracle(cuda):
    """The 24x24x24 forward configuration (100 ohm-m halfspace with a 1 ohm-m
    block, 0.1 Hz, both polarisations) through the batch entry point."""
    m, freqs = models.config_small_forward()
    g = m.grid
    omega = 2 * np.pi * freqs[0]
    o, s = make_pair(g, m, omega)
    bcs = np.stack([mbc.boundary_1d(m, omega, md) for md in (1, 2)])
    em = earth_mask(g, m)
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        s.set_control(precision=prec)
        eb, st, rc = s.fwdsolve_batch(np.array([omega, omega]), bc=bcs)
        assert rc == 0
        for r, md in enumerate((1, 2)):
            eo, rco = o.fwdsolve(bc=bcs[r])
            assert rco == 0
            assert relerr(eb[r][em], eo[em]) < 1e-5


def test_error_paths(cuda):
    g = small_grid()
    s = capi.Solver(g)
    m = random_model(g)
    bad = m.m_earth.copy()
    bad[3] = np.nan
    with pytest.raises(capi.MT3DError) as ei:
        s.update_cond(bad, m.air_cond)
    assert ei.value.code == 3
    with pytest.raises(capi.MT3DError) as ei:
        s.fwdsolve(bc=np.zeros(s.nE, complex))
    assert ei.value.code == 5  # conductivity not set
    s.update_cond(m.m_earth, m.air_cond)
    with pytest.raises(capi.MT3DError) as ei:
        s.update_freq(-1.0)
    assert ei.value.code == 5
    with pytest.raises(capi.MT3DError) as ei:
        s.set_control(precision=7)
    assert ei.value.code == 5
    s.update_freq(1.0)
    bcv = np.zeros(s.nE, complex)
    # Ex(i=1, j=0, k=1): a boundary edge that the interior equations read
    bcv[1 + g.nx * (g.ny + 1)] = np.nan
    e, rc = s.fwdsolve(bc=bcv)
    assert rc == 3


# ---------------------------------------------------------------------------
# Bi-CG for the complex-symmetric system (COCG) with the z-line preconditioner
# ---------------------------------------------------------------------------
def make_cocg_pair(g, m, omega, **ctl):
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=COCG, precond=PC_ZLINE, **ctl)
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(solver=capi.SOLVER_COCG, **ctl)
    return o, s


@pytest.fixture(scope="module")
def cprob(cuda):
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    o, s = make_cocg_pair(g, m, omega)
    return g, m, omega, o, s


@pytest.mark.parametrize("mode", [1, 2])
def test_cocg_fp64_matches_oracle(cprob, mode):
    g, m, omega, o, s = cprob
    bcv = mbc.boundary_1d(m, omega, mode)
    s.set_control(solver=capi.SOLVER_COCG, precision=capi.PREC_FP64)
    eg, rc = s.fwdsolve(bc=bcv)
    eo, rco = o.fwdsolve(bc=bcv)
    assert rc == 0 and rco == 0
    dg, do = s.diagnostics(), o.diagnostics()
    # same method: the residual histories agree over the first iterations
    k = min(15, len(do["EMrelErr"]), len(dg["EMrelErr"]))
    assert np.max(np.abs(dg["EMrelErr"][:k] - do["EMrelErr"][:k]) / do["EMrelErr"][:k]) < 1e-6
    em = earth_mask(g, m)
    assert relerr(eg[em], eo[em]) < 1e-5
    assert abs(dg["nIterTotal"] - do["nIterTotal"]) <= max(3, 0.1 * do["nIterTotal"])


def test_cocg_mixed_matches_fp64(cprob):
    g, m, omega, o, s = cprob
    bcv = mbc.boundary_1d(m, omega, 2)
    s.set_control(solver=capi.SOLVER_COCG, precision=capi.PREC_FP64)
    e64, rc64 = s.fwdsolve(bc=bcv)
    s.set_control(solver=capi.SOLVER_COCG, precision=capi.PREC_MIXED)
    emx, rcm = s.fwdsolve(bc=bcv)
    d = s.diagnostics()
    assert rc64 == 0 and rcm == 0 and d["final_relres"] <= 1e-7
    em = earth_mask(g, m)
    assert relerr(emx[em], e64[em]) < 1e-5


def test_cocg_transposed_and_batch(cprob):
    g, m, omega, o, s = cprob
    mask = interior_edge_mask(g)
    em = mask & earth_mask(g, m)
    rng = np.random.default_rng(4)
    src = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0) * o.VE
    oms = np.array([omega, 2 * np.pi * 0.05, omega, 2 * np.pi * 0.05])
    srcs = np.stack([src] * 4)
    s.set_control(solver=capi.SOLVER_COCG, precision=capi.PREC_MIXED, MaxDivCor=100)
    eb, st, rc = s.fwdsolve_batch(oms, trans=np.ones(4, np.int32), src=srcs)
    assert rc == 0 and np.all(st == 0)
    o.set_control(solver=COCG, precond=PC_ZLINE, MaxDivCor=100)
    for r in (0, 1):
        o.update_freq(oms[r])
        eo, rco = o.fwdsolve(trans=True, src=src)
        assert rco == 0
        sel = earth_mask(g, m)
        assert relerr(eb[r][sel], eo[sel]) < 1e-5
    o.update_freq(omega)


def test_cocg_config_small_forward(cuda):
    m, freqs = models.config_small_forward()
    g = m.grid
    omega = 2 * np.pi * freqs[0]
    o, s = make_cocg_pair(g, m, omega)
    bcs = np.stack([mbc.boundary_1d(m, omega, md) for md in (1, 2)])
    em = earth_mask(g, m)
    s.set_control(solver=capi.SOLVER_COCG, precision=capi.PREC_MIXED)
    eb, st, rc = s.fwdsolve_batch(np.array([omega, omega]), bc=bcs)
    assert rc == 0
    for r in range(2):
        eo, rco = o.fwdsolve(bc=bcs[r])
        assert rco == 0
        assert relerr(eb[r][em], eo[em]) < 1e-5


# ---------------------------------------------------------------------------
# BiCGStab with the z-line preconditioner
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("prec", [0, 1])
def test_bicg_zline_matches_oracle(cuda, prec):
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=BICG, precond=PC_ZLINE)
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(solver=capi.SOLVER_BICG_ZLINE, precision=prec)
    bcv = mbc.boundary_1d(m, omega, 1)
    eg, rc = s.fwdsolve(bc=bcv)
    eo, rco = o.fwdsolve(bc=bcv)
    assert rc == 0 and rco == 0
    dg, do = s.diagnostics(), o.diagnostics()
    if prec == 0:
        k = min(12, len(do["EMrelErr"]), len(dg["EMrelErr"]))
        assert np.max(np.abs(dg["EMrelErr"][:k] - do["EMrelErr"][:k]) / do["EMrelErr"][:k]) < 1e-6
    em = earth_mask(g, m)
    assert relerr(eg[em], eo[em]) < 1e-5


# ---------------------------------------------------------------------------
# SP2 formulation (curl-curl + grad-div, no divergence correction)
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def gprob(cuda):
    from oracle.sp2 import SP2
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    ref = SP2(g, m)
    ref.set_freq(omega)
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(IterPerDivCor=120, MaxDivCor=20)
    return g, m, omega, ref, s


def test_ccgd_operator_matches_sp2(gprob):
    g, m, omega, ref, s = gprob
    rng = np.random.default_rng(0)
    xi = rng.standard_normal(s.nEi) + 1j * rng.standard_normal(s.nEi)
    assert relerr(s.mult_aii(xi), ref.A @ xi) < 1e-12


def test_ccgd_node_weights_match_sp2(gprob):
    """Signed grad-div node weights built on the device against the SP2
    restatement: -1/(sigma_N V_N) at earth nodes, 1/V_N at air nodes."""
    g, m, omega, ref, s = gprob
    _, _, w = s.get_cond()
    t = ref.topo
    want = np.where(ref.nearth, -1.0 / (ref.sig_n * t.Vnode), np.where(ref.nair, 1.0 / t.Vnode, 0.0))
    assert np.array_equal(w < 0, ref.nearth)
    assert np.max(np.abs(w - want) / np.max(np.abs(want))) < 1e-14


@pytest.mark.parametrize("prec", [0, 1])
def test_ccgd_forward_matches_sp2_and_ccdc(gprob, prec):
    g, m, omega, ref, s = gprob
    bcv = mbc.boundary_1d(m, omega, 2)
    s.set_control(IterPerDivCor=120, MaxDivCor=20, precision=prec)
    eg, rc = s.fwdsolve(bc=bcv)
    er, it, rerr, conv = ref.fwdsolve(bc=bcv)
    assert rc == 0 and conv
    em = earth_mask(g, m)
    assert relerr(eg[em], er[em]) < 1e-5
    assert s.diagnostics()["final_relres"] <= 1e-7
    # the same discrete solution as the divergence-corrected curl-curl system
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=BICG, precond=PC_JACOBI, tolEMfwd=1e-9)
    eo, rco = o.fwdsolve(bc=bcv)
    assert relerr(eg[em], eo[em]) < 1e-5


def test_ccgd_sources_match_sp2(gprob):
    g, m, omega, ref, s = gprob
    mask = interior_edge_mask(g)
    em = mask & earth_mask(g, m)
    rng = np.random.default_rng(6)
    src = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    s.set_control(IterPerDivCor=120, MaxDivCor=20, precision=capi.PREC_MIXED)
    for trans in (False, True):
        sv = src * ref.topo.Vedge if trans else src
        eg, rc = s.fwdsolve(trans=trans, src=sv)
        er, it, rerr, conv = ref.fwdsolve(trans=trans, src=sv)
        assert rc == 0 and conv
        assert relerr(eg[mask], er[mask]) < 1e-5


def test_restart_length_gives_the_same_solution(gprob):
    """The grad-div formulation without cuBiCG's 120-iteration restarts
    (restart only at cycle starts) converges to the same field."""
    g, m, omega, ref, s = gprob
    oms = np.array([omega, omega])
    bcs = np.stack([mbc.boundary_1d(m, omega, md) for md in (1, 2)])
    s.set_control(IterPerDivCor=300, MaxDivCor=20, precision=capi.PREC_MIXED)
    e120, st120, _ = s.fwdsolve_batch(oms, bc=bcs)
    s.set_restart(0)
    e0, st0, _ = s.fwdsolve_batch(oms, bc=bcs)
    it0, rr0 = s.batch_diagnostics(2)
    s.set_restart(120)
    s.set_control(IterPerDivCor=120, MaxDivCor=20, precision=capi.PREC_FP64)
    assert np.all(st120 == 0) and np.all(st0 == 0) and np.all(rr0 <= 1e-7)
    mask = earth_mask(g, m)
    for r in range(2):
        assert relerr(e0[r][mask], e120[r][mask]) < 1e-5
    with pytest.raises(capi.MT3DError):
        s.set_restart(-1)


def test_mixed_cycles_fall_back_to_fp64(gprob):
    """Mixed precision with short (8-iteration) FP32 cycles, which do not
    always halve the FP64 residual, so right-hand sides may continue with FP64
    cycles; either way the batch must converge to the FP64 solution (1e-5 on
    earth edges) with a true residual <= 1e-7."""
    g, m, omega, ref, s = gprob
    oms = np.array([omega, omega])
    bcs = np.stack([mbc.boundary_1d(m, omega, md) for md in (1, 2)])
    s.set_control(IterPerDivCor=120, MaxDivCor=20, precision=capi.PREC_FP64)
    e64, st64, rc64 = s.fwdsolve_batch(oms, bc=bcs)
    s.set_control(IterPerDivCor=8, MaxDivCor=4000, precision=capi.PREC_MIXED)
    em_, st, rc = s.fwdsolve_batch(oms, bc=bcs)
    it, rr = s.batch_diagnostics(2)
    s.set_control(IterPerDivCor=120, MaxDivCor=20, precision=capi.PREC_FP64)
    assert rc64 == 0 and rc == 0 and np.all(st == 0)
    assert np.all(rr <= 1e-7)
    mask = earth_mask(g, m)
    for r in range(2):
        assert relerr(em_[r][mask], e64[r][mask]) < 1e-5


# ---------------------------------------------------------------------------
# Full_Impedance data functional (mt3d_impedance) against oracle/datafunc.py
# ---------------------------------------------------------------------------
def test_impedance_matches_oracle(prob):
    import torch
    from oracle import datafunc as df
    g, m, omega, o, s = prob
    origin = (-1000.0, -800.0, 0.0)
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir, origin)
    rng = np.random.default_rng(8)
    e1 = rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges)
    e2 = rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges)
    sites = np.column_stack([rng.uniform(c["xC"][2], c["xC"][g.nx - 1], 12),
                             rng.uniform(c["yC"][2], c["yC"][g.ny - 1], 12),
                             np.concatenate([np.zeros(8), rng.uniform(10.0, 400.0, 4)])])
    zo = df.impedance(c, omega, sites, e1, e2)
    zg = s.impedance(omega, sites, e1, e2, origin)
    assert relerr(zg, zo) < 1e-12
    d1, d2 = torch.from_numpy(e1).cuda(), torch.from_numpy(e2).cuda()
    zd = s.impedance(omega, sites, d1.data_ptr(), d2.data_ptr(), origin)
    assert relerr(zd, zo) < 1e-12


def test_impedance_of_halfspace_solution(cuda):
    """Both polarisations solved on a 30 ohm-m halfspace at 10 Hz: Zxx = Zyy = 0,
    Zxy = -Zyx, and |Zxy| = sqrt(omega rho / mu0) with phase 45 degrees, to the
    grid's discretisation error (5 % in modulus, 3 degrees in phase)."""
    g = small_grid()
    rho = 30.0
    m = models.halfspace_model(g, rho)
    omega = 2 * np.pi * 10.0
    s = capi.Solver(g)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(tolEMfwd=1e-9)
    e = [s.fwdsolve(bc=mbc.boundary_1d(m, omega, mode))[0] for mode in (1, 2)]
    from oracle import datafunc as df
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir)
    sites = np.array([[c["xC"][5], c["yC"][6], 0.0], [c["xC"][4] + 50.0, c["yC"][7] - 30.0, 0.0]])
    Z = s.impedance(omega, sites, e[0], e[1])
    mu0 = 4e-7 * np.pi
    zabs = np.sqrt(omega * rho / mu0)
    for z in Z:
        assert abs(z[0, 0]) < 1e-6 * zabs and abs(z[1, 1]) < 1e-6 * zabs
        assert abs(z[0, 1] + z[1, 0]) < 1e-6 * zabs
        assert abs(abs(z[0, 1]) / zabs - 1) < 0.05
        ph = np.degrees(np.angle(z[0, 1])) % 180.0
        assert min(abs(ph - 45.0), abs(ph - 135.0)) < 3.0
    zo = df.impedance(c, omega, sites, e[0], e[1])
    assert relerr(Z, zo) < 1e-12


def test_lmult_t_matches_oracle(prob):
    import torch
    from oracle import datafunc as df
    g, m, omega, o, s = prob
    origin = (-1000.0, -800.0, 0.0)
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir, origin)
    rng = np.random.default_rng(12)
    e1 = rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges)
    e2 = rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges)
    sites = np.column_stack([rng.uniform(c["xC"][2], c["xC"][g.nx - 1], 6),
                             rng.uniform(c["yC"][2], c["yC"][g.ny - 1], 6), np.zeros(6)])
    d = rng.standard_normal((6, 2, 2)) + 1j * rng.standard_normal((6, 2, 2))
    o1, o2 = df.lmult_t(c, omega, sites, e1, e2, d)
    g1, g2 = s.lmult_t(omega, sites, e1, e2, d, origin)
    assert relerr(g1, o1) < 1e-12 and relerr(g2, o2) < 1e-12
    t1, t2 = torch.from_numpy(e1).cuda(), torch.from_numpy(e2).cuda()
    u1 = torch.full((g.n_edges,), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    u2 = u1.clone()
    s.lmult_t_device(omega, sites, t1.data_ptr(), t2.data_ptr(), d, u1.data_ptr(), u2.data_ptr(), origin)
    torch.cuda.synchronize()
    assert relerr(u1.cpu().numpy(), o1) < 1e-12 and relerr(u2.cpu().numpy(), o2) < 1e-12

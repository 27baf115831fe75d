"""CPU tests of the oracle (the checker of the CUDA path).

The oracle restates ModEM's matrix-free operator and solver.  These tests pin
it independently of its own code: against the SP2 sparse-matrix construction
of the same operator, against direct sparse solves, against the closed-form
solution of a layered model, and against the reference's own identities
(symmetry of the operator; AdjtBC = A_IB^T; PmultT = transpose of Pmult,
the Stest-style check of f90/SENS/SymmetryTest.f90:205-272).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from helpers import assemble_A, assemble_cc, direct_solve, earth_mask, edge_volumes, random_model, relerr, small_grid
from mt3d import bc as mbc
from mt3d import models
from oracle.oracle import BICG, PC_DILU, PC_JACOBI, QMR, Oracle, interior_edge_mask


@pytest.fixture(scope="module")
def setup():
    g = small_grid()
    m = random_model(g, seed=3)
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    omega = 2 * np.pi * 0.5
    o.update_freq(omega)
    return g, m, o, omega


def test_edge_conductivity_matches_numpy(setup):
    g, m, o, _ = setup
    assert np.allclose(o.sigE, mbc.edge_conductivity(m), rtol=1e-14, atol=0)


def test_edge_volume(setup):
    g, m, o, _ = setup
    assert np.allclose(o.VE, edge_volumes(g), rtol=1e-15)


def test_stencil_matches_sparse_assembly(setup):
    g, m, o, omega = setup
    A = assemble_A(g, m, omega)
    mask = interior_edge_mask(g)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges)
    y = o.multA(x)
    yref = A @ x
    assert relerr(y[mask], yref[mask]) < 1e-13
    assert np.all(y[~mask] == 0)


def test_operator_complex_symmetric_and_adjoint(setup):
    g, m, o, _ = setup
    mask = interior_edge_mask(g)
    rng = np.random.default_rng(1)
    x = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    y = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    # A^T = A on the interior system
    assert abs(y @ o.multA(x) - x @ o.multA(y)) < 1e-12 * abs(y @ o.multA(x))
    # conjugate transpose: <y, A x> = <A^H y, x>
    lhs = np.vdot(y, o.multA(x))
    rhs = np.vdot(o.multA(y, adjt=True), x)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_layered_model_closed_form():
    g = small_grid()
    m = models.halfspace_model(g, 30.0)
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    omega = 2 * np.pi * 0.1
    o.update_freq(omega)
    o.set_control(solver=BICG, precond=PC_JACOBI, tolEMfwd=1e-10)
    for mode in (1, 2):
        e, rc = o.fwdsolve(bc=mbc.boundary_1d(m, omega, mode))
        assert rc == 0
        ref = mbc.layered_solution(m, omega, mode)
        assert relerr(e, ref) < 1e-7


@pytest.mark.parametrize("solver,pc", [(QMR, PC_DILU), (BICG, PC_DILU), (BICG, PC_JACOBI)])
def test_fwdsolve_matches_direct_solve(setup, solver, pc):
    g, m, o, omega = setup
    bcv = mbc.boundary_1d(m, omega, 2)
    edir, _ = direct_solve(g, m, omega, bcv)
    o.set_control(solver=solver, precond=pc, tolEMfwd=1e-9)
    e, rc = o.fwdsolve(bc=bcv)
    assert rc == 0
    em = earth_mask(g, m)
    assert relerr(e[em], edir[em]) < 1e-6
    d = o.diagnostics()
    assert d["nDivCor"] >= 1 and d["EMrelErr"][-1] < 1e-9


def test_bicg_rhs_equals_minus_aib_bc(setup):
    g, m, o, omega = setup
    bcv = mbc.boundary_1d(m, omega, 1)
    mask = interior_edge_mask(g)
    A = assemble_A(g, m, omega)
    b_ref = -(A[mask][:, ~mask] @ bcv[~mask])
    b = -o.multA(np.where(mask, 0, bcv))[mask]
    assert relerr(b, b_ref) < 1e-13


def test_adjt_bc_is_transpose_of_aib(setup):
    """AdjtBC(e) computes A_IB^T e for the curl-curl part (AdjtBC comment,
    f90/3D_MT/FWD/modelOperator3D.f90:920-943); only boundary edges that are
    not shared by two faces are well defined through the face arrays."""
    g, m, o, omega = setup
    mask = interior_edge_mask(g)
    cc = assemble_cc(g)
    VE = edge_volumes(g)
    rng = np.random.default_rng(5)
    e = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    # AdjtBC works on the unsymmetric Maxwell coefficients: its input in the
    # reference is V_E*e, and (V_E^-1 CC)_IB^T V_E e = CC_BI e
    got = o.adjt_bc(VE * e)
    ref = cc[~mask][:, mask] @ e[mask]
    gb = got[~mask]
    # edges on face intersections are forced to zero by the reference
    sel = gb != 0
    assert sel.sum() > 0.5 * gb.size
    assert relerr(gb[sel], ref[sel]) < 1e-12


def test_transpose_solve_identity(setup):
    """Stest-style identity (f90/SENS/SymmetryTest.f90:205-272): for the
    interior system S = A_II^-1, b2^T S b1 = b1^T S^T b2 with S^T from the
    transposed solve (FWDsolve3D with TRN)."""
    g, m, o, omega = setup
    mask = interior_edge_mask(g)
    VE = o.VE
    rng = np.random.default_rng(11)
    # sources on earth edges only: the air part of A_II^-1 is fixed only up to
    # gradients, which such sources do not see
    em = mask & earth_mask(g, m)
    s1 = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    s2 = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    o.set_control(solver=QMR, precond=PC_DILU, tolEMfwd=1e-9, tolEMadj=1e-9, tolDivCor=1e-8)
    # forward solve with interior source s1 (b = V_E s1), transposed solve with source V_E s2
    e1, rc1 = o.fwdsolve(trans=False, src=s1)
    e2, rc2 = o.fwdsolve(trans=True, src=VE * s2)
    assert rc1 == 0 and rc2 == 0
    # transposed solution is V_E-weighted on output (EMsolve3D.f90:356-359)
    lhs = (VE * s2)[mask] @ e1[mask]
    rhs = (VE * s1)[mask] @ (e2[mask] / VE[mask])
    assert abs(lhs - rhs) < 1e-6 * abs(lhs)


def test_pmult_t_is_transpose_of_linearised_map(setup):
    """<dm, PmultT(e0, ea)> = Re sum(ea * (i mu0 w dsigma_E(dm)) * e0): the
    sigma gradient is the transpose of the linearised ModelParamToEdge
    (ModelMap.inc:88-188 with m0) scaled by i*omega*mu0 (SolverSens.f90:63-116)."""
    g, m, o, omega = setup
    rng = np.random.default_rng(7)
    e0 = rng.standard_normal((2, g.n_edges)) + 1j * rng.standard_normal((2, g.n_edges))
    ea = rng.standard_normal((2, g.n_edges)) + 1j * rng.standard_normal((2, g.n_edges))
    dm = rng.standard_normal(g.nx * g.ny * g.nzEarth)
    grad = o.pmult_t(e0, ea, m.m_earth)
    dsig = o.model_to_edge(dm, m.air_cond, m0_earth=m.m_earth)
    lin = np.real(np.sum(ea * (1j * models.MU_0 * omega * dsig) * e0))
    assert abs(grad @ dm - lin) < 1e-10 * abs(lin)


def test_divcorr_reduces_divergence(setup):
    g, m, o, omega = setup
    o.set_control(solver=BICG, precond=PC_JACOBI, tolEMfwd=1e-7)
    e, rc = o.fwdsolve(bc=mbc.boundary_1d(m, omega, 1))
    d = o.diagnostics()
    assert np.all(d["divJ"][:, 1] <= d["divJ"][:, 0])


def test_sp2_restatement_matches_ccdc():
    """The SP2 (curl-curl + grad-div) restatement reaches the same discrete
    solution as the divergence-corrected curl-curl oracle (the grad-div term
    vanishes at the solution, f90/3D_MT/FWD_SP2/modelOperator3D.f90:797-830)."""
    from oracle.sp2 import SP2
    g = small_grid()
    m = random_model(g, seed=3)
    w = 2 * np.pi * 0.5
    s = SP2(g, m)
    s.set_freq(w)
    assert abs(s.topo.CC - assemble_cc(g)).max() == 0.0
    bcv = mbc.boundary_1d(m, w, 2)
    e, it, rerr, conv = s.fwdsolve(bc=bcv)
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(w)
    o.set_control(solver=BICG, precond=PC_JACOBI, tolEMfwd=1e-9)
    eo, rc = o.fwdsolve(bc=bcv)
    em = earth_mask(g, m)
    assert conv and rc == 0 and relerr(e[em], eo[em]) < 1e-6


# ---------------------------------------------------------------------------
# Full_Impedance data functional (oracle/datafunc.py)
# ---------------------------------------------------------------------------
def _linear_fields(c, f):
    """Full edge vectors holding f(x, y, z) at the edge midpoints, per component."""
    from oracle import datafunc as df
    nx, ny, nz = c["n"]
    nE = nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz
    out = []
    for comp in (1, 2, 3):
        e = np.zeros(nE, complex)
        X = c["xC"] if comp == 1 else c["xE"]
        Y = c["yC"] if comp == 2 else c["yE"]
        Zc = c["zC"] if comp == 3 else c["zE"]
        ni, nj, nk = (nx if comp == 1 else nx + 1), (ny if comp == 2 else ny + 1), (nz if comp == 3 else nz + 1)
        for k in range(1, nk + 1):
            for j in range(1, nj + 1):
                for i in range(1, ni + 1):
                    e[df.flat(c, comp, i, j, k)] = f(X[i], Y[j], Zc[k])
        out.append(e)
    return out


def test_datafunc_interpolation_exact_for_linear_fields():
    from oracle import datafunc as df
    g = small_grid()
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir, origin=(-2000.0, -1500.0, 0.0))
    f = lambda X, Y, Z: 1.0 + 2e-3 * X - 1e-3 * Y + 5e-4 * Z
    ex, ey, _ = _linear_fields(c, f)
    rng = np.random.default_rng(4)
    for _ in range(10):
        x = np.array([rng.uniform(c["xC"][2], c["xC"][g.nx - 1]), rng.uniform(c["yC"][2], c["yC"][g.ny - 1]),
                      rng.uniform(-50.0, 300.0)])
        assert abs(df.apply(c, df.e_interp(c, x, 1), ex) - f(*x)) < 1e-12
        assert abs(df.apply(c, df.e_interp(c, x, 2), ey) - f(*x)) < 1e-12


def test_datafunc_b_is_curl_e_over_minus_i_omega():
    """E_y = a z, E_x = b z: (curl E)_x = -a, (curl E)_y = b, so B = (i ISIGN /
    omega) curl E exactly at any site."""
    from oracle import datafunc as df
    g = small_grid()
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir)
    a, b, omega = 3e-4, -2e-4, 2 * np.pi * 0.7
    ex, _, _ = _linear_fields(c, lambda X, Y, Z: b * Z)
    _, ey, _ = _linear_fields(c, lambda X, Y, Z: a * Z)
    e = ex + ey
    x = np.array([c["xC"][5] + 11.0, c["yC"][6] - 7.0, 0.0])
    bx = df.apply(c, df.b_from_e(c, omega, x, 1), e)
    by = df.apply(c, df.b_from_e(c, omega, x, 2), e)
    assert abs(bx - (-1j / omega) * (-a)) < 1e-12 * abs(a / omega)
    assert abs(by - (-1j / omega) * b) < 1e-12 * abs(b / omega)


def test_datafunc_lmult_t_is_the_derivative_of_z():
    """sum_k s_k . de_k = sum_ij conj(d_ij) dZ_ij for the adjoint sources of
    LmultT, dZ by central differences of the impedance functional."""
    from oracle import datafunc as df
    g = small_grid()
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir)
    rng = np.random.default_rng(6)
    nE = g.n_edges
    e1, e2, de1, de2 = (rng.standard_normal(nE) + 1j * rng.standard_normal(nE) for _ in range(4))
    sites = np.array([[c["xC"][4] + 10.0, c["yC"][5] + 20.0, 0.0], [c["xC"][6] - 30.0, c["yC"][7], 0.0]])
    omega = 2 * np.pi * 0.3
    d = rng.standard_normal((2, 2, 2)) + 1j * rng.standard_normal((2, 2, 2))
    s1, s2 = df.lmult_t(c, omega, sites, e1, e2, d)
    h = 1e-6
    zp = df.impedance(c, omega, sites, e1 + h * de1, e2 + h * de2)
    zm = df.impedance(c, omega, sites, e1 - h * de1, e2 - h * de2)
    dz = (zp - zm) / (2 * h)
    lhs = s1 @ de1 + s2 @ de2
    rhs = np.sum(np.conj(d) * dz)
    assert abs(lhs - rhs) < 1e-7 * abs(rhs)


def test_bc2d_layered_slices_equal_the_1d_column():
    """For a layered earth every 2-D TE slice of BC_x0_WS reduces to the 1-D TE
    column solution (the lateral terms cancel and the 2-D vertical terms equal
    Fwd1D_TE's), so E0 on each x-edge column equals fwd1d_te of that column."""
    from oracle import bc2d
    g = small_grid()
    rho = np.array([100.0, 30.0, 3.0, 300.0, 10.0, 10.0, 50.0, 50.0])
    m = np.broadcast_to(-np.log(rho)[None, None, :], (g.nx, g.ny, g.nzEarth))
    model = models.Model(g, models.flat_f(m))
    s = bc2d.sigma_cells(g, model.m_earth, model.air_cond)
    omega = 2 * np.pi * 0.7
    om2 = (2 * bc2d.PI_REF) / ((2 * bc2d.PI_REF) / omega)
    col = bc2d.fwd1d_te(om2, g.nzAir, np.asarray(g.dz, float), s[0, 0, g.nzAir:])
    for imode in (1, 2):
        e = bc2d.compute_bc(g, s, omega, imode)
        nX, nY = g.nx * (g.ny + 1) * (g.nz + 1), (g.nx + 1) * g.ny * (g.nz + 1)
        if imode == 2:
            f = e[:nX].reshape(g.nx, g.ny + 1, g.nz + 1, order="F")
        else:
            f = e[nX:nX + nY].reshape(g.nx + 1, g.ny, g.nz + 1, order="F")
        want = np.broadcast_to(col[:g.nz], f[:, :, :g.nz].shape)
        assert np.max(np.abs(f[:, :, :g.nz] - want)) < 1e-10 * np.max(np.abs(col))
        assert np.all(f[:, :, g.nz] == 0)  # bottom face zeroed
        other = e[nX:] if imode == 2 else np.concatenate([e[:nX], e[nX + nY:]])
        assert np.all(other == 0)


def test_bc1d_halfspace_impedance():
    """Fwd1D_TE restated (oracle/bc2d.py) against the halfspace's analytic
    impedance: with E linear in the air, E / (dE/dz) at the surface times
    omega is sqrt(omega / (mu0 sigma)) in magnitude with a 45 degree phase."""
    from oracle import bc2d
    nza = 6
    air = 60.0 * 1.5 ** np.arange(nza)[::-1]
    earth = 10.0 * 1.08 ** np.arange(90)
    dz = np.concatenate([air, earth])
    sigma, f = 0.01, 1.0
    omega = 2 * np.pi * f
    e = bc2d.fwd1d_te(omega, nza, dz, np.full(earth.size, sigma))
    dedz = (e[nza] - e[nza - 1]) / dz[nza - 1]
    z = -omega * e[nza] / dedz  # z down: E decays with depth
    want = np.sqrt(omega / (bc2d.MU_0 * sigma))
    assert abs(abs(z) / want - 1) < 0.01
    assert abs(abs(np.degrees(np.angle(z))) - 45.0) < 1.0


def test_bc2d_contact_far_field_is_1d():
    """A 2-D TE slice with a vertical contact (0.1 S/m | 0.01 S/m): columns
    many skin depths away from the contact carry the 1-D solution of their own
    side (within 1e-3 of the surface field)."""
    from oracle import bc2d
    nza = 6
    dz = np.concatenate([60.0 * 1.5 ** np.arange(nza)[::-1], 20.0 * 1.12 ** np.arange(60)])
    dy = np.full(60, 2000.0)
    cond = np.empty((60, dz.size))
    cond[:30] = 0.1
    cond[30:] = 0.01
    omega = 2 * np.pi * 1.0
    e = bc2d.fwd2d_te(omega, nza, dy, dz, cond)
    for col, s in ((5, 0.1), (55, 0.01)):
        want = bc2d.fwd1d_te(omega, nza, dz, np.full(dz.size - nza, s))
        assert np.max(np.abs(e[col] - want)) < 1e-3 * abs(want[nza])
    # at the contact the field is neither side's 1-D one
    for s in (0.1, 0.01):
        want = bc2d.fwd1d_te(omega, nza, dz, np.full(dz.size - nza, s))
        assert abs(e[30, nza] - want[nza]) > 0.05 * abs(want[nza])


def test_oracle_chain_halfspace_impedance():
    """The oracle's own chain on a 30 ohm-m halfspace at 10 Hz: the 2-D
    boundary conditions (which reduce to 1-D here), the divergence-corrected
    QMR solve and the impedance functional give Zxx = Zyy = 0, Zxy = -Zyx and
    |Zxy| = sqrt(omega rho / mu0) at 45 degrees, within the grid's
    discretisation error (0.2 % between the polarisations, 5 % in modulus,
    3 degrees in phase)."""
    from oracle import bc2d
    from oracle import datafunc as df
    g = small_grid()
    rho = 30.0
    m = models.halfspace_model(g, rho)
    omega = 2 * np.pi * 10.0
    o = Oracle(g)
    o.update_cond(m.m_earth, m.air_cond)
    o.update_freq(omega)
    o.set_control(solver=QMR, precond=PC_DILU, tolEMfwd=1e-9)
    sig = bc2d.sigma_cells(g, m.m_earth, m.air_cond)
    e = []
    for imode in (1, 2):
        e0 = bc2d.compute_bc(g, sig, omega, imode)
        x, rc = o.fwdsolve(bc=e0, e0=e0)
        assert rc == 0
        e.append(x)
    c = df.coords(g.dx, g.dy, g.dz, g.nzAir)
    sites = np.array([[c["xC"][5], c["yC"][6], 0.0], [c["xC"][4] + 50.0, c["yC"][7] - 30.0, 0.0]])
    Z = df.impedance(c, omega, sites, e[0], e[1])
    zabs = np.sqrt(omega * rho / models.MU_0)
    for z in Z:
        assert abs(z[0, 0]) < 1e-6 * zabs and abs(z[1, 1]) < 1e-6 * zabs
        # the 1-D columns of BC_x0_WS close with a skin-depth layer and are not
        # the exact discrete 3-D solution, so the two polarisations agree to
        # the discretisation level only
        assert abs(z[0, 1] + z[1, 0]) < 2e-3 * zabs
        assert abs(abs(z[0, 1]) / zabs - 1) < 0.05
        ph = np.degrees(np.angle(z[0, 1])) % 180.0
        assert min(abs(ph - 45.0), abs(ph - 135.0)) < 3.0


def test_bc2d_modes_are_transposes_for_a_symmetric_model():
    """On a square grid with sigma(i, j, k) = sigma(j, i, k), the imode 1
    field on the y-edges is the imode 2 field on the x-edges with x and y
    swapped (BC_x0_WS treats both the same way)."""
    from oracle import bc2d
    g = models.make_grid(10, 10, 4, 8, core=400.0, n_pad=2, pad_growth=1.6, air_first=60.0, air_growth=2.0,
                         earth_first=60.0, earth_growth=1.4)
    rng = np.random.default_rng(4)
    a = rng.uniform(-5, 0, (g.nx, g.ny, g.nzEarth))
    a = 0.5 * (a + a.transpose(1, 0, 2))
    m = models.Model(g, models.flat_f(a))
    sig = bc2d.sigma_cells(g, m.m_earth, m.air_cond)
    omega = 2 * np.pi * 0.3
    e1 = bc2d.compute_bc(g, sig, omega, 1)
    e2 = bc2d.compute_bc(g, sig, omega, 2)
    nx, ny, nz = g.nx, g.ny, g.nz
    nX = nx * (ny + 1) * (nz + 1)
    ex = e2[:nX].reshape(nx, ny + 1, nz + 1, order="F")
    ey = e1[nX:2 * nX].reshape(nx + 1, ny, nz + 1, order="F")
    assert np.allclose(ey, ex.transpose(1, 0, 2), rtol=1e-12, atol=1e-14)


def gradient_problem():
    """Small gradient problem: 10 x 12 x 12 grid, data of a random 'true'
    model with 5 % noise at four surface sites and two frequencies, gradient
    at a second random model; boundary data held fixed (the sensitivity does
    not differentiate them)."""
    from oracle import sens
    from oracle.oracle import PC_DILU, QMR
    g = small_grid()
    true = random_model(g, seed=3)
    start = random_model(g, seed=4)
    freqs = np.array([0.5, 4.0])
    xe = np.concatenate([[0.0], np.cumsum(g.dx)])
    ye = np.concatenate([[0.0], np.cumsum(g.dy)])
    sites = np.array([[0.5 * (xe[i] + xe[i + 1]), 0.5 * (ye[j] + ye[j + 1]), 0.0] for j in (4, 7) for i in (3, 6)])
    bcs = [[mbc.boundary_1d(start, 2 * np.pi * f, p) for p in (1, 2)] for f in freqs]
    ctl = dict(solver=QMR, precond=PC_DILU, tolEMfwd=1e-10, tolEMadj=1e-10, MaxDivCor=200, tolDivCor=1e-10)
    Zt, _, _, _ = sens.predict(g, true, freqs, bcs, sites, ctl)
    rng = np.random.default_rng(1)
    err = 0.05 * np.abs(Zt).max(axis=(2, 3))[..., None, None] * np.ones(Zt.shape)
    d_obs = Zt + err * (rng.standard_normal(Zt.shape) + 1j * rng.standard_normal(Zt.shape)) / np.sqrt(2)
    cells = [(3, 4, 0), (6, 7, 1), (4, 5, 2), (5, 6, 3), (2, 8, 1), (7, 3, 4)]
    return g, start, freqs, bcs, sites, d_obs, err, ctl, [i + g.nx * (j + g.ny * k) for i, j, k in cells]


def test_oracle_misfit_gradient_matches_finite_differences():
    """The oracle's JmultT_TX chain (LmultT -> transposed solve -> PmultT,
    f90/SENS/SensComp.f90:408-488) summed into the misfit gradient of
    f90/INV/INVcore.f90:141-206 is the derivative of the misfit: central
    differences with step 1e-4 in ln(sigma) on six earth cells agree to
    1e-6 of the largest gradient entry (solves to relative residual 1e-10)."""
    from oracle import sens
    g, start, freqs, bcs, sites, d_obs, err, ctl, cells = gradient_problem()
    phi, grad = sens.misfit_gradient(g, start, freqs, bcs, sites, d_obs, err, ctl)
    h = 1e-4
    for c in cells:
        mp, mm = (models.Model(g, start.m_earth.copy(), start.air_cond) for _ in range(2))
        mp.m_earth[c] += h
        mm.m_earth[c] -= h
        fd = (sens.misfit(g, mp, freqs, bcs, sites, d_obs, err, ctl) -
              sens.misfit(g, mm, freqs, bcs, sites, d_obs, err, ctl)) / (2 * h)
        assert abs(fd - grad[c]) <= 1e-6 * np.abs(grad).max(), (c, fd, grad[c])

"""Direct checks of the internal operator kernels (through mt3d_apply_kernel)
and of the bounded-wait error path.

The BiCGStab stencils are otherwise only exercised through converged solves,
where an error that slows convergence without changing the answer would go
unseen.  Here each kernel applies the operator to a random field on a grid
that spans several tiles of the staged kernels in x (nx + 1 = 71: three
32-column tiles) and y (ny + 1 = 21: three 8-row tiles) and several chunks of
node planes (nz = 30), so every halo between tiles and chunks is read.  The
reference is the assembled sparse operator: the SP2 curl-curl construction of
tests/helpers.py for the divergence-corrected formulation (an independent
restatement, CurlCurlSetUp of f90/3D_MT/FWD_SP2/modelOperator3D.f90:371-405)
and oracle/sp2.py's CCGD operator for the grad-div formulation
(GradDivSetup2, :916-1008).

Tolerances:
  * FP64 kernels: relative 2-norm difference <= 1e-13 (summation order);
  * FP32 kernel: per edge |y32 - A x32| <= 64 * 2^-24 * (|A| |x|)_e, the
    forward-error bound of an FP32 sum of the stencil's terms (x32 is x
    rounded to FP32, as the kernel reads it), and relative 2-norm <= 1e-5.
"""
import numpy as np
import pytest

from helpers import assemble_A, random_model, relerr
from mt3d import capi, models
from oracle.oracle import interior_edge_mask

pytestmark = pytest.mark.gpu


def tiled_grid():
    return models.make_grid(70, 20, 8, 22, core=400.0, n_pad=4, pad_growth=1.5, air_first=60.0, air_growth=2.0,
                            earth_first=60.0, earth_growth=1.25)


@pytest.fixture(scope="module", params=[capi.FORM_CCDC, capi.FORM_CCGD], ids=["ccdc", "ccgd"])
def kprob(cuda, request):
    from oracle.sp2 import SP2
    g = tiled_grid()
    m = random_model(g, seed=11)
    omega = 2 * np.pi * 3.0
    mask = interior_edge_mask(g)
    if request.param == capi.FORM_CCGD:
        ref = SP2(g, m)
        ref.set_freq(omega)
        A = ref.A
    else:
        A = assemble_A(g, m, omega)[mask][:, mask].tocsr()
    s = capi.Solver(g)
    s.set_formulation(request.param)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(precision=capi.PREC_MIXED)
    rng = np.random.default_rng(5)
    x = np.zeros(g.n_edges, complex)
    x[mask] = rng.standard_normal(mask.sum()) + 1j * rng.standard_normal(mask.sum())
    return g, mask, A, s, x


def test_tiled_grid_spans_tiles_and_chunks():
    g = tiled_grid()
    assert (g.nx + 1 + 31) // 32 >= 3 and (g.ny + 1 + 7) // 8 >= 2 and g.nz + 1 >= 24


@pytest.mark.parametrize("kernel", [0, 1])
def test_fp64_kernels_match_assembled_operator(kprob, kernel):
    g, mask, A, s, x = kprob
    y = s.apply_kernel(kernel, x)
    assert np.all(y[~mask] == 0)
    assert relerr(y[mask], A @ x[mask]) < 1e-13


def test_fp32_tma_stencil_matches_assembled_operator(kprob):
    g, mask, A, s, x = kprob
    y = s.apply_kernel(2, x)
    x32 = x.astype(np.complex64).astype(np.complex128)
    want = A @ x32[mask]
    bound = 64 * 2.0 ** -24 * (abs(A) @ np.abs(x32[mask]))
    err = np.abs(y[mask] - want)
    worst = int(np.argmax(err / bound))
    assert np.all(err <= bound), (worst, err[worst], bound[worst])
    assert relerr(y[mask], want) < 1e-5
    assert np.all(y[~mask] == 0)


def test_fused_stencil_is_preconditioned_operator(kprob):
    """The operator kernel of the fused FP32 iteration returns D^-1 A x with
    D = diag(A): the FP32 stencil bound above, divided per edge by |D|."""
    g, mask, A, s, x = kprob
    y = s.apply_kernel(3, x)
    x32 = x.astype(np.complex64).astype(np.complex128)
    D = A.diagonal()
    want = (A @ x32[mask]) / D
    bound = 64 * 2.0 ** -24 * (abs(A) @ np.abs(x32[mask])) / np.abs(D)
    err = np.abs(y[mask] - want)
    worst = int(np.argmax(err / bound))
    assert np.all(err <= bound), (worst, err[worst], bound[worst])
    assert np.all(y[~mask] == 0)


@pytest.mark.parametrize("formulation", [capi.FORM_CCDC, capi.FORM_CCGD], ids=["ccdc", "ccgd"])
def test_fused_and_unfused_iterations_reach_the_same_solution(cuda, formulation):
    """Mixed precision with the fused FP32 iteration (preconditioned
    variables, pseudo-random shadow) and with the unfused one: both reach the
    FP64 tolerance and the same field within it (relative 2-norm 1e-5 on the
    edges where the field is unique)."""
    from helpers import earth_mask
    from mt3d import bc as mbc
    g = tiled_grid()
    m = random_model(g, seed=11)
    omega = 2 * np.pi * 3.0
    bcv = mbc.boundary_1d(m, omega, 1)
    out = []
    for fused in (True, False):
        s = capi.Solver(g)
        s.set_formulation(formulation)
        s.update_cond(m.m_earth, m.air_cond)
        s.update_freq(omega)
        s.set_control(IterPerDivCor=200, MaxDivCor=40, tolEMfwd=1e-8, precision=capi.PREC_MIXED)
        s.set_fused(fused)
        e, rc = s.fwdsolve(bc=bcv)
        d = s.diagnostics()
        assert rc == 0 and d["final_relres"] <= 1e-8
        out.append(e)
    em = earth_mask(g, m)
    assert relerr(out[0][em], out[1][em]) < 1e-5


def test_ccgd_transposed_product_matches_sp2(cuda):
    """mt3d_mult_aii(adjt=1) in the grad-div formulation is Mult_Aii(adjt):
    AAii^T x - i ISIGN VomegaMuSig x (f90/3D_MT/FWD_SP2/modelOperator3D.f90:
    415-436), with the unsymmetric grad-div term transposed."""
    from helpers import small_grid
    from oracle.sp2 import SP2
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    ref = SP2(g, m)
    ref.set_freq(omega)
    asym = abs(ref.AAii - ref.AAii.T).max() / abs(ref.AAii).max()
    assert asym > 1e-3  # the grad-div term makes AAii unsymmetric
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    rng = np.random.default_rng(2)
    xi = rng.standard_normal(s.nEi) + 1j * rng.standard_normal(s.nEi)
    want = ref.AAii.T @ xi - 1j * (-1) * ref.vwms * xi
    assert relerr(s.mult_aii(xi, adjt=True), want) < 1e-12
    assert relerr(s.mult_aii(xi), ref.A @ xi) < 1e-12


def test_bounded_wait_reports_timeout_and_recovers(cuda):
    """A wait limit of zero polls makes the FP32 stencil's mbarrier waits give
    up on a valid problem (after the block has waited, under the default
    limit, for the copies it issued): the call returns MT3D_DEVICE_TIMEOUT,
    and after the default limit is restored the same handle solves normally.
    Both FP32 iterations (fused and unfused) are covered."""
    from helpers import small_grid
    from mt3d import bc as mbc
    g = small_grid()
    m = random_model(g, seed=3)
    omega = 2 * np.pi * 0.5
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    s.set_control(IterPerDivCor=100, MaxDivCor=20, precision=capi.PREC_MIXED)
    bcv = mbc.boundary_1d(m, omega, 1)
    for fused in (True, False):
        s.set_fused(fused)
        s.set_wait_limit(0)
        with pytest.raises(capi.MT3DError) as ei:
            s.fwdsolve(bc=bcv)
        assert ei.value.code == 6
        s.set_wait_limit(1 << 22)
        e, rc = s.fwdsolve(bc=bcv)
        assert rc == 0
        assert s.diagnostics()["final_relres"] <= 1e-7


@pytest.mark.parametrize("formulation", [capi.FORM_CCDC, capi.FORM_CCGD], ids=["ccdc", "ccgd"])
def test_polynomial_preconditioner_reaches_the_same_solution(cuda, formulation):
    """The fused FP32 iteration with the polynomial preconditioner
    c D^-1 (2 I - c A D^-1) (mt3d_set_poly, c = 0.8) and with the diagonal
    one: both reach the FP64 tolerance 1e-8 and the same field within it
    (relative 2-norm 1e-5 on the edges where the field is unique)."""
    from helpers import earth_mask
    from mt3d import bc as mbc
    g = tiled_grid()
    m = random_model(g, seed=11)
    omega = 2 * np.pi * 3.0
    bcv = mbc.boundary_1d(m, omega, 2)
    out, its = [], []
    for c in (0.0, 0.8):
        s = capi.Solver(g)
        s.set_formulation(formulation)
        s.update_cond(m.m_earth, m.air_cond)
        s.update_freq(omega)
        s.set_control(IterPerDivCor=200, MaxDivCor=40, tolEMfwd=1e-8, precision=capi.PREC_MIXED)
        s.set_poly(c)
        e, rc = s.fwdsolve(bc=bcv)
        d = s.diagnostics()
        assert rc == 0 and d["final_relres"] <= 1e-8
        out.append(e)
        its.append(d["nIterTotal"])
    print(f"formulation {formulation}: iterations diagonal {its[0]}, polynomial {its[1]}")
    em = earth_mask(g, m)
    assert relerr(out[0][em], out[1][em]) < 1e-5


def test_polynomial_coefficient_range(cuda):
    s = capi.Solver(tiled_grid())
    for bad in (-0.1, 1.6, float("nan")):
        with pytest.raises(capi.MT3DError):
            s.set_poly(bad)
    s.set_poly(1.0)
    s.set_poly(0.0)

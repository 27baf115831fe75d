"""Ragged batches on the GPU: right-hand sides that are zero sit in a batch
beside ones that are not, as a batch of (frequency, polarisation, forward /
adjoint) solves can hold them (an adjoint right-hand side of a polarisation
with no data, a forward one without boundary data).

The reference's Krylov call returns a zero solution for a zero right-hand
side without iterating and reports one iteration with relative residual 0
(`bnorm .eq. 0.0`, f90/3D_MT/FWD_SP2/solver.f90:780-786); a transposed
problem without a source returns a zero solution before any Krylov call
(f90/3D_MT/FWD_SP2/EMsolve3D.f90:233-245).  So: those rows come back exactly
zero with status 0 and those iteration counts (1 and 0), a batch of nothing
but such rows returns at once, and the other rows equal the same right-hand
sides solved
one at a time (bitwise for FP64, whose kernels reduce each right-hand side
on its own; within the 1e-5 solution bound of the parity tests for the mixed
path, whose FP32 cycles may run in different batch shapes).  Both the
reference's formulation (FP64) and the benchmark's configuration (grad-div,
mixed precision, fused iteration with the polynomial preconditioner) run.
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, relerr, small_grid
from mt3d import bc as mbc
from mt3d import capi
from oracle.oracle import interior_edge_mask

pytestmark = pytest.mark.gpu

CONFIGS = {
    "ccdc-fp64": dict(formulation=capi.FORM_CCDC, precision=capi.PREC_FP64, poly=0.0),
    "ccgd-mixed-poly": dict(formulation=capi.FORM_CCGD, precision=capi.PREC_MIXED, poly=0.9),
}


def _solver(g, m, cfg):
    s = capi.Solver(g)
    s.set_formulation(cfg["formulation"])
    s.set_fused(True)
    s.set_poly(cfg["poly"])
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=100, MaxDivCor=100, tolEMfwd=1e-8, tolEMadj=1e-8, precision=cfg["precision"])
    return s


@pytest.mark.parametrize("name", list(CONFIGS))
def test_zero_rows_in_a_batch(cuda, name):
    cfg = CONFIGS[name]
    g = small_grid()
    m = random_model(g, seed=6)
    s = _solver(g, m, cfg)
    w1, w2 = 2 * np.pi * 0.5, 2 * np.pi * 0.02
    mask = interior_edge_mask(g) & earth_mask(g, m)
    rng = np.random.default_rng(21)
    src = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    zero = np.zeros(s.nE, complex)
    # rows: forward with data, zero forward, adjoint with a source, adjoint
    # without a source, forward with data at another frequency
    oms = np.array([w1, w1, w1, w2, w2])
    trans = np.array([0, 0, 1, 1, 0], np.int32)
    bcs = np.stack([mbc.boundary_1d(m, w1, 1), zero, zero, zero, mbc.boundary_1d(m, w2, 2)])
    srcs = np.stack([zero, zero, src, zero, zero])
    e, st, rc = s.fwdsolve_batch(oms, trans=trans, bc=bcs, src=srcs)
    it, rr = s.batch_diagnostics(len(oms))
    assert rc == 0 and np.all(st == 0), st
    for r, n in ((1, 1), (3, 0)):
        assert np.all(e[r] == 0) and it[r] == n and rr[r] == 0.0, (r, it[r], rr[r])
    bound = 1e-12 if cfg["precision"] == capi.PREC_FP64 else 1e-5
    for r in (0, 2, 4):
        assert np.abs(e[r]).max() > 0
        s.update_freq(oms[r])
        e1, rc1 = s.fwdsolve(trans=bool(trans[r]), bc=bcs[r], src=srcs[r])
        assert rc1 == 0
        err = relerr(e[r], e1)
        print(f"{name} row {r}: batch vs single {err:.2e}, iterations {it[r]}")
        assert err <= bound


@pytest.mark.parametrize("name", list(CONFIGS))
def test_batch_of_zero_rows_only(cuda, name):
    cfg = CONFIGS[name]
    g = small_grid()
    m = random_model(g, seed=6)
    s = _solver(g, m, cfg)
    n = 3
    oms = np.full(n, 2 * np.pi * 0.5)
    trans = np.array([0, 1, 0], np.int32)
    e0 = np.ones((n, s.nE), complex)  # a first guess the zero solution must overwrite
    e, st, rc = s.fwdsolve_batch(oms, trans=trans, bc=np.zeros((n, s.nE), complex),
                                 src=np.zeros((n, s.nE), complex), e0=e0)
    it, rr = s.batch_diagnostics(n)
    assert rc == 0 and np.all(st == 0)
    assert np.all(e == 0) and it.tolist() == [1, 0, 1] and np.all(rr == 0.0)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_nan_row_leaves_the_others_alone(cuda, name):
    """A row whose source holds a NaN is reported with status 3 (the
    reference stops on `isnan(bnorm)`, f90/3D_MT/FWD_SP2/solver.f90:776-779;
    a library must not stop its host) and the call returns 3; the rows beside
    it still equal their single solves (each row's inner products are its
    own, so a NaN cannot reach them)."""
    cfg = CONFIGS[name]
    g = small_grid()
    m = random_model(g, seed=6)
    s = _solver(g, m, cfg)
    w = 2 * np.pi * 0.5
    mask = interior_edge_mask(g) & earth_mask(g, m)
    rng = np.random.default_rng(22)
    src = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    bad = src.copy()
    bad[np.flatnonzero(mask)[5]] = np.nan
    zero = np.zeros(s.nE, complex)
    oms = np.full(3, w)
    trans = np.array([0, 1, 1], np.int32)
    bcs = np.stack([mbc.boundary_1d(m, w, 1), zero, zero])
    srcs = np.stack([zero, bad, src])
    e, st, rc = s.fwdsolve_batch(oms, trans=trans, bc=bcs, src=srcs)
    assert rc == 3 and st.tolist() == [0, 3, 0], st
    s.update_freq(w)
    for r in (0, 2):
        e1, rc1 = s.fwdsolve(trans=bool(trans[r]), bc=bcs[r], src=srcs[r])
        assert rc1 == 0
        err = relerr(e[r], e1)
        print(f"{name} row {r} beside a NaN row: batch vs single {err:.2e}")
        assert err <= (1e-12 if cfg["precision"] == capi.PREC_FP64 else 1e-5)


def test_batch_larger_than_the_launch_limit_is_refused(cuda):
    """More right-hand sides than a launch grid's y extent (65535) are
    refused with MT3D_INVALID_ARGUMENT before any buffer is read (the
    device buffer given here holds one edge vector only)."""
    import torch
    g = small_grid()
    m = random_model(g, seed=6)
    s = _solver(g, m, CONFIGS["ccgd-mixed-poly"])
    e = torch.zeros(s.nE, dtype=torch.complex128, device="cuda")
    with pytest.raises(capi.MT3DError) as ei:
        s.fwdsolve_batch_device(np.full(65536, 2 * np.pi), e.data_ptr())
    assert ei.value.code == 5 and "65535" in str(ei.value)
    st, rc = s.fwdsolve_batch_device(np.array([2 * np.pi]), e.data_ptr(), bc_ptr=None)
    assert rc == 0  # the handle stays usable (a zero right-hand side)

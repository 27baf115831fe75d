"""The solves do not read device memory that they did not write first.

A handle's workspace comes from cudaMalloc, which hands back whatever the
memory last held.  A kernel that read such memory before writing it (a
padding slot of the FP32 layout, a vector of the previous cycle, a partial
sum of another batch shape) would make results depend on earlier work in the
process, and a NaN left there would turn up as a rare failed solve.  So the
test fills most of the device's free memory with NaN (and then with 1e300),
returns it to the driver, creates a fresh handle, whose allocations come
from that memory, and requires the fields, statuses and iteration counts of
a batch to be bitwise those of a handle created on clean memory.  Both the
benchmark's configuration (grad-div, mixed precision, polynomial
preconditioner) and the reference's (curl-curl + divergence correction,
FP64) run; forward and adjoint right-hand sides of two frequencies.
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, small_grid
from mt3d import bc as mbc
from mt3d import capi
from oracle.oracle import interior_edge_mask

pytestmark = pytest.mark.gpu

CONFIGS = {
    "ccgd-mixed-poly": (capi.FORM_CCGD, capi.PREC_MIXED, 0.9),
    "ccdc-fp64": (capi.FORM_CCDC, capi.PREC_FP64, 0.0),
}


def _poison(value):
    import torch
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    x = torch.empty(int(free * 0.9) // 8, dtype=torch.float64, device="cuda")
    x.fill_(value)
    torch.cuda.synchronize()
    del x
    torch.cuda.empty_cache()


def _solve(g, m, cfg, oms, trans, bcs, srcs):
    s = capi.Solver(g)
    s.set_formulation(cfg[0])
    s.set_restart(0)
    s.set_fused(True)
    s.set_poly(cfg[2])
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=100, MaxDivCor=100, tolEMfwd=1e-8, tolEMadj=1e-8, precision=cfg[1])
    e, st, rc = s.fwdsolve_batch(oms, trans=trans, bc=bcs, src=srcs)
    it, rr = s.batch_diagnostics(len(oms))
    s.close()
    return e, st, rc, it, rr


@pytest.mark.parametrize("name", list(CONFIGS))
def test_results_do_not_depend_on_stale_device_memory(cuda, name):
    cfg = CONFIGS[name]
    g = small_grid()
    m = random_model(g, seed=8)
    w1, w2 = 2 * np.pi * 0.5, 2 * np.pi * 0.02
    mask = interior_edge_mask(g) & earth_mask(g, m)
    rng = np.random.default_rng(23)
    src = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    zero = np.zeros(g.n_edges, complex)
    oms = np.array([w1, w2, w1, w2])
    trans = np.array([0, 0, 1, 1], np.int32)
    bcs = np.stack([mbc.boundary_1d(m, w1, 1), mbc.boundary_1d(m, w2, 2), zero, zero])
    srcs = np.stack([zero, zero, src, 0.5 * src])
    e0, st0, rc0, it0, rr0 = _solve(g, m, cfg, oms, trans, bcs, srcs)
    assert rc0 == 0 and np.all(st0 == 0)
    for value in (float("nan"), 1e300):
        _poison(value)
        e, st, rc, it, rr = _solve(g, m, cfg, oms, trans, bcs, srcs)
        assert rc == 0 and np.array_equal(st, st0) and np.array_equal(it, it0), (value, it, it0)
        assert np.array_equal(e, e0) and np.array_equal(rr, rr0), value

"""The allocation-free operator product on device vectors
(mt3d_mult_aii_device_noalloc) against the host entry mt3d_mult_aii.

The entry serves callers that cannot allocate device memory per call (a
memory pool that owns all free memory, or a loop that must not meet the
device-wide synchronisation of cudaMalloc/cudaFree).  So the test calls it
first, on a freshly created handle whose workspace has never been allocated,
and checks that those calls make no device allocation: the library's own
allocation counter (every cudaMalloc it makes) stays put, and so does the
device's free memory.  The references come from mt3d_mult_aii on a second
handle, itself checked against the oracle and the SP2 restatement in the
parity tests.  Both run the same FP64 kernels on the same inputs, so the
bound is the operator tolerance of those tests: relative 2-norm difference
<= 1e-13.  Two calls in a row on one stream (different inputs) check that
the fixed scratch is re-initialised on every call.  This file is collected
last so that it also runs after every other GPU test in the same process.
"""
import numpy as np
import pytest
import torch

from helpers import random_model, relerr, small_grid
from mt3d import capi, models

pytestmark = pytest.mark.gpu

TOL = 1e-13


def _solver(g, m, omega, formulation):
    s = capi.Solver(g)
    s.set_formulation(formulation)
    s.update_cond(m.m_earth, m.air_cond)
    s.update_freq(omega)
    return s


@pytest.mark.parametrize("formulation", [capi.FORM_CCDC, capi.FORM_CCGD])
@pytest.mark.parametrize("adjt", [False, True])
def test_noalloc_matches_mult_aii(cuda, formulation, adjt):
    g = small_grid()
    m = random_model(g, seed=5)
    omega = 2 * np.pi * 0.3
    ref = _solver(g, m, omega, formulation)
    rng = np.random.default_rng(11)
    xs = [rng.standard_normal(ref.nEi) + 1j * rng.standard_normal(ref.nEi) for _ in range(2)]
    refs = [ref.mult_aii(x, adjt=adjt) for x in xs]
    xd = [torch.from_numpy(x).to("cuda") for x in xs]
    yd = [torch.full((ref.nEi,), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda") for _ in xs]
    s = _solver(g, m, omega, formulation)  # fresh handle: no workspace yet
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    L = capi.load()
    allocs0 = L.mt3d_alloc_counter()
    free0 = torch.cuda.mem_get_info()[0]
    for x, y in zip(xd, yd):  # two calls in a row on one stream
        s.mult_aii_device_noalloc(x.data_ptr(), y.data_ptr(), adjt=adjt)
    torch.cuda.synchronize()
    assert L.mt3d_alloc_counter() == allocs0
    assert torch.cuda.mem_get_info()[0] == free0
    for y, want in zip(yd, refs):
        got = y.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert relerr(got, want) <= TOL


def test_noalloc_rejects_large_grid_and_host_memory(cuda):
    g = small_grid()
    m = random_model(g, seed=5)
    s = _solver(g, m, 2 * np.pi * 0.3, capi.FORM_CCDC)
    x = np.zeros(s.nEi, np.complex128)
    with pytest.raises(capi.MT3DError) as ei:
        s.mult_aii_device_noalloc(x.ctypes.data, x.ctypes.data)
    assert ei.value.code == 5 and "device memory" in str(ei.value)
    big = models.make_grid(60, 60, 8, 52)
    mb = random_model(big, seed=1)
    sb = _solver(big, mb, 2 * np.pi, capi.FORM_CCDC)
    xb = torch.zeros(sb.nEi, dtype=torch.complex128, device="cuda")
    with pytest.raises(capi.MT3DError) as ei:
        sb.mult_aii_device_noalloc(xb.data_ptr(), xb.data_ptr())
    assert ei.value.code == 5 and "scratch" in str(ei.value)

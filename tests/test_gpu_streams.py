"""Stream ordering of the device entries.

A caller that fills device buffers on the legacy default stream (torch's
default stream, whose handle is 0, as the runtime's is) and then calls a
device entry of a handle that runs on its own stream must get a solve of
the filled buffers.  The handle's own stream is a blocking stream, so it
waits for work the caller queued on the default stream: the test delays that
stream with a bounded spin kernel, queues the zeroing of the first guess
behind it, calls mt3d_fwdsolve_batch_device at once, and requires the fields
to equal, bit for bit, those of the same solve from a first guess zeroed and
synchronised beforehand.  (With an unordered stream the solve would start
from the stale buffer, here all ones, and return other fields.)
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, small_grid
from mt3d import bc as mbc
from mt3d import capi
from oracle.oracle import interior_edge_mask

pytestmark = pytest.mark.gpu


def test_own_stream_waits_for_the_default_stream(cuda):
    import torch
    g = small_grid()
    m = random_model(g, seed=9)
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.set_poly(0.9)
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=100, MaxDivCor=100, tolEMfwd=1e-8, tolEMadj=1e-8, precision=capi.PREC_MIXED)
    w = 2 * np.pi * 0.5
    mask = interior_edge_mask(g) & earth_mask(g, m)
    rng = np.random.default_rng(24)
    src = np.where(mask, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0)
    zero = np.zeros(g.n_edges, complex)
    oms = np.array([w, w])
    trans = np.array([0, 1], np.int32)
    dbc = torch.from_numpy(np.stack([mbc.boundary_1d(m, w, 1), zero])).cuda()
    dsrc = torch.from_numpy(np.stack([zero, src])).cuda()
    e = torch.zeros((2, s.nE), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    st, rc = s.fwdsolve_batch_device(oms, e.data_ptr(), bc_ptr=dbc.data_ptr(), src_ptr=dsrc.data_ptr(), trans=trans)
    torch.cuda.synchronize()
    assert rc == 0
    ref = e.cpu().numpy().copy()
    e.fill_(1.0)
    torch.cuda.synchronize()
    torch.cuda._sleep(200_000_000)  # about 0.1 s of spinning on the default stream
    e.zero_()
    st, rc = s.fwdsolve_batch_device(oms, e.data_ptr(), bc_ptr=dbc.data_ptr(), src_ptr=dsrc.data_ptr(), trans=trans)
    torch.cuda.synchronize()
    assert rc == 0
    assert np.array_equal(e.cpu().numpy(), ref)

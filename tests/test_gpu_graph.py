"""The fused FP32 cycles run as captured CUDA graphs (replayed while their
arguments hold) and, with mt3d_profile on, as directly issued launches with
timing events.  Both issue the same kernels with the same arguments, and the
reductions are deterministic, so the fields agree bit for bit; the timed path
reports its launches, time and right-hand-side sweeps; the launch counter
counts a replayed graph's kernels."""
import numpy as np
import pytest

from helpers import random_model
from mt3d import bc as mbc
from mt3d import capi, models

pytestmark = pytest.mark.gpu


def _grid():
    return models.make_grid(40, 20, 6, 18, core=400.0, n_pad=3, pad_growth=1.5, air_first=60.0, air_growth=2.0,
                            earth_first=60.0, earth_growth=1.25)


def _solver(g, m):
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.set_restart(0)
    s.set_poly(0.9)
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=100, MaxDivCor=20, precision=capi.PREC_MIXED)
    return s


def test_graph_replay_and_timed_launches_agree(cuda):
    g = _grid()
    m = random_model(g, seed=9)
    om = 2 * np.pi * np.array([0.01, 0.01, 3.0, 3.0])
    bc = np.stack([mbc.boundary_1d(m, w, 1 + i % 2) for i, w in enumerate(om)])
    s = _solver(g, m)
    L = capi.load()
    c0 = L.mt3d_launch_counter()
    e1, st1, rc1 = s.fwdsolve_batch(om, bc=bc)
    c1 = L.mt3d_launch_counter()
    e2, st2, rc2 = s.fwdsolve_batch(om, bc=bc)  # the captured cycle replayed
    c2 = L.mt3d_launch_counter()
    s.profile(True)
    e3, st3, rc3 = s.fwdsolve_batch(om, bc=bc)
    n, ms, sweeps = s.kernel_time(1)
    s.profile(False)
    assert rc1 == rc2 == rc3 == 0
    assert np.array_equal(e1, e2) and np.array_equal(e1, e3)
    assert c2 - c1 == c1 - c0 > 0
    assert n > 0 and ms > 0 and sweeps > 0


def test_multi_graph_and_timed_launches_agree(cuda):
    shapes = [(14, 14, 4, 10), (24, 16, 5, 13)]
    probs = []
    for k, (nx, ny, na, ne) in enumerate(shapes):
        g = models.make_grid(nx, ny, na, ne, core=400.0, n_pad=3, pad_growth=1.5, air_first=60.0, air_growth=2.0,
                             earth_first=60.0, earth_growth=1.25)
        m = random_model(g, seed=30 + k)
        om = 2 * np.pi * np.array([0.05, 2.0])
        bc = np.stack([mbc.boundary_1d(m, w, 1 + i) for i, w in enumerate(om)])
        probs.append((g, m, om, bc))
    ss = [_solver(g, m) for g, m, *_ in probs]
    out = []
    for prof in (False, True):
        for s in ss:
            s.profile(prof)
        es = [np.zeros((2, g.n_edges), complex) for g, *_ in probs]
        st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], es, bc=[p[3] for p in probs])
        assert rc == 0
        out.append(es)
    timed = [s.kernel_time(1) for s in ss]
    for s in ss:
        s.profile(False)
    for a, b in zip(*out):
        assert np.array_equal(a, b)
    # the shared launches are timed on the first grid's handle; every handle
    # counts its own grid's sweeps
    assert timed[0][0] > 0 and timed[0][1] > 0
    assert all(t[2] > 0 for t in timed)

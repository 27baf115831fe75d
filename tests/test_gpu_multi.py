"""Multi-grid batches (mt3d_fwdsolve_multi): three models of uneven size solved
in one call, the FP32 iterations of all grids sharing their launches, against
the same right-hand sides solved per grid (mt3d_fwdsolve_batch).

Both reach the FP64 tolerance 1e-7; their fields agree to 1e-5 (relative
2-norm on the edges where the field is unique), the bound of the other
mixed-precision parity tests.  Also: the device-memory entry gives the host
entry's fields bit for bit, and the chunk tuner returns a valid choice and
caches it.
"""
import numpy as np
import pytest

from helpers import earth_mask, random_model, relerr
from mt3d import bc as mbc
from mt3d import capi, models

pytestmark = pytest.mark.gpu


def _problems():
    shapes = [(14, 14, 4, 10), (20, 24, 5, 13), (28, 18, 6, 16)]
    out = []
    for k, (nx, ny, na, ne) in enumerate(shapes):
        g = models.make_grid(nx, ny, na, ne, core=400.0, n_pad=3, pad_growth=1.5, air_first=60.0, air_growth=2.0,
                             earth_first=60.0, earth_growth=1.25)
        m = random_model(g, seed=20 + k)
        om = 2 * np.pi * np.array([0.05, 0.05, 2.0, 2.0, 2.0])
        bcs = [mbc.boundary_1d(m, om[0], 1), mbc.boundary_1d(m, om[1], 2), mbc.boundary_1d(m, om[2], 1),
               mbc.boundary_1d(m, om[3], 2), np.zeros(g.n_edges, complex)]
        rng = np.random.default_rng(k)
        src = np.zeros((5, g.n_edges), complex)
        em = earth_mask(g, m)
        src[4] = np.where(em, rng.standard_normal(g.n_edges) + 1j * rng.standard_normal(g.n_edges), 0) * 1e-3
        tr = np.array([0, 0, 0, 0, 1], np.int32)
        out.append((g, m, om, np.stack(bcs), src, tr))
    return out


def _solver(g, m):
    s = capi.Solver(g)
    s.set_formulation(capi.FORM_CCGD)
    s.set_restart(0)
    s.update_cond(m.m_earth, m.air_cond)
    s.set_control(IterPerDivCor=150, MaxDivCor=40, precision=capi.PREC_MIXED)
    return s


@pytest.fixture(scope="module")
def mprob(cuda):
    probs = _problems()
    return probs, [_solver(g, m) for g, m, *_ in probs]


def test_multi_grid_batch_matches_per_grid_solves(mprob):
    probs, ss = mprob
    es = [np.zeros((5, g.n_edges), complex) for g, *_ in probs]
    st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs],
                                 bc=[p[3] for p in probs], src=[p[4] for p in probs])
    assert rc == 0 and all(np.all(x == 0) for x in st)
    for (g, m, om, bc, src, tr), s, e in zip(probs, ss, es):
        it, rr = s.batch_diagnostics(5)
        assert np.all(rr <= 1e-7)
        ref, st1, rc1 = s.fwdsolve_batch(om, trans=tr, bc=bc, src=src)
        assert rc1 == 0
        em = earth_mask(g, m)
        for r in range(5):
            assert relerr(e[r][em], ref[r][em]) < 1e-5, (g.nx, r)


def test_multi_device_entry_matches_host_entry(mprob):
    import torch
    probs, ss = mprob
    es = [np.zeros((5, g.n_edges), complex) for g, *_ in probs]
    capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs], bc=[p[3] for p in probs],
                        src=[p[4] for p in probs])
    dbc = [torch.from_numpy(p[3]).cuda() for p in probs]
    dsrc = [torch.from_numpy(p[4]).cuda() for p in probs]
    de = [torch.zeros((5, g.n_edges), dtype=torch.complex128, device="cuda") for g, *_ in probs]
    torch.cuda.synchronize()
    st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], [x.data_ptr() for x in de], trans=[p[5] for p in probs],
                                 bc=[x.data_ptr() for x in dbc], src=[x.data_ptr() for x in dsrc], device=True)
    torch.cuda.synchronize()
    assert rc == 0
    for e, d in zip(es, de):
        assert np.array_equal(d.cpu().numpy(), e)


def test_multi_with_polynomial_preconditioner(mprob):
    """The batch with the polynomial preconditioner (seven launches an
    iteration) reaches the per-grid diagonal-preconditioned solutions, both
    solved to 1e-9 so that their iteration errors stay below the 1e-5 bound
    (at 1e-7 the transposed solve of a random source differed by 2.6e-5); a
    batch whose handles disagree on the coefficient is refused."""
    probs, ss = mprob
    for s in ss:
        s.set_control(IterPerDivCor=150, MaxDivCor=60, tolEMfwd=1e-9, tolEMadj=1e-9, precision=capi.PREC_MIXED)
    refs = []
    try:
        for (g, m, om, bc, src, tr), s in zip(probs, ss):
            ref, _, rc1 = s.fwdsolve_batch(om, trans=tr, bc=bc, src=src)
            assert rc1 == 0
            refs.append(ref)
        ss[0].set_poly(0.8)
        es = [np.zeros((5, g.n_edges), complex) for g, *_ in probs]
        with pytest.raises(capi.MT3DError):
            capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs],
                                bc=[p[3] for p in probs], src=[p[4] for p in probs])
        for s in ss[1:]:
            s.set_poly(0.8)
        st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs],
                                     bc=[p[3] for p in probs], src=[p[4] for p in probs])
        assert rc == 0 and all(np.all(x == 0) for x in st)
        for (g, m, *_), e, ref in zip(probs, es, refs):
            em = earth_mask(g, m)
            for r in range(5):
                assert relerr(e[r][em], ref[r][em]) < 1e-5, (g.nx, r)
    finally:
        for s in ss:
            s.set_poly(0.0)
            s.set_control(IterPerDivCor=150, MaxDivCor=40, precision=capi.PREC_MIXED)


def test_grid_with_nothing_to_solve(mprob):
    """A grid of the batch whose right-hand sides are all zero (forward rows
    without boundary data, a transposed row without a source) is done before
    the first cycle: its fields come back zero with status 0 (one iteration
    for a zero right-hand side, none for the source-less transposed row, as
    the reference reports them), and the grids beside it, whose cycles run
    on without it, give their per-grid solutions."""
    probs, ss = mprob
    bcs = [p[3] for p in probs]
    srcs = [p[4] for p in probs]
    bcs[1] = np.zeros_like(bcs[1])
    srcs[1] = np.zeros_like(srcs[1])
    es = [np.zeros((5, g.n_edges), complex) for g, *_ in probs]
    st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs], bc=bcs, src=srcs)
    assert rc == 0 and all(np.all(x == 0) for x in st)
    it, rr = ss[1].batch_diagnostics(5)
    assert np.all(es[1] == 0) and it.tolist() == [1, 1, 1, 1, 0] and np.all(rr == 0.0)
    for k in (0, 2):
        g, m, om, bc, src, tr = probs[k]
        ref, _, rc1 = ss[k].fwdsolve_batch(om, trans=tr, bc=bc, src=src)
        assert rc1 == 0
        em = earth_mask(g, m)
        for r in range(5):
            assert relerr(es[k][r][em], ref[r][em]) < 1e-5, (g.nx, r)


def test_chunk_counts_with_empty_chunks(mprob):
    """Chunk counts whose last chunk starts past the last node plane (6 of 15
    planes for the first grid: chunks of 3, the sixth empty; 6 of 19 and 9 of
    23 likewise) give the solutions of the default counts: the blocks of an
    empty chunk issue no copy and add nothing."""
    probs, ss = mprob
    for (g, *_), c in zip(probs, (6, 6, 9)):
        planes = g.nz + 1
        assert (c - 1) * (-(-planes // c)) >= planes
    out = []
    for zch in ([0, 0, 0], [6, 6, 9]):
        es = [np.zeros((5, g.n_edges), complex) for g, *_ in probs]
        st, rc = capi.fwdsolve_multi(ss, [p[2] for p in probs], es, trans=[p[5] for p in probs],
                                     bc=[p[3] for p in probs], src=[p[4] for p in probs], zchunks=zch)
        assert rc == 0
        out.append(es)
    for (g, m, *_), a, b in zip(probs, *out):
        em = earth_mask(g, m)
        for r in range(5):
            assert relerr(b[r][em], a[r][em]) < 1e-5, (g.nx, r)


def test_chunk_tuner_returns_and_caches_a_choice(mprob, tmp_path):
    """The tuner's timed runs (forward and transposed right-hand sides, each
    run from a zero first guess) return a valid choice, cache it and leave
    the handles' control and finite fields behind."""
    import torch
    from mt3d import tune
    probs, ss = mprob
    dbc = [torch.from_numpy(p[3]).cuda() for p in probs]
    dsrc = [torch.from_numpy(p[4]).cuda() for p in probs]
    de = [torch.zeros((5, g.n_edges), dtype=torch.complex128, device="cuda") for g, *_ in probs]
    path = str(tmp_path / "tune.json")
    zch = tune.tune(ss, [p[2] for p in probs], [x.data_ptr() for x in de], [x.data_ptr() for x in dbc],
                    [x.data_ptr() for x in dsrc], [p[5] for p in probs], torch.cuda.synchronize, cache_path=path,
                    iters=20, reps=2, reset=lambda: [x.zero_() for x in de])
    assert len(zch) == 3 and all(z in tune.candidates(s.grid.nz) for z, s in zip(zch, ss))
    assert all(bool(torch.isfinite(x).all()) for x in de)
    assert tune.tune(ss, [p[2] for p in probs], None, None, None, None, None, cache_path=path) == zch
    assert all(s.control["IterPerDivCor"] == 150 for s in ss)

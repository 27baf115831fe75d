"""E-field solution files (write_solnVectorMTX / read_solnVectorMTX layout):
the library against oracle/solnio.py, byte for byte."""
import numpy as np
import pytest

from helpers import small_grid
from mt3d import capi
from oracle import solnio


def fields(g, ntx=2, npol=2, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((ntx, npol, g.n_edges)) + 1j * rng.standard_normal((ntx, npol, g.n_edges))


def test_oracle_round_trip_and_record_layout(tmp_path):
    g = small_grid()
    e = fields(g)
    p = tmp_path / "a.soln"
    solnio.write(p, g, [0.5, 2.0], e, origin=(-1.0, 2.0, 0.0), rotdeg=7.0)
    head, om, f, names = solnio.read(p)
    assert (head["nx"], head["ny"], head["nz"], head["nzAir"], head["nTx"], head["nPol"]) == \
        (g.nx, g.ny, g.nz, g.nzAir, 2, 2)
    assert np.array_equal(f, e) and np.array_equal(om, [0.5, 2.0]) and names == [["Ex", "Ey"], ["Ex", "Ey"]]
    # EfileRead's nRecSkip: the (j, k) header is record 4 + ((j-1) nMode + (k-1)) 4 (0-based)
    recs = solnio._records(p)
    assert len(recs) == 4 + 2 * 2 * 4 and len(recs[0]) == 76 and len(recs[4]) == 36


def test_library_reads_header_without_a_device(tmp_path):
    g = small_grid()
    p = tmp_path / "b.soln"
    solnio.write(p, g, [1.0, 3.0, 9.0], fields(g, ntx=3), origin=(10.0, -20.0, 5.0), rotdeg=30.0)
    h = capi.read_soln_header(str(p))
    assert (h["nTx"], h["nPol"], h["nzAir"]) == (3, 2, g.nzAir)
    assert np.array_equal(h["dx"], g.dx) and np.array_equal(h["dy"], g.dy) and np.array_equal(h["dz"], g.dz)
    assert tuple(h["origin"]) == (10.0, -20.0, 5.0) and h["rotdeg"] == 30.0
    bad = tmp_path / "bad.soln"
    bad.write_bytes(b"\x00" * 40)
    with pytest.raises(capi.MT3DError):
        capi.read_soln_header(str(bad))


@pytest.mark.gpu
def test_library_writes_the_oracle_bytes_and_reads_them_back(cuda, tmp_path):
    import torch
    g = small_grid()
    e = fields(g)
    om = [0.25, 4.0]
    s = capi.Solver(g)
    ref, lib_h, lib_d = tmp_path / "ref.soln", tmp_path / "host.soln", tmp_path / "dev.soln"
    solnio.write(ref, g, om, e, origin=(1.0, 2.0, 3.0), rotdeg=0.5)
    s.write_soln(str(lib_h), om, e, origin=(1.0, 2.0, 3.0), rotdeg=0.5)
    ed = torch.from_numpy(e.reshape(-1).view(np.float64)).cuda()
    s.write_soln(str(lib_d), om, (ed.data_ptr(), 2, 2), origin=(1.0, 2.0, 3.0), rotdeg=0.5)
    assert ref.read_bytes() == lib_h.read_bytes() == lib_d.read_bytes()
    for j in (1, 2):
        for k in (1, 2):
            w, f = s.read_soln(str(ref), j, k)
            assert w == om[j - 1] and np.array_equal(f, e[j - 1, k - 1])
            out = torch.zeros(2 * g.n_edges, dtype=torch.float64, device="cuda")
            w, _ = s.read_soln(str(ref), j, k, device_ptr=out.data_ptr())
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy().view(np.complex128), e[j - 1, k - 1])
    other = capi.Solver(small_grid(nx=11))
    with pytest.raises(capi.MT3DError):
        other.read_soln(str(ref), 1, 1)
    with pytest.raises(capi.MT3DError):
        s.read_soln(str(ref), 3, 1)


@pytest.mark.gpu
def test_entry_points_reject_bad_arguments(cuda, tmp_path):
    """Invalid arguments of the boundary, profiling and file entry points come
    back as MT3D_INVALID_ARGUMENT with a message, not as a crash."""
    import ctypes as C
    g = small_grid()
    s = capi.Solver(g)
    m_earth = np.full(g.nx * g.ny * g.nzEarth, -np.log(100.0))
    s.update_cond(m_earth, -23.0)
    e = np.zeros(g.n_edges, np.complex128)
    for imode, om in ((0, 1.0), (3, 1.0), (1, 0.0), (1, float("nan"))):
        rc = s.L.mt3d_compute_bc_device(s.h, imode, om, e.ctypes.data_as(C.c_void_p))
        assert rc == 5 and s._err(s.h)
    n, ms, sw = C.c_int(), C.c_double(), C.c_int64()
    assert s.L.mt3d_kernel_time(s.h, 2, C.byref(n), C.byref(ms), C.byref(sw)) == 5
    with pytest.raises(capi.MT3DError):
        s.write_soln(str(tmp_path / "x.soln"), [], np.zeros((0, 2, g.n_edges), np.complex128))
    s.write_soln(str(tmp_path / "y.soln"), [1.0], np.zeros((1, 2, g.n_edges), np.complex128))
    for itx, ipol in ((0, 1), (1, 0), (2, 1), (1, 3)):
        with pytest.raises(capi.MT3DError):
            s.read_soln(str(tmp_path / "y.soln"), itx, ipol)
    with pytest.raises(capi.MT3DError):
        s.read_soln(str(tmp_path / "missing.soln"), 1, 1)

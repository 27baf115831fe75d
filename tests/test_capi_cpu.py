"""CPU-side checks of the C ABI library: it loads without a GPU, exports every
symbol include/mt3d.h declares, and fails cleanly (no abort) without a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mt3d import capi, models

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "mt3d.h")).read()
    return sorted(set(re.findall(r"MT3D_API\s+(?:const\s+)?\w+\s*\*?\s*(mt3d_\w+)\s*\(", src)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(capi.EXPORTS)


def test_library_loads_and_exports_all_symbols():
    L = capi.load()
    for name in header_symbols():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.mt3d_version()


def test_no_device_is_a_status_not_a_crash():
    L = capi.load()
    if L.mt3d_device_count() > 0:
        return  # a GPU is present; covered by the gpu tests
    g = models.make_grid(8, 8, 2, 4)
    h = C.c_void_p()
    dx = np.ascontiguousarray(g.dx)
    rc = L.mt3d_create(0, g.nx, g.ny, g.nz, g.nzAir, dx.ctypes.data_as(C.POINTER(C.c_double)),
                       np.ascontiguousarray(g.dy).ctypes.data_as(C.POINTER(C.c_double)),
                       np.ascontiguousarray(g.dz).ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    assert rc == 7 and not h.value
    buf = C.create_string_buffer(256)
    L.mt3d_last_error(None, buf, 256)
    assert b"no CUDA device" in buf.value


def test_invalid_arguments_rejected_before_device_use():
    L = capi.load()
    h = C.c_void_p()
    dx = np.ones(3)
    p = dx.ctypes.data_as(C.POINTER(C.c_double))
    assert L.mt3d_create(0, 1, 3, 3, 1, p, p, p, C.byref(h)) == 5  # nx < 2
    assert L.mt3d_create(0, 3, 3, 3, 3, p, p, p, C.byref(h)) == 5  # nzAir >= nz
    assert L.mt3d_set_control(None, 40, 20, 100, 1e-7, 1e-7, 1e-5, 1, 0) == 5
    assert L.mt3d_fwdsolve(None, 0, None, None, None) == 5


def test_fwdsolve_batch_out_buffer_is_checked_before_the_library():
    """fwdsolve_batch(out=...) takes the caller's array as the library's
    in/out buffer; arrays it cannot pass through unchanged are refused before
    any device call."""
    import pytest

    class Fake:
        nE = 10
        fwdsolve_batch = capi.Solver.fwdsolve_batch

    f = Fake()
    om = np.ones(2)
    for bad in (np.zeros((2, 10), np.complex64), np.zeros((2, 20), np.complex128)[:, ::2],
                np.zeros((3, 10), np.complex128)):
        with pytest.raises(ValueError):
            f.fwdsolve_batch(om, out=bad)
    with pytest.raises(ValueError):
        f.fwdsolve_batch(om, e0=np.zeros((2, 10)), out=np.zeros((2, 10), np.complex128))


def test_missing_or_stale_library_fails_loudly(tmp_path):
    """The binding has no fallback: a library that is not there, or one built
    from other sources than the tree holds, is an error, not a slower path."""
    with pytest.raises(FileNotFoundError):
        _load_fresh(str(tmp_path / "libmt3d.so"))
    # a file that carries no source hash of this tree
    stale = tmp_path / "stale.so"
    stale.write_bytes(b"\x7fELF" + bytes(64))
    with pytest.raises(RuntimeError, match="rebuild"):
        capi.check_fresh(str(stale))


def _load_fresh(path):
    saved = capi._lib
    capi._lib = None
    try:
        return capi.load(path)
    finally:
        capi._lib = saved

"""ctypes binding of libmt3d.so (include/mt3d.h).

This mirrors, in Python, the calls a ModEM host makes around its forward
solver: ``ModelDataInit`` (Solver(...)), ``UpdateCond``, ``UpdateFreq``,
``Mult_Aii``, ``BICG`` and ``FWDsolve3D`` (f90/3D_MT/FWD/modelOperator3D.f90,
f90/3D_MT/FWD/EMsolve3D.f90, f90/3D_MT/FWD_SP2/solver.f90).  There is no CPU
fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libmt3d.so")

STATUS = {0: "MT3D_OK", 1: "MT3D_NOT_CONVERGED", 2: "MT3D_BREAKDOWN", 3: "MT3D_NAN_INPUT", 4: "MT3D_CUDA_ERROR",
          5: "MT3D_INVALID_ARGUMENT", 6: "MT3D_DEVICE_TIMEOUT", 7: "MT3D_NO_DEVICE", 8: "MT3D_OUT_OF_MEMORY"}
SOLVER_BICG, SOLVER_COCG, SOLVER_BICG_ZLINE, SOLVER_QMR = 1, 2, 3, 4
PREC_FP64, PREC_MIXED = 0, 1
FORM_CCDC, FORM_CCGD = 0, 1

#: every symbol include/mt3d.h declares
EXPORTS = ["mt3d_version", "mt3d_device_count", "mt3d_create", "mt3d_destroy", "mt3d_set_control", "mt3d_update_cond",
           "mt3d_get_cond", "mt3d_compute_bc", "mt3d_compute_bc_device", "mt3d_update_freq", "mt3d_set_formulation", "mt3d_set_restart", "mt3d_sizes", "mt3d_interior_index", "mt3d_mult_aii",
           "mt3d_mult_aii_device_noalloc", "mt3d_bicg", "mt3d_fwdsolve",
           "mt3d_fwdsolve_batch", "mt3d_fwdsolve_batch_device", "mt3d_fwdsolve_multi",
           "mt3d_fwdsolve_multi_device", "mt3d_set_stream", "mt3d_set_wait_limit", "mt3d_set_fused",
           "mt3d_set_poly",
           "mt3d_apply_kernel", "mt3d_profile",
           "mt3d_kernel_time", "mt3d_get_diag", "mt3d_get_batch_diag", "mt3d_pmult_t", "mt3d_impedance", "mt3d_impedance_device", "mt3d_lmult_t", "mt3d_lmult_t_device", "mt3d_jmult_t", "mt3d_jmult_t_device", "mt3d_write_soln", "mt3d_read_soln", "mt3d_read_soln_header", "mt3d_launch_counter", "mt3d_alloc_counter",
           "mt3d_last_error"]

_lib = None


class MT3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def check_fresh(path: str = LIB_PATH):
    """Raise if the library at `path` was built from other sources than the
    ones beside it (a stale build would run old kernels under new tests)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_mt3d_build", os.path.join(os.path.dirname(_HERE), "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    have, want = b.built_hash(path), b.expected_hash()
    if have != want:
        raise RuntimeError(f"{path} was built from sources {have}, the tree holds {want}: rebuild it "
                           "(python modem-gpu_b200/build.py)")


def load(path: str = LIB_PATH):
    """Load libmt3d.so; raises if it is missing (build it with build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not found: build the CUDA library first (python modem-gpu_b200/build.py)")
    if os.path.abspath(path) == os.path.abspath(LIB_PATH):
        check_fresh(path)
    L = C.CDLL(path)
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    I = C.c_int
    IP = C.POINTER(C.c_int)
    L.mt3d_version.restype = C.c_char_p
    L.mt3d_device_count.restype = I
    L.mt3d_create.argtypes = [I, I, I, I, I, D, D, D, C.POINTER(P)]
    L.mt3d_destroy.argtypes = [P]
    L.mt3d_set_control.argtypes = [P, I, I, I, C.c_double, C.c_double, C.c_double, I, I]
    L.mt3d_update_cond.argtypes = [P, D, C.c_double]
    L.mt3d_get_cond.argtypes = [P, D, D, D]
    L.mt3d_compute_bc.argtypes = [P, I, D]
    L.mt3d_compute_bc_device.argtypes = [P, I, C.c_double, C.c_void_p]
    L.mt3d_update_freq.argtypes = [P, C.c_double]
    L.mt3d_set_formulation.argtypes = [P, I]
    L.mt3d_set_restart.argtypes = [P, I]
    L.mt3d_sizes.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.mt3d_interior_index.argtypes = [P, C.POINTER(C.c_int32)]
    L.mt3d_mult_aii.argtypes = [P, I, D, D]
    L.mt3d_mult_aii_device_noalloc.argtypes = [P, I, C.c_void_p, C.c_void_p]
    L.mt3d_impedance.argtypes = [P, C.c_double, I, D, D, D, D, D]
    L.mt3d_impedance_device.argtypes = [P, C.c_double, I, D, D, C.c_void_p, C.c_void_p, D]
    L.mt3d_lmult_t.argtypes = [P, C.c_double, I, D, D, D, D, D, D, D]
    L.mt3d_lmult_t_device.argtypes = [P, C.c_double, I, D, D, C.c_void_p, C.c_void_p, D, C.c_void_p, C.c_void_p]
    L.mt3d_bicg.argtypes = [P, D, D, I, C.c_double, IP, D, IP]
    L.mt3d_fwdsolve.argtypes = [P, I, D, D, D]
    L.mt3d_fwdsolve_batch.argtypes = [P, I, D, IP, D, D, D, IP]
    L.mt3d_fwdsolve_batch_device.argtypes = [P, I, D, IP, C.c_void_p, C.c_void_p, C.c_void_p, IP]
    L.mt3d_set_stream.argtypes = [P, C.c_void_p]
    L.mt3d_set_wait_limit.argtypes = [P, I]
    PP = C.POINTER(C.c_void_p)
    for name in ("mt3d_fwdsolve_multi", "mt3d_fwdsolve_multi_device"):
        getattr(L, name).argtypes = [I, C.POINTER(P), IP, PP, PP, PP, PP, PP, PP, IP]
    L.mt3d_set_fused.argtypes = [P, I]
    L.mt3d_set_poly.argtypes = [P, C.c_double]
    L.mt3d_jmult_t.argtypes = [P, C.c_double, I, D, D, D, D, D, D, D]
    L.mt3d_jmult_t_device.argtypes = [P, C.c_double, I, D, D, C.c_void_p, D, D, C.c_void_p, C.c_void_p]
    L.mt3d_apply_kernel.argtypes = [P, I, D, D]
    L.mt3d_profile.argtypes = [P, I]
    L.mt3d_kernel_time.argtypes = [P, I, IP, D, C.POINTER(C.c_int64)]
    L.mt3d_get_diag.argtypes = [P, IP, IP, IP, D, I, D, I, D]
    L.mt3d_get_batch_diag.argtypes = [P, I, IP, D]
    L.mt3d_pmult_t.argtypes = [P, I, D, D, D, D]
    L.mt3d_last_error.argtypes = [P, C.c_char_p, I]
    L.mt3d_write_soln.argtypes = [P, C.c_char_p, I, I, D, D, C.c_double, C.c_void_p, I]
    L.mt3d_read_soln.argtypes = [P, C.c_char_p, I, I, D, C.c_void_p, I]
    L.mt3d_read_soln_header.argtypes = [C.c_char_p, IP, IP, IP, IP, IP, IP, D, D, D, D, D]
    for name in ("mt3d_launch_counter", "mt3d_alloc_counter"):
        getattr(L, name).restype = C.c_int64
        getattr(L, name).argtypes = []
    for name in EXPORTS:
        if name not in ("mt3d_version", "mt3d_launch_counter", "mt3d_alloc_counter"):
            getattr(L, name).restype = I
    _lib = L
    return L


def _d(a):
    if a is None:
        return None
    assert a.flags.c_contiguous and a.dtype in (np.float64, np.complex128)
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Solver:
    """One solver handle: a grid, its conductivity model and a frequency."""

    def __init__(self, grid, device: int = 0):
        self.L = load()
        self.grid = grid
        self.h = C.c_void_p()
        dx = np.ascontiguousarray(grid.dx, np.float64)
        dy = np.ascontiguousarray(grid.dy, np.float64)
        dz = np.ascontiguousarray(grid.dz, np.float64)
        rc = self.L.mt3d_create(device, grid.nx, grid.ny, grid.nz, grid.nzAir, _d(dx), _d(dy), _d(dz),
                                C.byref(self.h))
        if rc:
            raise MT3DError(rc, self._err(None))
        self.control = dict(IterPerDivCor=40, MaxDivCor=20, MaxIterDivCor=100, tolEMfwd=1e-7, tolEMadj=1e-7,
                            tolDivCor=1e-5, solver=SOLVER_BICG, precision=PREC_FP64)
        nE, nEi, nN = C.c_int64(), C.c_int64(), C.c_int64()
        self.L.mt3d_sizes(self.h, C.byref(nE), C.byref(nEi), C.byref(nN))
        self.nE, self.nEi, self.nN = nE.value, nEi.value, nN.value

    def _err(self, h):
        buf = C.create_string_buffer(512)
        self.L.mt3d_last_error(h, buf, 512)
        return buf.value.decode()

    def _check(self, rc, allow=(0,)):
        if rc not in allow:
            raise MT3DError(rc, self._err(self.h))
        return rc

    def close(self):
        if self.h:
            self.L.mt3d_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_control(self, IterPerDivCor=40, MaxDivCor=20, MaxIterDivCor=100, tolEMfwd=1e-7, tolEMadj=1e-7,
                    tolDivCor=1e-5, solver=SOLVER_BICG, precision=PREC_FP64):
        self._check(self.L.mt3d_set_control(self.h, IterPerDivCor, MaxDivCor, MaxIterDivCor, tolEMfwd, tolEMadj,
                                            tolDivCor, solver, precision))
        self.control = dict(IterPerDivCor=IterPerDivCor, MaxDivCor=MaxDivCor, MaxIterDivCor=MaxIterDivCor,
                            tolEMfwd=tolEMfwd, tolEMadj=tolEMadj, tolDivCor=tolDivCor, solver=solver,
                            precision=precision)

    def set_formulation(self, formulation):
        self._check(self.L.mt3d_set_formulation(self.h, int(formulation)))

    def set_restart(self, restart):
        self._check(self.L.mt3d_set_restart(self.h, int(restart)))

    def update_cond(self, m_earth, air_cond):
        m = np.ascontiguousarray(m_earth, np.float64)
        self._check(self.L.mt3d_update_cond(self.h, _d(m), float(air_cond)))

    def get_cond(self):
        """(sigma_e [nE], divcorr [7, nN], node_w [nN]) as mt3d_get_cond returns them."""
        sig, coef, w = np.zeros(self.nE), np.zeros(7 * self.nN), np.zeros(self.nN)
        self._check(self.L.mt3d_get_cond(self.h, _d(sig), _d(coef), _d(w)))
        return sig, coef.reshape(7, self.nN), w

    def compute_bc(self, imode):
        """E0 of BC_x0_WS for polarisation imode (1 or 2) at the handle's
        frequency: boundary entries are the BC, interior entries the first guess."""
        e0 = np.zeros(self.nE, np.complex128)
        self._check(self.L.mt3d_compute_bc(self.h, int(imode), _d(e0)))
        return e0

    def write_soln(self, path, omegas, e, origin=(0.0, 0.0, 0.0), rotdeg=0.0):
        """e: host array [nTx, nPol, nE] (complex128), or (device address as
        int, nTx, nPol) for fields in device memory."""
        om = np.ascontiguousarray(omegas, np.float64)
        org = np.ascontiguousarray(origin, np.float64)
        if isinstance(e, tuple):
            ptr, ntx, npol = e
            rc = self.L.mt3d_write_soln(self.h, os.fsencode(path), ntx, npol, _d(om), _d(org), float(rotdeg),
                                        C.c_void_p(ptr), 1)
        else:
            a = np.ascontiguousarray(e, np.complex128)
            rc = self.L.mt3d_write_soln(self.h, os.fsencode(path), a.shape[0], a.shape[1], _d(om), _d(org),
                                        float(rotdeg), a.ctypes.data_as(C.c_void_p), 0)
        self._check(rc)

    def read_soln(self, path, itx, ipol, device_ptr=None):
        """(omega, field) of transmitter itx, polarisation ipol (1-based); with
        device_ptr the field goes to that device address and None is returned."""
        om = C.c_double()
        if device_ptr is not None:
            self._check(self.L.mt3d_read_soln(self.h, os.fsencode(path), itx, ipol, C.byref(om),
                                              C.c_void_p(device_ptr), 1))
            return om.value, None
        e = np.zeros(self.nE, np.complex128)
        self._check(self.L.mt3d_read_soln(self.h, os.fsencode(path), itx, ipol, C.byref(om),
                                          e.ctypes.data_as(C.c_void_p), 0))
        return om.value, e

    def update_freq(self, omega):
        self._check(self.L.mt3d_update_freq(self.h, float(omega)))

    def interior_index(self):
        out = np.zeros(self.nEi, np.int32)
        self._check(self.L.mt3d_interior_index(self.h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def mult_aii(self, x, adjt=False):
        x = np.ascontiguousarray(x, np.complex128)
        y = np.zeros(self.nEi, np.complex128)
        self._check(self.L.mt3d_mult_aii(self.h, int(adjt), _d(x), _d(y)))
        return y

    def mult_aii_device_noalloc(self, x_ptr, y_ptr, adjt=False):
        """y = A x on device interior vectors (nEi complex128 each, given by
        device address, e.g. a torch tensor's data_ptr()); enqueued on the
        handle's stream, no device allocation."""
        self._check(self.L.mt3d_mult_aii_device_noalloc(self.h, int(adjt), C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def impedance(self, omega, sites, e1, e2, origin=(0.0, 0.0, 0.0)):
        """Full impedance tensors [nsite, 2, 2] (E / B, SI) at sites [nsite, 3]
        from the full edge fields e1, e2 of the two polarisations (host
        arrays, or device addresses as ints)."""
        xyz = np.ascontiguousarray(sites, np.float64).reshape(-1, 3)
        org = np.ascontiguousarray(origin, np.float64)
        Z = np.zeros(4 * len(xyz), np.complex128)
        if isinstance(e1, int):
            rc = self.L.mt3d_impedance_device(self.h, float(omega), len(xyz), _d(xyz), _d(org), C.c_void_p(e1),
                                              C.c_void_p(e2), _d(Z))
        else:
            a = np.ascontiguousarray(e1, np.complex128)
            b = np.ascontiguousarray(e2, np.complex128)
            rc = self.L.mt3d_impedance(self.h, float(omega), len(xyz), _d(xyz), _d(org), _d(a), _d(b), _d(Z))
        self._check(rc)
        return Z.reshape(-1, 2, 2)

    def lmult_t(self, omega, sites, e1, e2, d, origin=(0.0, 0.0, 0.0)):
        """Adjoint sources (s1, s2) of the impedance data weights d [nsite, 2, 2]
        for background fields e1, e2 (host arrays)."""
        xyz = np.ascontiguousarray(sites, np.float64).reshape(-1, 3)
        org = np.ascontiguousarray(origin, np.float64)
        dd = np.ascontiguousarray(d, np.complex128).reshape(-1)
        a = np.ascontiguousarray(e1, np.complex128)
        b = np.ascontiguousarray(e2, np.complex128)
        s1 = np.zeros(self.nE, np.complex128)
        s2 = np.zeros(self.nE, np.complex128)
        self._check(self.L.mt3d_lmult_t(self.h, float(omega), len(xyz), _d(xyz), _d(org), _d(a), _d(b), _d(dd),
                                        _d(s1), _d(s2)))
        return s1, s2

    def lmult_t_device(self, omega, sites, e1_ptr, e2_ptr, d, s1_ptr, s2_ptr, origin=(0.0, 0.0, 0.0)):
        """mt3d_lmult_t on device fields and sources (device addresses)."""
        xyz = np.ascontiguousarray(sites, np.float64).reshape(-1, 3)
        org = np.ascontiguousarray(origin, np.float64)
        dd = np.ascontiguousarray(d, np.complex128).reshape(-1)
        self._check(self.L.mt3d_lmult_t_device(self.h, float(omega), len(xyz), _d(xyz), _d(org), C.c_void_p(e1_ptr),
                                               C.c_void_p(e2_ptr), _d(dd), C.c_void_p(s1_ptr), C.c_void_p(s2_ptr)))

    def jmult_t(self, omega, sites, e1, e2, d, m0_earth, origin=(0.0, 0.0, 0.0), want_eadj=False):
        """J^T d of one frequency (JmultT_TX) from the background fields e1, e2
        (host arrays) and data weights d [nsite, 2, 2]: returns (dm, status)
        or (dm, eadj [2, nE], status)."""
        xyz = np.ascontiguousarray(sites, np.float64).reshape(-1, 3)
        org = np.ascontiguousarray(origin, np.float64)
        dd = np.ascontiguousarray(d, np.complex128).reshape(-1)
        e0 = np.ascontiguousarray(np.stack([np.asarray(e1), np.asarray(e2)]), np.complex128)
        m0 = np.ascontiguousarray(m0_earth, np.float64)
        g = self.grid
        dm = np.zeros(g.nx * g.ny * g.nzEarth)
        ea = np.zeros((2, self.nE), np.complex128) if want_eadj else None
        rc = self._check(self.L.mt3d_jmult_t(self.h, float(omega), len(xyz), _d(xyz), _d(org), _d(e0), _d(dd),
                                             _d(m0), _d(dm), _d(ea) if ea is not None else None), allow=(0, 1))
        return (dm, ea, rc) if want_eadj else (dm, rc)

    def jmult_t_device(self, omega, sites, e0_ptr, d, m0_earth, dm_ptr, eadj_ptr=None, origin=(0.0, 0.0, 0.0)):
        """mt3d_jmult_t_device: e0_ptr (two full edge fields), dm_ptr and
        eadj_ptr are device addresses."""
        xyz = np.ascontiguousarray(sites, np.float64).reshape(-1, 3)
        org = np.ascontiguousarray(origin, np.float64)
        dd = np.ascontiguousarray(d, np.complex128).reshape(-1)
        m0 = np.ascontiguousarray(m0_earth, np.float64)
        return self._check(self.L.mt3d_jmult_t_device(self.h, float(omega), len(xyz), _d(xyz), _d(org),
                                                      C.c_void_p(e0_ptr), _d(dd), _d(m0), C.c_void_p(dm_ptr),
                                                      C.c_void_p(eadj_ptr) if eadj_ptr else None), allow=(0, 1))

    def bicg(self, b, x0, maxit, tol):
        b = np.ascontiguousarray(b, np.complex128)
        x = np.array(x0, np.complex128)
        rerr = np.zeros(maxit)
        n, f = C.c_int(), C.c_int()
        rc = self._check(self.L.mt3d_bicg(self.h, _d(b), _d(x), int(maxit), float(tol), C.byref(n), _d(rerr),
                                          C.byref(f)), allow=(0, 1, 2, 3))
        return x, n.value, rerr, f.value, rc

    def fwdsolve(self, trans=False, bc=None, src=None, e0=None):
        e = np.zeros(self.nE, np.complex128) if e0 is None else np.array(e0, np.complex128)
        bcp = None if bc is None else np.ascontiguousarray(bc, np.complex128)
        srcp = None if src is None else np.ascontiguousarray(src, np.complex128)
        rc = self._check(self.L.mt3d_fwdsolve(self.h, int(trans), _d(bcp), _d(srcp), _d(e)), allow=(0, 1, 2, 3))
        return e, rc

    def fwdsolve_batch(self, omegas, trans=None, bc=None, src=None, e0=None, out=None):
        """Batched FWDsolve3D on host arrays.  e0: first guesses (zero if
        None; copied).  out: a C-contiguous complex128 [n, nE] array used in
        place as mt3d_fwdsolve_batch's e (first guess in, solution out), so
        a pinned buffer is copied to and from the device directly; then e0
        must be None.  Returns (e, status, rc)."""
        omegas = np.ascontiguousarray(omegas, np.float64)
        n = omegas.size
        tr = np.zeros(n, np.int32) if trans is None else np.ascontiguousarray(trans, np.int32)
        if out is not None:
            if e0 is not None:
                raise ValueError("fwdsolve_batch: give the first guess in out, not in e0")
            if not (isinstance(out, np.ndarray) and out.dtype == np.complex128 and out.flags.c_contiguous and
                    out.shape == (n, self.nE) and out.flags.writeable):
                raise ValueError("fwdsolve_batch: out must be a writeable C-contiguous complex128 [n, nE] array")
            e = out
        else:
            e = np.zeros((n, self.nE), np.complex128) if e0 is None else np.array(e0, np.complex128)
        bcp = None if bc is None else np.ascontiguousarray(bc, np.complex128)
        srcp = None if src is None else np.ascontiguousarray(src, np.complex128)
        st = np.zeros(n, np.int32)
        rc = self._check(self.L.mt3d_fwdsolve_batch(self.h, n, _d(omegas), tr.ctypes.data_as(C.POINTER(C.c_int)),
                                                    _d(bcp), _d(srcp), _d(e), st.ctypes.data_as(C.POINTER(C.c_int))),
                         allow=(0, 1, 2, 3))
        return e, st, rc

    def fwdsolve_batch_device(self, omegas, e_ptr, bc_ptr=None, src_ptr=None, trans=None):  # noqa: D401
        """Batched solve on device-resident fields: e_ptr, bc_ptr, src_ptr are
        device addresses (e.g. torch tensor data_ptr()) of nrhs full edge
        vectors each (complex128)."""
        omegas = np.ascontiguousarray(omegas, np.float64)
        n = omegas.size
        tr = np.zeros(n, np.int32) if trans is None else np.ascontiguousarray(trans, np.int32)
        st = np.zeros(n, np.int32)
        rc = self._check(self.L.mt3d_fwdsolve_batch_device(self.h, n, _d(omegas), tr.ctypes.data_as(C.POINTER(C.c_int)),
                                                           bc_ptr, src_ptr, e_ptr,
                                                           st.ctypes.data_as(C.POINTER(C.c_int))), allow=(0, 1, 2, 3))
        return st, rc

    def set_stream(self, stream_handle):
        self._check(self.L.mt3d_set_stream(self.h, stream_handle))

    def set_fused(self, on: bool = True):
        self._check(self.L.mt3d_set_fused(self.h, int(bool(on))))

    def set_poly(self, c: float):
        """Polynomial preconditioner c D^-1 (2 I - c A D^-1) in the fused FP32
        iteration (0: the diagonal preconditioner alone)."""
        self._check(self.L.mt3d_set_poly(self.h, float(c)))

    def set_wait_limit(self, polls: int):
        self._check(self.L.mt3d_set_wait_limit(self.h, int(polls)))

    def apply_kernel(self, kernel: int, x: np.ndarray) -> np.ndarray:
        """A x on full edge vectors through internal kernel 0 (FP64 apply),
        1 (staged FP64 stencil) or 2 (TMA-staged FP32 stencil); D^-1 A x
        through kernel 3 (the fused FP32 iteration's stencil)."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.nE, np.complex128)
        self._check(self.L.mt3d_apply_kernel(self.h, int(kernel), _d(x), _d(y)))
        return y

    def profile(self, enable=True):
        self._check(self.L.mt3d_profile(self.h, int(enable)))

    def kernel_time(self, precision):
        """(timed launches, device ms, right-hand-side sweeps) of the stencil
        launches of one precision (0 FP64, 1 FP32) since profile(True)."""
        n, ms, sw = C.c_int(), C.c_double(), C.c_int64()
        self._check(self.L.mt3d_kernel_time(self.h, int(precision), C.byref(n), C.byref(ms), C.byref(sw)))
        return n.value, ms.value, sw.value

    def diagnostics(self, maxlen=4000, maxdc=200):
        nit, ndc, fl = C.c_int(), C.c_int(), C.c_int()
        rel = np.zeros(maxlen)
        dj = np.zeros(2 * maxdc)
        fr = C.c_double()
        self._check(self.L.mt3d_get_diag(self.h, C.byref(nit), C.byref(ndc), C.byref(fl), _d(rel), maxlen, _d(dj),
                                         maxdc, C.byref(fr)))
        return dict(nIterTotal=nit.value, nDivCor=ndc.value, failed=bool(fl.value),
                    EMrelErr=rel[: min(nit.value, maxlen)].copy(), divJ=dj.reshape(-1, 2)[: ndc.value].copy(),
                    final_relres=fr.value)

    def batch_diagnostics(self, nrhs):
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        self._check(self.L.mt3d_get_batch_diag(self.h, nrhs, it.ctypes.data_as(C.POINTER(C.c_int)), _d(rr)))
        return it, rr

    def pmult_t(self, e0, eadj, m0_earth):
        e0 = np.ascontiguousarray(e0, np.complex128)
        ea = np.ascontiguousarray(eadj, np.complex128)
        npol = e0.shape[0] if e0.ndim == 2 else 1
        m0 = np.ascontiguousarray(m0_earth, np.float64)
        g = self.grid
        out = np.zeros(g.nx * g.ny * g.nzEarth)
        self._check(self.L.mt3d_pmult_t(self.h, npol, _d(e0), _d(ea), _d(m0), _d(out)))
        return out


def fwdsolve_multi(solvers, omegas, e, trans=None, bc=None, src=None, zchunks=None, device=False):
    """mt3d_fwdsolve_multi over several handles (one grid each).

    omegas, trans: per handle, arrays of its right-hand sides' angular
    frequencies and transposition flags.  e, bc, src: per handle, either host
    arrays [nrhs, nE] (complex128, e is updated in place) or, with
    device=True, device addresses (ints); bc / src (or entries) may be None.
    zchunks: per-handle node-plane chunk counts of the stencil blocks (None
    or 0: the default).  Returns (statuses per handle, worst status)."""
    L = load()
    nh = len(solvers)
    hs = (C.c_void_p * nh)(*[s.h for s in solvers])
    om = [np.ascontiguousarray(o, np.float64) for o in omegas]
    nr = (C.c_int * nh)(*[o.size for o in om])
    tr = [np.zeros(o.size, np.int32) if trans is None or trans[i] is None else np.ascontiguousarray(trans[i], np.int32)
          for i, o in enumerate(om)]
    st = [np.zeros(o.size, np.int32) for o in om]

    def ptrs(xs, kind):
        out = (C.c_void_p * nh)()
        for i in range(nh):
            x = None if xs is None else xs[i]
            if x is None:
                out[i] = None
            elif device:
                out[i] = int(x)
            else:
                assert x.dtype == kind and x.flags.c_contiguous
                out[i] = x.ctypes.data
        return out

    if not device:
        for i, x in enumerate(e):
            assert x.shape == (om[i].size, solvers[i].nE)
    ap = lambda arrs: (C.c_void_p * nh)(*[a.ctypes.data for a in arrs])
    zc = None if zchunks is None else (C.c_int * nh)(*[int(z) for z in zchunks])
    fn = L.mt3d_fwdsolve_multi_device if device else L.mt3d_fwdsolve_multi
    rc = fn(nh, hs, nr, ap(om), ap(tr), ptrs(bc, np.complex128), ptrs(src, np.complex128), ptrs(e, np.complex128),
            ap(st), zc)
    if rc not in (0, 1):
        buf = C.create_string_buffer(512)
        L.mt3d_last_error(None, buf, 512)
        raise MT3DError(rc, buf.value.decode())
    return st, rc


def device_count() -> int:
    return int(load().mt3d_device_count())


def read_soln_header(path):
    """Header of a solution file: dict with nTx, nPol, the grid (dx, dy, dz,
    nzAir), origin and rotation."""
    L = load()
    v = [C.c_int() for _ in range(6)]
    org, rot = np.zeros(3), C.c_double()
    rc = L.mt3d_read_soln_header(os.fsencode(path), *[C.byref(x) for x in v], _d(org), C.byref(rot), None, None, None)
    if rc:
        raise MT3DError(rc, _last_global_error(L))
    ntx, npol, nx, ny, nz, nza = (x.value for x in v)
    dx, dy, dz = np.zeros(nx), np.zeros(ny), np.zeros(nz)
    rc = L.mt3d_read_soln_header(os.fsencode(path), None, None, None, None, None, None, None, None, _d(dx), _d(dy),
                                 _d(dz))
    if rc:
        raise MT3DError(rc, _last_global_error(L))
    return dict(nTx=ntx, nPol=npol, dx=dx, dy=dy, dz=dz, nzAir=nza, origin=org, rotdeg=rot.value)


def _last_global_error(L):
    buf = C.create_string_buffer(512)
    L.mt3d_last_error(None, buf, 512)
    return buf.value.decode()

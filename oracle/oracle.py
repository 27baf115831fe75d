"""ctypes wrapper of the CPU oracle (``liboracle.so`` built from mt3d_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the cpu_baseline leg of bench.py, as the checker.  The product path never
imports it.

The oracle restates ModEM's matrix-free 3D-MT forward solver
(f90/3D_MT/FWD/modelOperator3D.f90, f90/3D_MT/FWD/EMsolve3D.f90,
f90/3D_MT/FWD/solver.f90) and the sensitivity glue
(f90/3D_MT/SolverSens.f90:63-116, f90/3D_MT/modelParam/ModelMap.inc).
Pinned against the reference's forward fixture
unit_testing/3D/CylinderModel_1per.dat: with the boundary conditions of
oracle/bc2d.py and the impedance functional of oracle/datafunc.py it
reproduces the file's 2501 impedance tensors to the 7 digits the file prints
(tests/test_golden.py).  Also checked against a closed-form layered solution,
scipy direct solves, the CC-DC/SP2 equivalence and operator identities
(tests/test_oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

QMR, BICG, COCG = 0, 1, 2
PC_DILU, PC_JACOBI, PC_RBDILU, PC_DILU_SWEEP, PC_ZLINE = 0, 1, 2, 3, 4

_lib = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (gcc)."""
    src = os.path.join(_HERE, "mt3d_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True, capture_output=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        I = C.c_int
        L.orc_create.restype = P
        L.orc_create.argtypes = [I, I, I, I, D, D, D]
        L.orc_destroy.argtypes = [P]
        L.orc_set_control.argtypes = [P, I, I, I, C.c_double, C.c_double, C.c_double, I, I]
        L.orc_update_cond.argtypes = [P, D, C.c_double]
        L.orc_update_freq.argtypes = [P, C.c_double]
        L.orc_multA.argtypes = [P, D, I, D]
        L.orc_divc.argtypes = [P, D, D]
        L.orc_divcgrad.argtypes = [P, D, D]
        L.orc_adjt_bc.argtypes = [P, D, D]
        L.orc_fwdsolve.restype = I
        L.orc_fwdsolve.argtypes = [P, I, D, D, D]
        L.orc_krylov.restype = I
        L.orc_krylov.argtypes = [P, D, D, I, C.c_double, D, C.POINTER(I)]
        L.orc_pmult_t.argtypes = [P, I, D, D, D, D]
        L.orc_model_to_edge.argtypes = [P, D, C.c_double, D, D]
        L.orc_nE.restype = C.c_long
        L.orc_nE.argtypes = [P]
        L.orc_nN.restype = C.c_long
        L.orc_nN.argtypes = [P]
        for name in ("orc_get_VE", "orc_get_VN", "orc_get_sigE", "orc_get_sigC"):
            getattr(L, name).argtypes = [P, D]
        L.orc_get_divcorr_coef.argtypes = [P, D, D, D]
        L.orc_get_diag.argtypes = [P, C.POINTER(I), C.POINTER(I), C.POINTER(I), D, D, C.POINTER(I)]
        L.orc_is_interior_edge.restype = I
        L.orc_is_interior_edge.argtypes = [P, C.c_long]
        L.orc_mu0.restype = C.c_double
        L.orc_sigma_air.restype = C.c_double
        _lib = L
    return _lib


def _d(a: np.ndarray):
    assert a.dtype in (np.float64, np.complex128) and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One model-operator context (grid, conductivity, frequency), mirroring
    the module state of f90/3D_MT/FWD/modelOperator3D.f90."""

    def __init__(self, grid):
        self.grid = grid
        L = lib()
        self._dx = np.ascontiguousarray(grid.dx, dtype=np.float64)
        self._dy = np.ascontiguousarray(grid.dy, dtype=np.float64)
        self._dz = np.ascontiguousarray(grid.dz, dtype=np.float64)
        self.h = L.orc_create(grid.nx, grid.ny, grid.nz, grid.nzAir, _d(self._dx), _d(self._dy), _d(self._dz))
        self.nE = L.orc_nE(self.h)
        self.nN = L.orc_nN(self.h)
        self.ctl = dict(IterPerDivCor=40, MaxDivCor=20, MaxIterDivCor=100, tolEMfwd=1e-7, tolEMadj=1e-7,
                        tolDivCor=1e-5, solver=QMR, precond=PC_DILU)

    def __del__(self):
        try:
            lib().orc_destroy(self.h)
        except Exception:
            pass

    def set_control(self, **kw):
        self.ctl.update(kw)
        c = self.ctl
        lib().orc_set_control(self.h, int(c["IterPerDivCor"]), int(c["MaxDivCor"]), int(c["MaxIterDivCor"]),
                              float(c["tolEMfwd"]), float(c["tolEMadj"]), float(c["tolDivCor"]),
                              int(c["solver"]), int(c["precond"]))

    def update_cond(self, m_earth: np.ndarray, air_cond: float):
        m = np.ascontiguousarray(m_earth, dtype=np.float64)
        lib().orc_update_cond(self.h, _d(m), float(air_cond))

    def update_freq(self, omega: float):
        lib().orc_update_freq(self.h, float(omega))

    def multA(self, x: np.ndarray, adjt: bool = False) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.nE, np.complex128)
        lib().orc_multA(self.h, _d(x), int(adjt), _d(y))
        return y

    def divc(self, e: np.ndarray) -> np.ndarray:
        e = np.ascontiguousarray(e, dtype=np.complex128)
        out = np.zeros(self.nN, np.complex128)
        lib().orc_divc(self.h, _d(e), _d(out))
        return out

    def divcgrad(self, phi: np.ndarray) -> np.ndarray:
        phi = np.ascontiguousarray(phi, dtype=np.complex128)
        out = np.zeros(self.nN, np.complex128)
        lib().orc_divcgrad(self.h, _d(phi), _d(out))
        return out

    def adjt_bc(self, e: np.ndarray) -> np.ndarray:
        e = np.ascontiguousarray(e, dtype=np.complex128)
        out = np.zeros(self.nE, np.complex128)
        lib().orc_adjt_bc(self.h, _d(e), _d(out))
        return out

    def fwdsolve(self, trans: bool = False, bc: np.ndarray | None = None, src: np.ndarray | None = None,
                 e0: np.ndarray | None = None):
        e = np.zeros(self.nE, np.complex128) if e0 is None else np.array(e0, dtype=np.complex128)
        bcp = None if bc is None else np.ascontiguousarray(bc, dtype=np.complex128)
        srcp = None if src is None else np.ascontiguousarray(src, dtype=np.complex128)
        rc = lib().orc_fwdsolve(self.h, int(trans), _d(bcp) if bcp is not None else None,
                                _d(srcp) if srcp is not None else None, _d(e))
        return e, rc

    def krylov(self, b: np.ndarray, x0: np.ndarray, maxit: int, tol: float):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = np.array(x0, dtype=np.complex128)
        rerr = np.zeros(maxit, np.float64)
        failed = C.c_int(0)
        n = lib().orc_krylov(self.h, _d(b), _d(x), int(maxit), float(tol), _d(rerr), C.byref(failed))
        return x, n, rerr, failed.value

    def diagnostics(self):
        c = self.ctl
        nit, ndc, fl = C.c_int(), C.c_int(), C.c_int()
        rel = np.zeros(c["MaxDivCor"] * c["IterPerDivCor"])
        divj = np.zeros(2 * c["MaxDivCor"])
        dci = np.zeros(c["MaxDivCor"], np.int32)
        lib().orc_get_diag(self.h, C.byref(nit), C.byref(ndc), C.byref(fl), _d(rel), _d(divj),
                           dci.ctypes.data_as(C.POINTER(C.c_int)))
        return dict(nIterTotal=nit.value, nDivCor=ndc.value, failed=bool(fl.value),
                    EMrelErr=rel[: nit.value].copy(), divJ=divj.reshape(-1, 2)[: ndc.value].copy(),
                    DivCorIters=dci[: ndc.value].copy())

    def pmult_t(self, e0: np.ndarray, eadj: np.ndarray, m0_earth: np.ndarray) -> np.ndarray:
        """e0, eadj: arrays of shape (npol, nE)."""
        e0 = np.ascontiguousarray(e0, dtype=np.complex128)
        ea = np.ascontiguousarray(eadj, dtype=np.complex128)
        npol = e0.shape[0] if e0.ndim == 2 else 1
        m0 = np.ascontiguousarray(m0_earth, dtype=np.float64)
        g = self.grid
        out = np.zeros(g.nx * g.ny * g.nzEarth)
        lib().orc_pmult_t(self.h, npol, _d(e0), _d(ea), _d(m0), _d(out))
        return out

    def model_to_edge(self, m_earth: np.ndarray, air_cond: float, m0_earth: np.ndarray | None = None):
        m = np.ascontiguousarray(m_earth, dtype=np.float64)
        m0 = None if m0_earth is None else np.ascontiguousarray(m0_earth, dtype=np.float64)
        out = np.zeros(self.nE)
        lib().orc_model_to_edge(self.h, _d(m), float(air_cond), _d(m0) if m0 is not None else None, _d(out))
        return out

    def _get(self, name, n):
        out = np.zeros(n)
        getattr(lib(), name)(self.h, _d(out))
        return out

    @property
    def VE(self):
        return self._get("orc_get_VE", self.nE)

    @property
    def VN(self):
        return self._get("orc_get_VN", self.nN)

    @property
    def sigE(self):
        return self._get("orc_get_sigE", self.nE)

    def divcorr_coef(self):
        db1, db2, c = np.zeros(self.nE), np.zeros(self.nE), np.zeros(self.nN)
        lib().orc_get_divcorr_coef(self.h, _d(db1), _d(db2), _d(c))
        return db1, db2, c

    def interior_mask(self) -> np.ndarray:
        return interior_edge_mask(self.grid)


def interior_edge_mask(grid) -> np.ndarray:
    """Boolean mask of interior edges in the full edge vector
    (boundaryIndex, f90/3D_MT/SP_Topology/vecTranslate.f90:436-526)."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    mx = np.zeros((nx, ny + 1, nz + 1), bool)
    mx[:, 1:ny, 1:nz] = True
    my = np.zeros((nx + 1, ny, nz + 1), bool)
    my[1:nx, :, 1:nz] = True
    mz = np.zeros((nx + 1, ny + 1, nz), bool)
    mz[1:nx, 1:ny, :] = True
    return np.concatenate([mx.ravel(order="F"), my.ravel(order="F"), mz.ravel(order="F")])

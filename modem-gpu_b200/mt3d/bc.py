"""Boundary data for the forward solve: tangential E on the boundary edges.

In ModEM the forward solve receives its boundary conditions from ``fwdSetup``
(f90/3D_MT/ForwardSolver.f90:333-460), which calls ``ComputeBC`` ->
``BC_x0_WS`` (f90/3D_MT/FWD/boundary_ws.f90:21-168): one 2D TE solve per grid
slice.  The library computes that on the device (mt3d_compute_bc); the
solve takes the boundary values as an input (a full edge vector whose
boundary entries are used), so any other boundary data can be passed too.

This module builds boundary data from 1D plane-wave solutions: for each
boundary edge column the 1D finite-difference problem of that column's
conductivity profile, discretised with exactly the z-part of the 3D curl-curl
stencil, normalised to E = 1 at the top of the air and E = 0 at the bottom
(the bottom boundary is zero in BC_x0_WS as well, boundary_ws.f90:160-161).
For a horizontally layered model the 3D discrete solution with these boundary
values equals the 1D solution on every column, which the tests use as a
closed-form check.

Polarisation numbering follows BC_x0_WS: mode 1 drives Ey (slices along y,
``E0%y``), mode 2 drives Ex (``E0%x``).
"""
from __future__ import annotations

import numpy as np

from .models import MU_0, SIGMA_AIR, Grid, Model


def _deltas(d: np.ndarray) -> np.ndarray:
    """delX etc. of setup_grid (f90/3D_MT/GridDef.f90:301-399), 0-based."""
    n = d.size
    out = np.empty(n + 1)
    out[0] = d[0]
    out[1:n] = d[:-1] + d[1:]
    out[n] = d[-1]
    return out / 2.0


def edge_conductivity(model: Model) -> np.ndarray:
    """Edge conductivity of the forward operator: ModelParamToEdge
    (f90/3D_MT/modelParam/ModelMap.inc:88-188, volume-weighted average of the
    adjacent cells) with the air edges (node planes / cells iz <= nzAir) set
    to zero as DivCorrSetUp leaves them (f90/3D_MT/FWD/modelOperator3D.f90:
    1625-1633).  Full edge vector."""
    g = model.grid
    nx, ny, nz, na = g.nx, g.ny, g.nz, g.nzAir
    sc = model.sigma_cells()
    vc = g.dx[:, None, None] * g.dy[None, :, None] * g.dz[None, None, :]
    num = sc * vc

    def avg_x(a):  # x-edges (nx, ny+1, nz+1): average over cells (iy-1,iy) x (iz-1,iz)
        p = np.zeros((nx, ny + 2, nz + 2))
        p[:, 1:-1, 1:-1] = a
        return p[:, :-1, :-1] + p[:, 1:, :-1] + p[:, :-1, 1:] + p[:, 1:, 1:]

    def avg_y(a):
        p = np.zeros((nx + 2, ny, nz + 2))
        p[1:-1, :, 1:-1] = a
        return p[:-1, :, :-1] + p[1:, :, :-1] + p[:-1, :, 1:] + p[1:, :, 1:]

    def avg_z(a):
        p = np.zeros((nx + 2, ny + 2, nz))
        p[1:-1, 1:-1, :] = a
        return p[:-1, :-1, :] + p[1:, :-1, :] + p[:-1, 1:, :] + p[1:, 1:, :]

    sx = avg_x(num) / avg_x(vc)
    sy = avg_y(num) / avg_y(vc)
    sz = avg_z(num) / avg_z(vc)
    sx[:nx, :ny, :na] = 0.0
    sy[:nx, :ny, :na] = 0.0
    sz[:nx, :ny, :na] = 0.0
    return np.concatenate([sx.ravel(order="F"), sy.ravel(order="F"), sz.ravel(order="F")])


def _solve_1d_columns(dz: np.ndarray, sig: np.ndarray, omega: float) -> np.ndarray:
    """Solve the 1D problems of many columns at once.

    sig: (ncol, nz+1) conductivity on the node planes (x/y-edge conductivity).
    Returns E (ncol, nz+1) with E[:,0] = 1 and E[:,nz] = 0.  Row iz (0-based,
    1..nz-1) reads  c2*E[iz+1] + c1*E[iz-1] - (c1+c2)*E[iz] - i*w*mu*sig*E[iz] = 0
    with c1 = -1/(delZ*dz[iz-1]), c2 = -1/(delZ*dz[iz]) (the xXZ coefficients of
    CurlcurleSetUp, f90/3D_MT/FWD/modelOperator3D.f90:434-437).
    """
    nz = dz.size
    dZ = _deltas(dz)
    ncol = sig.shape[0]
    m = nz - 1  # unknowns iz = 1..nz-1
    iz = np.arange(1, nz)
    c1 = -1.0 / (dZ[iz] * dz[iz - 1])
    c2 = -1.0 / (dZ[iz] * dz[iz])
    diag = -(c1 + c2)[None, :] - 1j * omega * MU_0 * sig[:, 1:nz]
    lower = np.broadcast_to(c1[None, :], (ncol, m)).astype(np.complex128)
    upper = np.broadcast_to(c2[None, :], (ncol, m)).astype(np.complex128)
    rhs = np.zeros((ncol, m), np.complex128)
    rhs[:, 0] -= c1[0] * 1.0  # E[0] = 1
    # Thomas algorithm, vectorised over columns
    cp = np.zeros((ncol, m), np.complex128)
    dp = np.zeros((ncol, m), np.complex128)
    cp[:, 0] = upper[:, 0] / diag[:, 0]
    dp[:, 0] = rhs[:, 0] / diag[:, 0]
    for k in range(1, m):
        den = diag[:, k] - lower[:, k] * cp[:, k - 1]
        cp[:, k] = upper[:, k] / den
        dp[:, k] = (rhs[:, k] - lower[:, k] * dp[:, k - 1]) / den
    x = np.zeros((ncol, m), np.complex128)
    x[:, -1] = dp[:, -1]
    for k in range(m - 2, -1, -1):
        x[:, k] = dp[:, k] - cp[:, k] * x[:, k + 1]
    E = np.zeros((ncol, nz + 1), np.complex128)
    E[:, 0] = 1.0
    E[:, 1:nz] = x
    return E


def boundary_1d(model: Model, omega: float, mode: int) -> np.ndarray:
    """Full edge vector holding plane-wave boundary values for polarisation
    ``mode`` (1: Ey, 2: Ex); interior entries are zero."""
    g = model.grid
    nx, ny, nz = g.nx, g.ny, g.nz
    sE = edge_conductivity(model)
    nX = nx * (ny + 1) * (nz + 1)
    nY = (nx + 1) * ny * (nz + 1)
    ex = np.zeros((nx, ny + 1, nz + 1), np.complex128)
    ey = np.zeros((nx + 1, ny, nz + 1), np.complex128)
    ez = np.zeros((nx + 1, ny + 1, nz), np.complex128)
    if mode == 2:
        sx = sE[:nX].reshape((nx, ny + 1, nz + 1), order="F")
        for iy in (0, ny):  # side faces iy = 1 and ny+1 (1-based)
            ex[:, iy, :] = _solve_1d_columns(g.dz, sx[:, iy, :], omega)
        # top and bottom faces: interior columns use their own profile
        cols = _solve_1d_columns(g.dz, sx.reshape(nx * (ny + 1), nz + 1), omega).reshape(nx, ny + 1, nz + 1)
        ex[:, :, 0] = cols[:, :, 0]
        ex[:, :, nz] = 0.0
    elif mode == 1:
        sy = sE[nX:nX + nY].reshape((nx + 1, ny, nz + 1), order="F")
        for ix in (0, nx):
            ey[ix, :, :] = _solve_1d_columns(g.dz, sy[ix, :, :], omega)
        cols = _solve_1d_columns(g.dz, sy.reshape((nx + 1) * ny, nz + 1), omega).reshape(nx + 1, ny, nz + 1)
        ey[:, :, 0] = cols[:, :, 0]
        ey[:, :, nz] = 0.0
    else:
        raise ValueError("mode must be 1 (Ey) or 2 (Ex)")
    return np.concatenate([ex.ravel(order="F"), ey.ravel(order="F"), ez.ravel(order="F")])


def layered_solution(model: Model, omega: float, mode: int) -> np.ndarray:
    """For a horizontally layered model: the exact discrete 3D solution (the
    1D solution on every column).  Used as a closed-form check."""
    g = model.grid
    nx, ny, nz = g.nx, g.ny, g.nz
    sE = edge_conductivity(model)
    nX = nx * (ny + 1) * (nz + 1)
    nY = (nx + 1) * ny * (nz + 1)
    ex = np.zeros((nx, ny + 1, nz + 1), np.complex128)
    ey = np.zeros((nx + 1, ny, nz + 1), np.complex128)
    ez = np.zeros((nx + 1, ny + 1, nz), np.complex128)
    if mode == 2:
        sx = sE[:nX].reshape((nx, ny + 1, nz + 1), order="F")
        e1 = _solve_1d_columns(g.dz, sx[nx // 2, ny // 2][None, :], omega)[0]
        ex[:] = e1[None, None, :]
    else:
        sy = sE[nX:nX + nY].reshape((nx + 1, ny, nz + 1), order="F")
        e1 = _solve_1d_columns(g.dz, sy[nx // 2, ny // 2][None, :], omega)[0]
        ey[:] = e1[None, None, :]
    return np.concatenate([ex.ravel(order="F"), ey.ravel(order="F"), ez.ravel(order="F")])

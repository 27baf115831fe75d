"""2-D boundary conditions of ModEM's 3D-MT forward problem restated with
numpy/scipy -- TEST INFRASTRUCTURE ONLY (the checker of mt3d_compute_bc).

Restates BC_x0_WS (f90/3D_MT/FWD/boundary_ws.f90:21-168), called through
ComputeBC (f90/3D_MT/FWD/modelOperator3D.f90:268-293), with the Weerachai
Siripunvaraporn 2-D TE code it wraps (f90/3D_MT/FWD/Mod2d):
  * for imode = 2 one 2-D TE problem per x-slice of the grid (horizontal axis
    y), the solution filling the x-edges; for imode = 1 one per y-slice
    (horizontal axis x), filling the y-edges;
  * SetupA_TE (WSfwd2Dmod.f90:325-418): 5-point operator on the interior
    nodes of the slice, the air rows at CondAir = SIGMA_AIR, the cell
    conductivity averaged over the four cells around each node with area
    weights;
  * SetBound2D_TE (:177-250): boundary values from 1-D TE solutions
    (Fwd1D_TE, WSfwd1Dmod.f90:70-126): the two side columns, the bottom row
    from the column conductivity averaged over the two cells next to each
    node, and 1 along the top of the air;
  * MulAibWithXb (:80-127) and the banded solve of FormAII / Fwd2DsolveTE
    (:32-76, FwdTEmod.f90:104-157), here a sparse direct solve;
  * getBC (f90/FIELDS/FiniteDiff3D/sg_boundary.f90:87-90) with the tangential
    field of the bottom face set to zero (boundary_ws.f90:155-156).
The period passed down is 2 pi / omega with the reference's pi, and the 2-D
code turns it back into 2 pi / period.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp
import scipy.sparse.linalg as spla

PI_REF = 3.14159265357898
MU_0 = PI_REF * 0.0000004
SIGMA_AIR = float(np.float32(1.0e-10))


def _centre_distance(d):
    """DistanceBetweenBlocks (WSutils.f90:182-193): c[0] = d[0],
    c[i] = d[i] + d[i-1], c[n] = d[n-1] (twice the node-centred widths)."""
    c = np.empty(d.size + 1)
    c[0] = d[0]
    c[1:-1] = d[1:] + d[:-1]
    c[-1] = d[-1]
    return c


def fwd1d_te(omega2, nza, dz, s_earth):
    """Fwd1D_TE: the 1-D TE field at the Nz+1 nodes of a column whose top node
    is 1; a half-space of the bottom cell's conductivity one skin depth thick
    closes it with a zero field."""
    nz = dz.size
    omue = omega2 * MU_0
    s1d = np.empty(nz + 1)
    s1d[:nza] = SIGMA_AIR
    s1d[nza:nz] = s_earth
    s1d[nz] = s1d[nz - 1]
    dz1 = np.append(np.asarray(dz, float), np.sqrt(2.0 / (s1d[nz] * omue)))
    au = 2.0 / dz1[:nz]
    ad = 2.0 / dz1[1:nz + 1]
    ss = s1d[1:nz + 1] * dz1[1:nz + 1] + s1d[:nz] * dz1[:nz]
    ac = 1j * omue * ss - au - ad
    ab = np.zeros((3, nz), complex)
    ab[0, 1:] = ad[:-1]
    ab[1] = ac
    ab[2, :-1] = ad[:-1]
    rhs = np.zeros(nz, complex)
    rhs[0] = -au[0]
    x = sla.solve_banded((1, 1), ab, rhs)
    return np.concatenate([[1.0 + 0j], x])


def fwd2d_te(omega2, nza, dy, dz, cond):
    """One slice: cond[ih, iz] (nh x nz cells, air rows ignored); returns the
    field at the (nh+1) x (nz+1) nodes."""
    ny, nz = dy.size, dz.size
    ccon = np.array(cond, float).copy()
    ccon[:, :nza] = SIGMA_AIR
    cy, cz = _centre_distance(dy), _centre_distance(dz)
    omue = omega2 * MU_0
    m = nz - 1
    n = (ny - 1) * m
    # interior nodes (iy, iz) = 1..ny-1, 1..nz-1 (0-based), iz fastest
    iy, iz = np.meshgrid(np.arange(1, ny), np.arange(1, nz), indexing="ij")
    iy, iz = iy.ravel(), iz.ravel()
    s00, s10 = ccon[iy, iz], ccon[iy, iz - 1]
    s01, s11 = ccon[iy - 1, iz], ccon[iy - 1, iz - 1]
    dzi, dzm, dyi, dym = dz[iz], dz[iz - 1], dy[iy], dy[iy - 1]
    s2d = (s00 * dzi * dyi + s01 * dzi * dym + s10 * dzm * dyi + s11 * dzm * dym) / \
        (dzi * dyi + dzi * dym + dzm * dyi + dzm * dym)
    ar, al = 2.0 * cz[iz] / dyi, 2.0 * cz[iz] / dym
    ad, au = 2.0 * cy[iy] / dzi, 2.0 * cy[iy] / dzm
    diag = (-ar - al - ad - au) + 1j * omue * (cy[iy] * cz[iz] * s2d)
    off1 = np.where(iz == nz - 1, 0.0, ad)[:-1]
    off2 = np.where(iy == ny - 1, 0.0, ar)[:n - m]
    A = sp.diags([diag, off1, off1, off2, off2], [0, 1, -1, m, -m], shape=(n, n), format="csc")

    # boundary values (SetBound2D_TE)
    earth = ccon[:, nza:]
    left = fwd1d_te(omega2, nza, dz, earth[0])
    right = fwd1d_te(omega2, nza, dz, earth[ny - 1])
    bottom = np.empty(ny + 1, complex)
    for j in range(1, ny):
        s = (earth[j - 1] * dy[j - 1] + earth[j] * dy[j]) / (dy[j - 1] + dy[j])
        bottom[j] = fwd1d_te(omega2, nza, dz, s)[nz]
    # right-hand side -Aib Xb (MulAibWithXb)
    b = np.zeros((ny - 1, m), complex)
    b[0, :] = -(2.0 * cz[1:nz] / dy[0]) * left[1:nz]
    b[ny - 2, :] = -(2.0 * cz[1:nz] / dy[ny - 1]) * right[1:nz]
    b[:, 0] -= 2.0 * cy[1:ny] / dz[0]
    b[:, m - 1] -= (2.0 * cy[1:ny] / dz[nz - 1]) * bottom[1:ny]
    x = spla.spsolve(A, b.ravel())
    e = np.empty((ny + 1, nz + 1), complex)
    e[1:ny, 1:nz] = x.reshape(ny - 1, m)
    e[0, :] = left
    e[ny, :] = right
    e[1:ny, 0] = 1.0
    e[1:ny, nz] = bottom[1:ny]
    return e


def compute_bc(grid, sigma_cells, omega, imode):
    """Full edge vector (getCVector order) of the 2-D initial field E0 with the
    bottom face's tangential values zeroed: its boundary entries are the BC,
    its interior entries the reference's first guess.
    sigma_cells: [nx, ny, nz] cell conductivity (air rows ignored)."""
    nx, ny, nz, nza = grid.nx, grid.ny, grid.nz, grid.nzAir
    omega2 = (2.0 * PI_REF) / ((2.0 * PI_REF) / omega)
    nX, nY = nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1)
    nZ = (nx + 1) * (ny + 1) * nz
    e = np.zeros(nX + nY + nZ, complex)
    if imode == 2:
        ex = np.zeros((nx, ny + 1, nz + 1), complex)
        for i in range(nx):
            ex[i] = fwd2d_te(omega2, nza, np.asarray(grid.dy, float), np.asarray(grid.dz, float), sigma_cells[i])
        ex[:, :, nz] = 0.0
        e[:nX] = ex.ravel(order="F")
    else:
        ey = np.zeros((nx + 1, ny, nz + 1), complex)
        for j in range(ny):
            ey[:, j, :] = fwd2d_te(omega2, nza, np.asarray(grid.dx, float), np.asarray(grid.dz, float),
                                   sigma_cells[:, j, :])
        ey[:, :, nz] = 0.0
        e[nX:nX + nY] = ey.ravel(order="F")
    return e


def sigma_cells(grid, m_earth, air_cond):
    """ModelParamToCell for LOGE: exp(m) in the earth, exp(airCond) in the air;
    [nx, ny, nz]."""
    nx, ny, nz, nza = grid.nx, grid.ny, grid.nz, grid.nzAir
    s = np.empty((nx, ny, nz))
    s[:, :, :nza] = np.exp(air_cond)
    s[:, :, nza:] = np.exp(np.asarray(m_earth, float).reshape(nx, ny, nz - nza, order="F"))
    return s

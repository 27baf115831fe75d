"""Shared test helpers: small grids/models and an independent sparse-matrix
assembly of the operator.

``assemble_cc`` restates the SP2 construction of the curl-curl operator
(CurlCurlSetUp, f90/3D_MT/FWD_SP2/modelOperator3D.f90:371-405):
CC = diag(EdgeL) T^T diag(DualEdgeL / FaceA) T diag(EdgeL), with the face-edge
incidence T of setCurlTopology (f90/3D_MT/SP_Topology/spOpTopology_SG.f90:24-140)
and the metric vectors of MetricElements_CSG.f90.  It is independent of the
matrix-free stencil that the oracle and the CUDA kernels implement, so
agreement pins the stencil.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from mt3d import bc as mbc
from mt3d import models


def small_grid(nx=10, ny=12, nair=4, nearth=8, seed=None):
    g = models.make_grid(nx, ny, nair, nearth, core=400.0, n_pad=2, pad_growth=1.6, air_first=60.0,
                         air_growth=2.0, earth_first=60.0, earth_growth=1.4)
    return g


def random_model(g, seed=1):
    lr = models.random_log10_rho(g, seed, corr_len=2.0)
    return models.Model(g, models.flat_f(models.loge_from_log10_rho(lr)))


def _deltas(d):
    out = np.empty(d.size + 1)
    out[0] = d[0]
    out[1:-1] = d[:-1] + d[1:]
    out[-1] = d[-1]
    return out / 2.0


def edge_index(g):
    nx, ny, nz = g.nx, g.ny, g.nz
    nX = nx * (ny + 1) * (nz + 1)
    nY = (nx + 1) * ny * (nz + 1)
    ix = lambda i, j, k: i + nx * (j + (ny + 1) * k)
    iy = lambda i, j, k: nX + i + (nx + 1) * (j + ny * k)
    iz = lambda i, j, k: nX + nY + i + (nx + 1) * (j + (ny + 1) * k)
    return ix, iy, iz


def assemble_cc(g):
    """Full-edge curl-curl matrix (real, symmetric), SP2 construction."""
    nx, ny, nz = g.nx, g.ny, g.nz
    dx, dy, dz = g.dx, g.dy, g.dz
    dX, dY, dZ = _deltas(dx), _deltas(dy), _deltas(dz)
    ix, iy, iz = edge_index(g)
    rows, cols, vals, fa, fl = [], [], [], [], []
    f = 0
    # x-faces (nx+1, ny, nz): +Ey(I,J,K) -Ey(I,J,K+1) -Ez(I,J,K) +Ez(I,J+1,K)
    for K in range(nz):
        for J in range(ny):
            for I in range(nx + 1):
                for e, v in ((iy(I, J, K), 1), (iy(I, J, K + 1), -1), (iz(I, J, K), -1), (iz(I, J + 1, K), 1)):
                    rows.append(f); cols.append(e); vals.append(v)
                fa.append(dy[J] * dz[K]); fl.append(dX[I]); f += 1
    # y-faces (nx, ny+1, nz): -Ex(I,J,K) +Ex(I,J,K+1) +Ez(I,J,K) -Ez(I+1,J,K)
    for K in range(nz):
        for J in range(ny + 1):
            for I in range(nx):
                for e, v in ((ix(I, J, K), -1), (ix(I, J, K + 1), 1), (iz(I, J, K), 1), (iz(I + 1, J, K), -1)):
                    rows.append(f); cols.append(e); vals.append(v)
                fa.append(dx[I] * dz[K]); fl.append(dY[J]); f += 1
    # z-faces (nx, ny, nz+1): +Ex(I,J,K) -Ex(I,J+1,K) -Ey(I,J,K) +Ey(I+1,J,K)
    for K in range(nz + 1):
        for J in range(ny):
            for I in range(nx):
                for e, v in ((ix(I, J, K), 1), (ix(I, J + 1, K), -1), (iy(I, J, K), -1), (iy(I + 1, J, K), 1)):
                    rows.append(f); cols.append(e); vals.append(v)
                fa.append(dx[I] * dy[J]); fl.append(dZ[K]); f += 1
    T = sp.csr_matrix((vals, (rows, cols)), shape=(f, g.n_edges))
    el = edge_lengths(g)
    W = sp.diags(np.asarray(fl) / np.asarray(fa))
    L = sp.diags(el)
    return (L @ T.T @ W @ T @ L).tocsr()


def edge_lengths(g):
    nx, ny, nz = g.nx, g.ny, g.nz
    lx = np.broadcast_to(g.dx[:, None, None], (nx, ny + 1, nz + 1)).ravel(order="F")
    ly = np.broadcast_to(g.dy[None, :, None], (nx + 1, ny, nz + 1)).ravel(order="F")
    lz = np.broadcast_to(g.dz[None, None, :], (nx + 1, ny + 1, nz)).ravel(order="F")
    return np.concatenate([lx, ly, lz])


def edge_volumes(g):
    nx, ny, nz = g.nx, g.ny, g.nz
    dX, dY, dZ = _deltas(g.dx), _deltas(g.dy), _deltas(g.dz)
    vx = (g.dx[:, None, None] * (dY[None, :, None] * dZ[None, None, :])).ravel(order="F")
    vy = (g.dy[None, :, None] * (dX[:, None, None] * dZ[None, None, :])).ravel(order="F")
    vz = (g.dz[None, None, :] * (dX[:, None, None] * dY[None, :, None])).ravel(order="F")
    return np.concatenate([vx, vy, vz])


def assemble_A(g, model, omega, air_sigma=0.0):
    """Full-edge A = CC - i omega mu0 sigma_E V_E (forward operator); air edges
    take air_sigma (zero in the operator the solver uses)."""
    cc = assemble_cc(g)
    s = mbc.edge_conductivity(model)
    if air_sigma:
        s = np.where(s == 0.0, air_sigma, s)
    return (cc - 1j * omega * models.MU_0 * sp.diags(s * edge_volumes(g))).tocsr()


def earth_mask(g, model):
    """Edges whose field is unique: A_II is singular on gradients of
    potentials supported on the air nodes (sigma = 0 there), which only touch
    air edges; the divergence correction fixes that part."""
    return mbc.edge_conductivity(model) > 0.0


def direct_solve(g, model, omega, bcv):
    """Solution of the interior system A_II e_I = -A_IB bc (scipy), with the
    air conductivity set to SIGMA_AIR so the system is non-singular; compare
    only on earth_mask edges."""
    from oracle.oracle import interior_edge_mask
    A = assemble_A(g, model, omega, air_sigma=models.SIGMA_AIR)
    m = interior_edge_mask(g)
    Aii = A[m][:, m].tocsc()
    Aib = A[m][:, ~m]
    b = -(Aib @ bcv[~m])
    import scipy.sparse.linalg as spla
    ei = spla.spsolve(Aii, b)
    e = bcv.copy()
    e[m] = ei
    return e, b


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

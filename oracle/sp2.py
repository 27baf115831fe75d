"""SP2 (curl-curl + grad-div, "CCGD") formulation restated with scipy sparse
matrices -- TEST INFRASTRUCTURE ONLY (the checker of the CUDA CCGD path).

Restates, for ModEM's FWD_SP2 solver:
  * CurlCurlSetUp (f90/3D_MT/FWD_SP2/modelOperator3D.f90:371-405):
      CC = diag(EdgeL) T^T diag(DualEdgeL / FaceA) T diag(EdgeL)
    with the face-edge incidence T of setCurlTopology
    (f90/3D_MT/SP_Topology/spOpTopology_SG.f90:24-140);
  * GradDivSetup2 (modelOperator3D.f90:916-1008) with airNIndex (:1086-1130):
      GD = diag(DualFaceA) G diag(Nair/Vnode) G^T diag(DualFaceA)
         + diag(DualFaceA) G diag(Nearth/(SigNode Vnode)) G^T diag(SigEdge DualFaceA)
      AAii = CCii + GDii,
    and the source-correction operator of the second half of GradDivSetup2
      GD2 = diag(1/EdgeL) G diag(Nearth/(SigNode Vnode)) G^T diag(DualFaceA);
  * UpdateCond / updateOmegaMuSig (:176-282): SigEdge = ModelParamToEdge with
    the boundary edges forced to zero, SigNode = ModelParamToNode,
    VomegaMuSig = mu0 omega SigEdge Vedge; Mult_Aii (:415-436):
      A = AAii + i ISIGN VomegaMuSig (ISIGN = -1);
  * FWDsolve3D (f90/3D_MT/FWD_SP2/EMsolve3D.f90:129-501): right-hand sides
      FWD: b = -CCib bc (+ V_E s + V_E GD2 (s / (i ISIGN w mu0)) for a source s)
      TRN: b = s + V_E GD2 (s / (i ISIGN w mu0) / V_E),
    post-processing of the transposed solution (e = V_E e, boundary
    bc - CCib^T e);
  * cuBiCG (f90/3D_MT/FWD_SP2/solver.f90:931-2009): BiCGStab restarted every
    120 iterations, the converged residual re-checked with b - A x, the best
    iterate returned when not converged.  The reference preconditions with a
    block D-ILU; the GPU path uses the diagonal, which this restatement
    applies too.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

PI_REF = 3.14159265357898
MU_0 = PI_REF * 0.0000004
SIGMA_AIR = float(np.float32(1.0e-10))
ISIGN = -1


def _deltas(d):
    out = np.empty(d.size + 1)
    out[0] = d[0]
    out[1:-1] = d[:-1] + d[1:]
    out[-1] = d[-1]
    return out / 2.0


def _grid_idx(shape):
    I, J, K = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    return I.ravel(order="F"), J.ravel(order="F"), K.ravel(order="F")


class Topology:
    """Edge/face/node numbering, incidence matrices and metric vectors."""

    def __init__(self, g):
        self.g = g
        nx, ny, nz = g.nx, g.ny, g.nz
        self.nX = nx * (ny + 1) * (nz + 1)
        self.nY = (nx + 1) * ny * (nz + 1)
        self.nZ = (nx + 1) * (ny + 1) * nz
        self.nE = self.nX + self.nY + self.nZ
        self.nN = (nx + 1) * (ny + 1) * (nz + 1)
        dX, dY, dZ = _deltas(g.dx), _deltas(g.dy), _deltas(g.dz)
        self.ix = lambda i, j, k: i + nx * (j + (ny + 1) * k)
        self.iy = lambda i, j, k: self.nX + i + (nx + 1) * (j + ny * k)
        self.iz = lambda i, j, k: self.nX + self.nY + i + (nx + 1) * (j + (ny + 1) * k)
        self.nd = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
        ex, ey, ez = _grid_idx((nx, ny + 1, nz + 1)), _grid_idx((nx + 1, ny, nz + 1)), _grid_idx((nx + 1, ny + 1, nz))
        self.ex, self.ey, self.ez = ex, ey, ez
        # metric vectors (GridCalc.f90 EdgeLength/EdgeArea/FaceLength/FaceArea)
        self.EdgeL = np.concatenate([g.dx[ex[0]], g.dy[ey[1]], g.dz[ez[2]]])
        self.DualFaceA = np.concatenate([dY[ex[1]] * dZ[ex[2]], dX[ey[0]] * dZ[ey[2]], dX[ez[0]] * dY[ez[1]]])
        self.Vedge = np.concatenate([g.dx[ex[0]] * (dY[ex[1]] * dZ[ex[2]]), g.dy[ey[1]] * (dX[ey[0]] * dZ[ey[2]]),
                                     g.dz[ez[2]] * (dX[ez[0]] * dY[ez[1]])])
        n = _grid_idx((nx + 1, ny + 1, nz + 1))
        self.Vnode = dX[n[0]] * dY[n[1]] * dZ[n[2]]
        self.node_boundary = (n[0] == 0) | (n[0] == nx) | (n[1] == 0) | (n[1] == ny) | (n[2] == 0) | (n[2] == nz)
        # interior edges (boundaryIndex)
        self.interior = np.concatenate([(ex[1] > 0) & (ex[1] < ny) & (ex[2] > 0) & (ex[2] < nz),
                                        (ey[0] > 0) & (ey[0] < nx) & (ey[2] > 0) & (ey[2] < nz),
                                        (ez[0] > 0) & (ez[0] < nx) & (ez[1] > 0) & (ez[1] < ny)])
        # G: edges x nodes, -1 at the start node, +1 at the end node (setGradTopology)
        rows = np.arange(self.nE)
        start = np.concatenate([self.nd(*ex), self.nd(*ey), self.nd(*ez)])
        end = np.concatenate([self.nd(ex[0] + 1, ex[1], ex[2]), self.nd(ey[0], ey[1] + 1, ey[2]),
                              self.nd(ez[0], ez[1], ez[2] + 1)])
        self.G = sp.csr_matrix((np.concatenate([-np.ones(self.nE), np.ones(self.nE)]),
                                (np.concatenate([rows, rows]), np.concatenate([start, end]))),
                               shape=(self.nE, self.nN))
        # T: faces x edges (setCurlTopology), faces ordered x-, y-, z-faces
        fx, fy, fz = _grid_idx((nx + 1, ny, nz)), _grid_idx((nx, ny + 1, nz)), _grid_idx((nx, ny, nz + 1))
        I, J, K = fx
        cx = [self.iy(I, J, K), self.iy(I, J, K + 1), self.iz(I, J, K), self.iz(I, J + 1, K)]
        I, J, K = fy
        cy = [self.ix(I, J, K), self.ix(I, J, K + 1), self.iz(I, J, K), self.iz(I + 1, J, K)]
        I, J, K = fz
        cz = [self.ix(I, J, K), self.ix(I, J + 1, K), self.iy(I, J, K), self.iy(I + 1, J, K)]
        sx, sy, sz = [1, -1, -1, 1], [-1, 1, 1, -1], [1, -1, -1, 1]
        nfx, nfy, nfz = fx[0].size, fy[0].size, fz[0].size
        r = np.concatenate([np.tile(np.arange(nfx), 4), nfx + np.tile(np.arange(nfy), 4),
                            nfx + nfy + np.tile(np.arange(nfz), 4)])
        c = np.concatenate(cx + cy + cz)
        v = np.concatenate([np.full(nfx, s) for s in sx] + [np.full(nfy, s) for s in sy] +
                           [np.full(nfz, s) for s in sz]).astype(float)
        self.T = sp.csr_matrix((v, (r, c)), shape=(nfx + nfy + nfz, self.nE))
        FaceA = np.concatenate([g.dy[fx[1]] * g.dz[fx[2]], g.dx[fy[0]] * g.dz[fy[2]], g.dx[fz[0]] * g.dy[fz[1]]])
        DualEdgeL = np.concatenate([dX[fx[0]], dY[fy[1]], dZ[fz[2]]])
        L = sp.diags(self.EdgeL)
        self.CC = (L @ self.T.T @ sp.diags(DualEdgeL / FaceA) @ self.T @ L).tocsr()


def cell_conductivity(model):
    return model.sigma_cells()


def edge_conductivity_sp2(topo: Topology, model) -> np.ndarray:
    """ModelParamToEdge (air cells at exp(airCond)) with boundary edges zero."""
    g = model.grid
    nx, ny, nz = g.nx, g.ny, g.nz
    sc = model.sigma_cells()
    vc = g.dx[:, None, None] * g.dy[None, :, None] * g.dz[None, None, :]

    def avg(a, axes):
        shp = [nx, ny, nz]
        pad = np.zeros([s + 2 for s in shp])
        pad[1:-1, 1:-1, 1:-1] = a
        out_shape = [shp[ax] + (ax in axes) for ax in range(3)]
        s = 0
        for da in (0, 1):
            for db in (0, 1):
                sl = []
                q = 0
                for ax in range(3):
                    if ax in axes:
                        o = (da, db)[q]
                        q += 1
                        sl.append(slice(o, o + out_shape[ax]))
                    else:
                        sl.append(slice(1, 1 + shp[ax]))
                s = s + pad[tuple(sl)]
        return s

    def e(axes):
        return (avg(sc * vc, axes) / avg(vc, axes)).ravel(order="F")

    s = np.concatenate([e((1, 2)), e((0, 2)), e((0, 1))])
    s[~topo.interior] = 0.0
    return s


def node_conductivity(topo: Topology, model) -> np.ndarray:
    """ModelParamToNode: volume-weighted average of the cells around a node."""
    g = model.grid
    nx, ny, nz = g.nx, g.ny, g.nz
    sc = model.sigma_cells()
    vc = g.dx[:, None, None] * g.dy[None, :, None] * g.dz[None, None, :]

    def c2n(a):
        p = np.zeros((nx + 2, ny + 2, nz + 2))
        p[1:-1, 1:-1, 1:-1] = a
        return sum(p[a0:a0 + nx + 1, b0:b0 + ny + 1, c0:c0 + nz + 1] for a0 in (0, 1) for b0 in (0, 1)
                   for c0 in (0, 1))

    return (c2n(sc * vc) / c2n(vc)).ravel(order="F")


class SP2:
    """CCGD operator and FWDsolve3D of the SP2 solver for one model."""

    def __init__(self, grid, model):
        self.topo = t = Topology(grid)
        self.sig_e = edge_conductivity_sp2(t, model)
        self.sig_n = node_conductivity(t, model)
        eearth = self.sig_e >= 1.1 * SIGMA_AIR
        nearth = (abs(t.G).T @ eearth.astype(float)) > 0
        nair = ~nearth
        nearth = nearth & ~t.node_boundary
        nair = nair & ~t.node_boundary
        self.nearth, self.nair = nearth, nair
        D = sp.diags(t.DualFaceA)
        GDa = D @ t.G @ sp.diags(nair / t.Vnode) @ t.G.T @ D
        GDe = D @ t.G @ sp.diags(nearth / (self.sig_n * t.Vnode)) @ t.G.T @ sp.diags(self.sig_e * t.DualFaceA)
        self.GD = (GDa + GDe).tocsr()
        self.GD2 = (sp.diags(1.0 / t.EdgeL) @ t.G @ sp.diags(nearth / (self.sig_n * t.Vnode)) @ t.G.T @ D).tocsr()
        m = t.interior
        self.AAii = (t.CC + self.GD)[m][:, m].tocsr()
        self.CCib = t.CC[m][:, ~m].tocsr()
        self.omega = None

    def set_freq(self, omega):
        t = self.topo
        self.omega = omega
        self.vwms = MU_0 * omega * self.sig_e[t.interior] * t.Vedge[t.interior]
        self.A = (self.AAii + 1j * ISIGN * sp.diags(self.vwms)).tocsr()

    def rhs(self, trans=False, bc=None, src=None):
        t = self.topo
        m = t.interior
        inv = 1.0 / (1j * ISIGN * self.omega * MU_0)
        if trans:
            si = src[m] * inv / t.Vedge[m]
            return src[m] + (self.GD2[m][:, m] @ si) * t.Vedge[m]
        b = np.zeros(m.sum(), complex)
        if bc is not None:
            b = b - self.CCib @ bc[~m]
        if src is not None:
            si = src[m] * inv
            b = b + src[m] * t.Vedge[m] + (self.GD2[m][:, m] @ si) * t.Vedge[m]
        return b

    def bicg(self, b, x, maxit, tol, restart=120):
        """cuBiCG with the diagonal preconditioner (see module docstring)."""
        A = self.A
        dinv = 1.0 / A.diagonal()
        bnorm = np.linalg.norm(b)
        r = b - A @ x
        rnorm = np.linalg.norm(r)
        btol = tol * bnorm
        rerr = [rnorm / bnorm]
        if rnorm <= btol:
            return x, 1, rerr, True
        x0 = x.copy()
        rnorm0 = rnorm
        for it in range(1, maxit + 1):
            if it % restart == 1:
                rt = r.copy()
                rho = np.vdot(rt, r)
                p = r.copy()
                omega = 1.0
            else:
                rho1 = rho
                rho = np.vdot(rt, r)
                beta = (rho / rho1) * (alpha / omega)
                p = r + beta * (p - omega * v)
            ph = dinv * p
            v = A @ ph
            alpha = rho / np.vdot(rt, v)
            x = x + alpha * ph
            s = r - alpha * v
            sh = dinv * s
            tt = A @ sh
            omega = np.vdot(tt, s) / np.vdot(tt, tt)
            x = x + omega * sh
            r = s - omega * tt
            rnorm = np.linalg.norm(r)
            rerr.append(rnorm / bnorm)
            if rnorm < btol:
                rt_true = b - A @ x
                rn = np.linalg.norm(rt_true)
                if rn < btol:
                    return x, it, rerr, True
            if rnorm < rnorm0:
                rnorm0 = rnorm
                x0 = x.copy()
        return x0, maxit, rerr, False

    def fwdsolve(self, trans=False, bc=None, src=None, maxit=2000, tol=1e-7):
        t = self.topo
        m = t.interior
        b = self.rhs(trans, bc, src)
        xi, it, rerr, conv = self.bicg(b, np.zeros(m.sum(), complex), maxit, tol)
        e = np.zeros(t.nE, complex)
        e[m] = xi
        if trans:
            sb = np.zeros(t.nE, complex)
            sb[~m] = self.CCib.T @ xi
            e = t.Vedge * e
            e[~m] = (bc[~m] if bc is not None else 0) - sb[~m]
        elif bc is not None:
            e[~m] = bc[~m]
        return e, it, rerr, conv

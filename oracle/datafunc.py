"""Full_Impedance data functional restated with numpy -- TEST INFRASTRUCTURE
ONLY (the checker of mt3d_impedance).

Restates, for ModEM's 3D-MT data functionals:
  * setup_grid coordinates (f90/3D_MT/GridDef.f90:301-394): xEdge, xCenter,
    ..., z measured down from the Earth's surface (zEdge(nzAir+1) = oz);
  * clean / minNode (f90/UTILS/utilities.f90:100-114, 196-225);
  * EinterpSetUp without conductivity weights
    (f90/3D_MT/EMfieldInterp.f90:141-324): trilinear weights of the edges of
    one component around a site;
  * BinterpSetUp (:329-465) and BfromESetUp (:470-647): magnetic field from
    the circulation of E around the faces next to the site, times
    i ISIGN / omega;
  * dataResp for Full_Impedance (f90/3D_MT/DataFunc.f90:143-189):
    Z = E B^-1 by Kramer's rule, site azimuths zero.
Functionals are lists of (flat edge index, complex coefficient); indices are
0-based in the getCVector order (x-edges, y-edges, z-edges, x fastest).
"""
from __future__ import annotations

import numpy as np

ISIGN = -1


def coords(dx, dy, dz, nz_air, origin=(0.0, 0.0, 0.0)):
    """1-based coordinate arrays (index 0 unused) of setup_grid."""
    dx, dy, dz = (np.asarray(a, float) for a in (dx, dy, dz))

    def dual(d):
        de = np.empty(d.size + 1)
        de[0] = d[0]
        de[1:-1] = d[:-1] + d[1:]
        de[-1] = d[-1]
        return de / 2.0

    c = {}
    for name, d, o in (("x", dx, origin[0]), ("y", dy, origin[1])):
        e = np.zeros(d.size + 2)
        e[1] = o
        e[2:] = np.cumsum(d) + o
        dd = dual(d)
        cen = np.zeros(d.size + 1)
        cen[1:] = np.cumsum(dd[:-1]) + o
        c[name + "E"], c[name + "C"] = e, cen
        c["d" + name], c["D" + name] = np.concatenate([[0.0], d]), np.concatenate([[0.0], dd])
    ze = np.zeros(dz.size + 2)
    ze[2:] = np.cumsum(dz)
    air = ze[nz_air + 1]
    ddz = dual(dz)
    zc = np.zeros(dz.size + 1)
    zc[1:] = np.cumsum(ddz[:-1])
    zc[1:] = zc[1:] - air + origin[2]
    ze[1:] = ze[1:] - air + origin[2]
    c["zE"], c["zC"], c["dz"], c["Dz"] = ze, zc, np.concatenate([[0.0], dz]), np.concatenate([[0.0], ddz])
    c["n"] = (dx.size, dy.size, dz.size)
    return c


def _clean(x):
    return np.round(x * 1.0e13) / 1.0e13


def _min_node(x, node, n):
    for i in range(1, n + 1):
        if _clean(node[i]) > _clean(x):
            return i - 1
    return n


def _weights(c, x, grids):
    """grids[a] = (kind, n0, nMax) with kind 'E' (edge) or 'C' (centre)."""
    w = np.zeros((3, 2))
    for a, ax in enumerate("xyz"):
        kind, n0, nmax = grids[a]
        if 0 < n0 < nmax:
            if kind == "C":
                w[a, 1] = (x[a] - c[ax + "C"][n0]) / c["D" + ax][n0 + 1]
            else:
                w[a, 1] = (x[a] - c[ax + "E"][n0]) / c["d" + ax][n0]
        else:
            w[a, 1] = 1.0 if n0 <= 0 else 0.0
        w[a, 0] = 1.0 - w[a, 1]
    return w


def _terms(w, comp, i0, j0, k0):
    out = []
    for n in range(2):
        for m in range(2):
            for p in range(2):
                wadd = w[0, n] * w[1, m] * w[2, p]
                if wadd > 0:
                    out.append((comp, i0 + n, j0 + m, k0 + p, complex(wadd)))
    return out


def e_interp(c, x, xyz):
    nx, ny, nz = c["n"]
    i0 = _min_node(x[0], c["xE"], nx + 1)
    j0 = _min_node(x[1], c["yE"], ny + 1)
    k0 = _min_node(x[2], c["zE"], nz + 1)
    g = [["E", i0, nx + 1], ["E", j0, ny + 1], ["E", k0, nz + 1]]
    a = xyz - 1
    ax = "xyz"[a]
    n = c["n"][a]
    g[a] = ["C", _min_node(x[a], c[ax + "C"], n), n]
    w = _weights(c, x, g)
    return _terms(w, xyz, g[0][1], g[1][1], g[2][1])


def b_interp(c, x, xyz):
    nx, ny, nz = c["n"]
    g = [["C", _min_node(x[0], c["xC"], nx), nx], ["C", _min_node(x[1], c["yC"], ny), ny],
         ["C", _min_node(x[2], c["zC"], nz), nz]]
    a = xyz - 1
    ax = "xyz"[a]
    n = c["n"][a]
    g[a] = ["E", _min_node(x[a], c[ax + "E"], n + 1), n + 1]
    w = _weights(c, x, g)
    return _terms(w, xyz, g[0][1], g[1][1], g[2][1])


def b_from_e(c, omega, x, xyz):
    ioi = ISIGN * 1j / omega
    dx, dy, dz = c["dx"], c["dy"], c["dz"]
    out = []
    for comp, I, J, K, wf in b_interp(c, x, xyz):
        if comp == 1:
            S = dy[J] * dz[K]
            e = [(2, I, J, K, dy[J] / S), (2, I, J, K + 1, -dy[J] / S), (3, I, J, K, -dz[K] / S),
                 (3, I, J + 1, K, dz[K] / S)]
        elif comp == 2:
            S = dx[I] * dz[K]
            e = [(3, I, J, K, dz[K] / S), (3, I + 1, J, K, -dz[K] / S), (1, I, J, K, -dx[I] / S),
                 (1, I, J, K + 1, dx[I] / S)]
        else:
            S = dx[I] * dy[J]
            e = [(1, I, J, K, dx[I] / S), (1, I, J + 1, K, -dx[I] / S), (2, I, J, K, -dy[J] / S),
                 (2, I + 1, J, K, dy[J] / S)]
        out += [(a, b, cc, d, v * wf * ioi) for a, b, cc, d, v in e]
    return out


def flat(c, comp, i, j, k):
    nx, ny, nz = c["n"]
    nX, nY = nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1)
    i, j, k = i - 1, j - 1, k - 1
    if comp == 1:
        assert 0 <= i < nx and 0 <= j <= ny and 0 <= k <= nz
        return i + nx * (j + (ny + 1) * k)
    if comp == 2:
        assert 0 <= i <= nx and 0 <= j < ny and 0 <= k <= nz
        return nX + i + (nx + 1) * (j + ny * k)
    assert 0 <= i <= nx and 0 <= j <= ny and 0 <= k < nz
    return nX + nY + i + (nx + 1) * (j + (ny + 1) * k)


def apply(c, terms, e):
    return sum(v * e[flat(c, a, i, j, k)] for a, i, j, k, v in terms)


def impedance(c, omega, sites, e1, e2):
    """[nsite, 2, 2] impedance tensors (E / B)."""
    Z = np.zeros((len(sites), 2, 2), complex)
    for s, x in enumerate(np.asarray(sites, float)):
        L = [e_interp(c, x, 1), e_interp(c, x, 2), b_from_e(c, omega, x, 1), b_from_e(c, omega, x, 2)]
        EE = np.array([[apply(c, L[i], e) for e in (e1, e2)] for i in (0, 1)])
        BB = np.array([[apply(c, L[2 + i], e) for e in (e1, e2)] for i in (0, 1)])
        det = BB[0, 0] * BB[1, 1] - BB[0, 1] * BB[1, 0]
        Bi = np.array([[BB[1, 1], -BB[0, 1]], [-BB[1, 0], BB[0, 0]]]) / det
        Z[s] = EE @ Bi
    return Z


def lmult_t(c, omega, sites, e1, e2, d):
    """Adjoint sources (s1, s2) of Lrows + LmultT for Full_Impedance
    (f90/3D_MT/DataFunc.f90:465-869, f90/SENS/DataSens.f90:130-225):
    s_k = sum_ij conj(d_ij) B^-1(k, j) (Le_i - Z_i1 Lbx - Z_i2 Lby)."""
    nE = e1.size
    out = [np.zeros(nE, complex), np.zeros(nE, complex)]
    d = np.asarray(d, complex).reshape(-1, 2, 2)
    for s, x in enumerate(np.asarray(sites, float)):
        L = [e_interp(c, x, 1), e_interp(c, x, 2), b_from_e(c, omega, x, 1), b_from_e(c, omega, x, 2)]
        EE = np.array([[apply(c, L[i], e) for e in (e1, e2)] for i in (0, 1)])
        BB = np.array([[apply(c, L[2 + i], e) for e in (e1, e2)] for i in (0, 1)])
        det = BB[0, 0] * BB[1, 1] - BB[0, 1] * BB[1, 0]
        Bi = np.array([[BB[1, 1], -BB[0, 1]], [-BB[1, 0], BB[0, 0]]]) / det
        Z = EE @ Bi
        for k in range(2):
            for i in range(2):
                for j in range(2):
                    w = np.conj(d[s, i, j]) * Bi[k, j]
                    for a, ii, jj, kk, v in L[i]:
                        out[k][flat(c, a, ii, jj, kk)] += w * v
                    for m in range(2):
                        for a, ii, jj, kk, v in L[2 + m]:
                            out[k][flat(c, a, ii, jj, kk)] -= w * Z[i, m] * v
    return out[0], out[1]

// colstencil.cuh -- column-marching form of the curl-curl + i*omega*mu*sigma
// edge stencil.
//
// A thread owns the column (i, j) of the staggered grid and marches the
// node planes k of its chunk [k0, k1).  At plane k it produces the three
// edges that hang off node (i, j, k): Ex(i,j,k), Ey(i,j,k) and Ez(i,j,k)
// (whichever exist).  Its own Ex/Ey values of planes k-1, k, k+1 and Ez of
// planes k-1, k stay in registers as a sliding window; values of the
// neighbouring columns come through the L1 read-only path, where the
// neighbouring threads have just brought them.  Adjacent threads own
// adjacent i, so every access is coalesced along x.  The 1-D geometry
// factors are loaded once per column (x, y) or once per plane (z).
//
// The arithmetic is the same as stencil() in common.cuh (the Maxwell
// operator of f90/3D_MT/FWD/modelOperator3D.f90:692-800 times V_E).
#pragma once
#include "common.cuh"

namespace mt3d {

template <typename T> struct ColGeo {
    // per column
    T dxi, delXi, rdxi, rdxim1;
    T dyj, delYj, rdyj, rdyjm1;
    bool hasX, hasY;        // Ex(i,j,.) / Ey(i,j,.) exist (i < nx / j < ny)
    bool intX, intY, intZ;  // in-plane interior tests of the three components
};

template <typename T> __device__ __forceinline__ ColGeo<T> col_geo(const Geo<T> &g, int i, int j)
{
    ColGeo<T> c;
    c.hasX = i < g.nx;
    c.hasY = j < g.ny;
    c.dxi = c.hasX ? g.dx[i] : T(0);
    c.rdxi = c.hasX ? g.rdx[i] : T(0);
    c.rdxim1 = i > 0 ? g.rdx[i - 1] : T(0);
    c.delXi = g.delX[i];
    c.dyj = c.hasY ? g.dy[j] : T(0);
    c.rdyj = c.hasY ? g.rdy[j] : T(0);
    c.rdyjm1 = j > 0 ? g.rdy[j - 1] : T(0);
    c.delYj = g.delY[j];
    c.intX = c.hasX && j >= 1 && j <= g.ny - 1;
    c.intY = c.hasY && i >= 1 && i <= g.nx - 1;
    c.intZ = i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1;
    return c;
}

template <typename T> struct PlaneGeo {
    T dzk, delZk, rdzk, rdzkm1;
};
template <typename T> __device__ __forceinline__ PlaneGeo<T> plane_geo(const Geo<T> &g, int k)
{
    PlaneGeo<T> p;
    p.dzk = k < g.nz ? g.dz[k] : T(0);
    p.rdzk = k < g.nz ? g.rdz[k] : T(0);
    p.rdzkm1 = k > 0 ? g.rdz[k - 1] : T(0);
    p.delZk = g.delZ[k];
    return p;
}

template <typename C> __device__ __forceinline__ C ldg_c(const C *p) { return __ldg(p); }

// Column march over planes [k0, k1) of column (i, j) for the input field x
// (one right-hand side).  For every existing edge at (i, j, k) calls
//   f(comp, e, interior, Ax, x_e, dterm)
// where Ax is (A x)_e for interior edges (undefined otherwise), x_e the
// input value and dterm = wmu * sigma_e * V_E the imaginary diagonal part.
//
// With phi non-null the grad-div term of the SP2 operator, DFA_e (phi_end -
// phi_start) (GradDivSetup2, f90/3D_MT/FWD_SP2/modelOperator3D.f90:916-1008),
// is added to every interior edge; phi holds the node potentials of x.
template <typename T, typename F>
__device__ __forceinline__ void col_march(const Geo<T> &g, const C2<T> *__restrict__ x, const T *__restrict__ sig,
                                          int i, int j, int k0, int k1, T wmu, F &&f,
                                          const C2<T> *__restrict__ phi = nullptr)
{
    using C = C2<T>;
    const ColGeo<T> cg = col_geo(g, i, j);
    const C zero = mk<T>(0, 0);
    const int sxj = g.nx, sxk = g.nx * (g.ny + 1);              // Ex strides (j, k)
    const int syj = g.nx + 1, syk = (g.nx + 1) * g.ny;          // Ey strides
    const int szj = g.nx + 1, szk = (g.nx + 1) * (g.ny + 1);    // Ez strides
    const int bx = i + sxj * j;                                  // Ex(i, j, 0)
    const int by = g.nXe + i + syj * j;                          // Ey(i, j, 0)
    const int bz = g.nXe + g.nYe + i + szj * j;                  // Ez(i, j, 0)
    // sliding windows of the own column
    C X0 = zero, X1 = zero, X2 = zero;  // Ex(k-1), Ex(k), Ex(k+1)
    C Y0 = zero, Y1 = zero, Y2 = zero;
    C Z0 = zero, Z1 = zero;             // Ez(k-1), Ez(k)
    if (cg.hasX) {
        if (k0 >= 1) X0 = ldg_c(x + bx + sxk * (k0 - 1));
        X1 = ldg_c(x + bx + sxk * k0);
    }
    if (cg.hasY) {
        if (k0 >= 1) Y0 = ldg_c(x + by + syk * (k0 - 1));
        Y1 = ldg_c(x + by + syk * k0);
    }
    if (k0 >= 1) Z0 = ldg_c(x + bz + szk * (k0 - 1));
    // node potentials phi(i, j, k) and phi(i, j, k+1) of the own node column
    const int bn = i + (g.nx + 1) * j, snj = g.nx + 1, snk = (g.nx + 1) * (g.ny + 1);
    C P0 = zero, P1 = zero;
    if (phi) P0 = ldg_c(phi + bn + snk * k0);
    for (int k = k0; k < k1; k++) {
        const PlaneGeo<T> pg = plane_geo(g, k);
        const bool kin = k >= 1 && k <= g.nz - 1;
        if (phi) P1 = (k < g.nz) ? ldg_c(phi + bn + snk * (k + 1)) : zero;
        X2 = (cg.hasX && k < g.nz) ? ldg_c(x + bx + sxk * (k + 1)) : zero;
        Y2 = (cg.hasY && k < g.nz) ? ldg_c(x + by + syk * (k + 1)) : zero;
        Z1 = (k < g.nz) ? ldg_c(x + bz + szk * k) : zero;
        // ---- Ex(i, j, k)
        if (cg.hasX) {
            const int e = bx + sxk * k;
            const T ve = cg.dxi * (cg.delYj * pg.delZk);
            const T dt = wmu * sig[e] * ve;
            C out = zero;
            const bool in = cg.intX && kin;
            if (in) {
                const int ey = by + syk * k;  // Ey(i, j, k)
                const int ez = bz + szk * k;  // Ez(i, j, k)
                const C yy = csub(cadd(csub(ldg_c(x + ey + 1), Y1), ldg_c(x + ey - syj)), ldg_c(x + ey + 1 - syj));
                const C zz = csub(cadd(csub(ldg_c(x + ez + 1), Z1), Z0), ldg_c(x + ez + 1 - szk));
                const C fyp = cscale(csub(ldg_c(x + e + sxj), X1), cg.rdyj);
                const C fym = cscale(csub(X1, ldg_c(x + e - sxj)), cg.rdyjm1);
                const C fzp = cscale(csub(X2, X1), pg.rdzk);
                const C fzm = cscale(csub(X1, X0), pg.rdzkm1);
                out = cadd(cscale(yy, pg.delZk), cscale(zz, cg.delYj));
                out = csub(out, cscale(csub(fyp, fym), cg.dxi * pg.delZk));
                out = csub(out, cscale(csub(fzp, fzm), cg.dxi * cg.delYj));
                out.x -= dt * X1.y;
                out.y += dt * X1.x;
                if (phi) out = cadd(out, cscale(csub(ldg_c(phi + bn + snk * k + 1), P0), cg.delYj * pg.delZk));
            }
            f(0, e, in, out, X1, dt);
        }
        // ---- Ey(i, j, k)
        if (cg.hasY) {
            const int e = by + syk * k;
            const T ve = cg.dyj * (cg.delXi * pg.delZk);
            const T dt = wmu * sig[e] * ve;
            C out = zero;
            const bool in = cg.intY && kin;
            if (in) {
                const int ez = bz + szk * k;  // Ez(i, j, k)
                const int ex = bx + sxk * k;  // Ex(i, j, k)
                const C zz = csub(cadd(csub(ldg_c(x + ez + szj), Z1), Z0), ldg_c(x + ez + szj - szk));
                const C xx = csub(cadd(csub(ldg_c(x + ex + sxj), X1), ldg_c(x + ex - 1)), ldg_c(x + ex - 1 + sxj));
                const C fzp = cscale(csub(Y2, Y1), pg.rdzk);
                const C fzm = cscale(csub(Y1, Y0), pg.rdzkm1);
                const C fxp = cscale(csub(ldg_c(x + e + 1), Y1), cg.rdxi);
                const C fxm = cscale(csub(Y1, ldg_c(x + e - 1)), cg.rdxim1);
                out = cadd(cscale(zz, cg.delXi), cscale(xx, pg.delZk));
                out = csub(out, cscale(csub(fzp, fzm), cg.dyj * cg.delXi));
                out = csub(out, cscale(csub(fxp, fxm), cg.dyj * pg.delZk));
                out.x -= dt * Y1.y;
                out.y += dt * Y1.x;
                if (phi) out = cadd(out, cscale(csub(ldg_c(phi + bn + snk * k + snj), P0), cg.delXi * pg.delZk));
            }
            f(1, e, in, out, Y1, dt);
        }
        // ---- Ez(i, j, k)
        if (k < g.nz) {
            const int e = bz + szk * k;
            const T ve = pg.dzk * (cg.delXi * cg.delYj);
            const T dt = wmu * sig[e] * ve;
            C out = zero;
            const bool in = cg.intZ;
            if (in) {
                const int ex = bx + sxk * k;  // Ex(i, j, k)
                const int ey = by + syk * k;  // Ey(i, j, k)
                const C xx = csub(cadd(csub(X2, X1), ldg_c(x + ex - 1)), ldg_c(x + ex - 1 + sxk));
                const C yy = csub(cadd(csub(Y2, Y1), ldg_c(x + ey - syj)), ldg_c(x + ey - syj + syk));
                const C fxp = cscale(csub(ldg_c(x + e + 1), Z1), cg.rdxi);
                const C fxm = cscale(csub(Z1, ldg_c(x + e - 1)), cg.rdxim1);
                const C fyp = cscale(csub(ldg_c(x + e + szj), Z1), cg.rdyj);
                const C fym = cscale(csub(Z1, ldg_c(x + e - szj)), cg.rdyjm1);
                out = cadd(cscale(xx, cg.delYj), cscale(yy, cg.delXi));
                out = csub(out, cscale(csub(fxp, fxm), pg.dzk * cg.delYj));
                out = csub(out, cscale(csub(fyp, fym), pg.dzk * cg.delXi));
                out.x -= dt * Z1.y;
                out.y += dt * Z1.x;
                if (phi) out = cadd(out, cscale(csub(P1, P0), cg.delXi * cg.delYj));
            }
            f(2, e, in, out, Z1, dt);
        }
        X0 = X1; X1 = X2;
        Y0 = Y1; Y1 = Y2;
        Z0 = Z1;
        P0 = P1;
    }
}

// V_E times the curl-curl diagonal, per component, from column/plane factors
template <typename T>
__device__ __forceinline__ T col_ccdiag(int comp, const ColGeo<T> &c, const PlaneGeo<T> &p)
{
    if (comp == 0) return c.dxi * p.delZk * (c.rdyj + c.rdyjm1) + c.dxi * c.delYj * (p.rdzk + p.rdzkm1);
    if (comp == 1) return c.dyj * c.delXi * (p.rdzk + p.rdzkm1) + c.dyj * p.delZk * (c.rdxi + c.rdxim1);
    return p.dzk * c.delYj * (c.rdxi + c.rdxim1) + p.dzk * c.delXi * (c.rdyj + c.rdyjm1);
}

}  // namespace mt3d

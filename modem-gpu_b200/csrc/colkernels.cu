// colkernels.cu -- column-marching kernels: operator apply, the z-line
// preconditioner and the Bi-CG iteration for the complex-symmetric system.
//
// Bi-CG on A x = b with A^T = A and the shadow residual chosen as conj(r0)
// generates shadow vectors that are the conjugates of the primary ones, so
// the method needs one operator application per iteration and bilinear
// (unconjugated) products: the conjugate-orthogonal CG (COCG).  Preconditioner
// M (complex symmetric): for Ex and Ey the exact tridiagonal solve along each
// vertical line of interior edges (the same-component z couplings of the
// curl-curl operator with the full diagonal), for Ez the diagonal.  The
// pivots of each line are factorised once per frequency (kc_zl_setup).
//
// Grids: blockIdx.x tiles the (i, j) columns (kColX x kColY threads),
// blockIdx.y the right-hand side, blockIdx.z (stencil kernels only) chunks of
// node planes.
#include <algorithm>
#include <atomic>

#include "colstencil.cuh"
#include "finalize.cuh"
#include "kernels.h"

namespace mt3d {

extern std::atomic<long long> g_launch_count;
static inline void counted(int n) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

constexpr int kColX = 32, kColY = 8;  // kThreads threads per block

__device__ __forceinline__ bool col_of(const ColMap &m, int nx, int ny, int &i, int &j)
{
    const int tx = blockIdx.x % m.tiles_x, ty = blockIdx.x / m.tiles_x;
    i = tx * kColX + (threadIdx.x % kColX);
    j = ty * kColY + (threadIdx.x / kColX);
    return i <= nx && j <= ny;
}

template <typename T> __device__ __forceinline__ T c_wmu(const OuterState *ost, int r, double dsgn)
{
    return (T)(dsgn * ost[r].omega * kMu0);
}

// bilinear product a*b accumulated into v[0], v[1]
template <typename C> __device__ __forceinline__ void acc_bil(double *v, C a, C b)
{
    v[0] += (double)a.x * b.x - (double)a.y * b.y;
    v[1] += (double)a.x * b.y + (double)a.y * b.x;
}

// ---------------------------------------------------------------------------
// y = A x on all edges (zero on boundary edges); optionally y = -A x
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) kc_apply(ColArgs<T> a, const C2<T> *x, C2<T> *y, int neg)
{
    const int r = blockIdx.y;
    int i, j;
    if (!col_of(a.map, a.g.nx, a.g.ny, i, j)) return;
    const size_t off = (size_t)r * a.stride;
    const int kc = (a.g.nz + 1 + gridDim.z - 1) / gridDim.z;
    const int k0 = blockIdx.z * kc, k1 = min(k0 + kc, a.g.nz + 1);
    const T wmu = c_wmu<T>(a.ost, r, a.dsgn);
    C2<T> *yo = y + off;
    col_march(a.g, x + off, a.sigma, i, j, k0, k1, wmu, [&](int, int e, bool in, C2<T> out, C2<T>, T) {
        if (!in) out = mk<T>(0, 0);
        if (neg) { out.x = -out.x; out.y = -out.y; }
        yo[e] = out;
    });
}

// ---------------------------------------------------------------------------
// z-line preconditioner set-up: pivots m_k = 1/(d_k - l_k c'_{k-1}) and
// c'_k = u_k m_k of every interior Ex / Ey vertical line; m = 1/d for Ez.
// ---------------------------------------------------------------------------
template <typename T> __global__ void __launch_bounds__(kThreads) kc_zl_setup(ColArgs<T> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    int i, j;
    if (!col_of(a.map, a.g.nx, a.g.ny, i, j)) return;
    const Geo<T> &g = a.g;
    const size_t off = (size_t)r * a.stride;
    const T wmu = c_wmu<T>(a.ost, r, a.dsgn);
    const ColGeo<T> cg = col_geo(g, i, j);
    C2<T> *M = a.zm + off, *CP = a.zc + off;
    const int bx = i + g.nx * j, by = g.nXe + i + (g.nx + 1) * j, bz = g.nXe + g.nYe + i + (g.nx + 1) * j;
    const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
    for (int comp = 0; comp < 2; comp++) {
        const bool live = comp == 0 ? cg.intX : cg.intY;
        if (!live) continue;
        const int base = comp == 0 ? bx : by, sk = comp == 0 ? sxk : syk;
        const T w = comp == 0 ? cg.dxi * cg.delYj : cg.dyj * cg.delXi;  // V_E * |xXZ| factor
        C2<T> cprev = mk<T>(0, 0);
        for (int k = 1; k <= g.nz - 1; k++) {
            const PlaneGeo<T> pg = plane_geo(g, k);
            const int e = base + sk * k;
            const T ve = comp == 0 ? cg.dxi * (cg.delYj * pg.delZk) : cg.dyj * (cg.delXi * pg.delZk);
            const T dr = col_ccdiag(comp, cg, pg), di = wmu * a.sigma[e] * ve;
            const T lo = -w * pg.rdzkm1, up = -w * pg.rdzk;
            C2<T> den = mk<T>(dr, di);
            if (k > 1) den = csub(den, cscale(cprev, lo));
            const T inv = T(1) / (den.x * den.x + den.y * den.y);
            const C2<T> m = mk<T>(den.x * inv, -den.y * inv);
            M[e] = m;
            cprev = cscale(m, up);
            CP[e] = cprev;
        }
    }
    if (cg.intZ) {
        for (int k = 0; k < g.nz; k++) {
            const PlaneGeo<T> pg = plane_geo(g, k);
            const int e = bz + szk * k;
            const T ve = pg.dzk * (cg.delXi * cg.delYj);
            const T dr = col_ccdiag(2, cg, pg), di = wmu * a.sigma[e] * ve;
            const T inv = T(1) / (dr * dr + di * di);
            M[e] = mk<T>(dr * inv, -di * inv);
        }
    }
}

// z-line solve of one interior Ex/Ey line: forward elimination already
// written as y into z[]; backward substitution z_k = y_k - c'_k z_{k+1},
// accumulating rho += r_k z_k (bilinear)
template <typename T>
__device__ __forceinline__ void zl_backward(const Geo<T> &g, int base, int sk, const C2<T> *__restrict__ CP,
                                            const C2<T> *__restrict__ r, C2<T> *__restrict__ z, double *rho)
{
    C2<T> znext = mk<T>(0, 0);
    for (int k = g.nz - 1; k >= 1; k--) {
        const int e = base + sk * k;
        const C2<T> zk = csub(z[e], cmul(CP[e], znext));
        z[e] = zk;
        acc_bil(rho, r[e], zk);
        znext = zk;
    }
}

// out = M^-1 in (z-line preconditioner) for every active, running right-hand
// side; used by BiCGStab for ph = M^-1 p and sh = M^-1 s
template <typename T>
__global__ void __launch_bounds__(kThreads) kc_prec(ColArgs<T> a, const C2<T> *in, C2<T> *out)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active || a.st[r].status != KS_RUNNING) return;
    int i, j;
    if (!col_of(a.map, a.g.nx, a.g.ny, i, j)) return;
    const Geo<T> &g = a.g;
    const size_t off = (size_t)r * a.stride;
    const C2<T> *R = in + off, *M = a.zm + off, *CP = a.zc + off;
    C2<T> *Z = out + off;
    const ColGeo<T> cg = col_geo(g, i, j);
    const int bx = i + g.nx * j, by = g.nXe + i + (g.nx + 1) * j, bz = g.nXe + g.nYe + i + (g.nx + 1) * j;
    const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
    for (int comp = 0; comp < 3; comp++) {
        const bool has = comp == 0 ? cg.hasX : comp == 1 ? cg.hasY : true;
        if (!has) continue;
        const bool lin = comp == 0 ? cg.intX : comp == 1 ? cg.intY : cg.intZ;
        const int base = comp == 0 ? bx : comp == 1 ? by : bz, sk = comp == 0 ? sxk : comp == 1 ? syk : szk;
        const int kmax = comp == 2 ? g.nz - 1 : g.nz;
        const T w = comp == 0 ? cg.dxi * cg.delYj : cg.dyj * cg.delXi;
        C2<T> yprev = mk<T>(0, 0);
        for (int k = 0; k <= kmax; k++) {
            const int e = base + sk * k;
            C2<T> zz = mk<T>(0, 0);
            if (comp == 2) {
                if (lin) zz = cmul(R[e], M[e]);
            } else if (lin && k >= 1 && k <= g.nz - 1) {
                const T lo = -w * plane_geo(g, k).rdzkm1;
                zz = cmul(csub(R[e], cscale(yprev, k > 1 ? lo : T(0))), M[e]);
                yprev = zz;
            }
            Z[e] = zz;
        }
        if (comp < 2 && lin) {
            C2<T> znext = mk<T>(0, 0);
            for (int k = g.nz - 1; k >= 1; k--) {
                const int e = base + sk * k;
                const C2<T> zk = csub(Z[e], cmul(CP[e], znext));
                Z[e] = zk;
                znext = zk;
            }
        }
    }
}

// z = M^-1 r and rho = r . z, |r|^2 (start of a call)
template <typename T> __global__ void __launch_bounds__(kThreads) kc_cocg_start(ColArgs<T> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    BicgState &st = a.st[r];
    int i, j;
    const bool live = col_of(a.map, a.g.nx, a.g.ny, i, j);
    double v[2] = {0, 0};
    if (live && st.status == KS_RUNNING) {
        const Geo<T> &g = a.g;
        const size_t off = (size_t)r * a.stride;
        const C2<T> *R = a.r + off, *M = a.zm + off, *CP = a.zc + off;
        C2<T> *Z = a.z + off;
        const ColGeo<T> cg = col_geo(g, i, j);
        const int bx = i + g.nx * j, by = g.nXe + i + (g.nx + 1) * j, bz = g.nXe + g.nYe + i + (g.nx + 1) * j;
        const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
        for (int comp = 0; comp < 3; comp++) {
            const bool has = comp == 0 ? cg.hasX : comp == 1 ? cg.hasY : true;
            if (!has) continue;
            const bool lin = comp == 0 ? cg.intX : comp == 1 ? cg.intY : cg.intZ;
            const int base = comp == 0 ? bx : comp == 1 ? by : bz, sk = comp == 0 ? sxk : comp == 1 ? syk : szk;
            const int kmax = comp == 2 ? g.nz - 1 : g.nz;
            const T w = comp == 0 ? cg.dxi * cg.delYj : cg.dyj * cg.delXi;
            C2<T> yprev = mk<T>(0, 0);
            for (int k = 0; k <= kmax; k++) {
                const int e = base + sk * k;
                const C2<T> rr = R[e];
                C2<T> zz = mk<T>(0, 0);
                if (comp == 2) {
                    if (lin) { zz = cmul(rr, M[e]); acc_bil(v, rr, zz); }
                } else if (lin && k >= 1 && k <= g.nz - 1) {
                    const T lo = -w * plane_geo(g, k).rdzkm1;
                    zz = cmul(csub(rr, cscale(yprev, k > 1 ? lo : T(0))), M[e]);
                    yprev = zz;
                }
                Z[e] = zz;
            }
            if (comp < 2 && lin) zl_backward(g, base, sk, CP, R, Z, v);
        }
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        if (st.status == KS_RUNNING) {
            st.rho = {tot[0], tot[1]};
            st.beta = {0.0, 0.0};
            st.first = 1;
            if (!cd_finite(st.rho)) st.status = KS_NAN;
            else if (cd_zero(st.rho)) st.status = KS_BREAKDOWN;
        }
    }
}

// p = z (first iteration) or p = z + beta p
template <typename T> __global__ void __launch_bounds__(kThreads) kc_p(ColArgs<T> a, int nE)
{
    const int r = blockIdx.y;
    const BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const C2<T> be = mk<T>((T)st.beta.re, (T)st.beta.im);
    const bool first = st.first;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < nE; e += gridDim.x * kThreads) {
        const C2<T> zz = a.z[off + e];
        a.p[off + e] = first ? zz : cadd(zz, cmul(be, a.p[off + e]));
    }
}

// q = A p ; mu = p . q (bilinear) ; alpha = rho / mu
template <typename T> __global__ void __launch_bounds__(kThreads) kc_q(ColArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    int i, j;
    const bool live = col_of(a.map, a.g.nx, a.g.ny, i, j);
    double v[2] = {0, 0};
    if (live) {
        const size_t off = (size_t)r * a.stride;
        const int kc = (a.g.nz + 1 + gridDim.z - 1) / gridDim.z;
        const int k0 = blockIdx.z * kc, k1 = min(k0 + kc, a.g.nz + 1);
        const T wmu = c_wmu<T>(a.ost, r, a.dsgn);
        C2<T> *q = a.q + off;
        col_march(a.g, a.p + off, a.sigma, i, j, k0, k1, wmu, [&](int, int e, bool in, C2<T> out, C2<T> pe, T) {
            if (!in) out = mk<T>(0, 0);
            else acc_bil(v, pe, out);
            q[e] = out;
        });
    }
    const int blk = blockIdx.x + gridDim.x * blockIdx.z, nblk = gridDim.x * gridDim.z;
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blk, nblk, tot) && threadIdx.x == 0) {
        cd mu = {tot[0], tot[1]};
        if (!cd_finite(mu)) { st.status = KS_NAN; return; }
        if (cd_zero(mu)) { st.status = KS_BREAKDOWN; return; }
        st.alpha = cd_div(st.rho, mu);
        if (cd_zero(st.alpha)) st.status = KS_BREAKDOWN;
    }
}

// x += alpha p (best-iterate double buffer), r -= alpha q, z = M^-1 r (z-line
// solves on the thread's column), |r|, rho_new = r . z ; convergence, best
// iterate, beta
template <typename T> __global__ void __launch_bounds__(kThreads) kc_xrz(ColArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    int i, j;
    const bool live = col_of(a.map, a.g.nx, a.g.ny, i, j);
    double v[4] = {0, 0, 0, 0};  // rho (2), |r|^2, pad
    const int cur = st.xcur, dst = (st.xcur == st.xbest) ? 1 - st.xcur : st.xcur;
    if (live) {
        const Geo<T> &g = a.g;
        const size_t off = (size_t)r * a.stride;
        const C2<T> al = mk<T>((T)st.alpha.re, (T)st.alpha.im);
        const C2<T> *xs = (cur == 0 ? a.x0 : a.x1) + off;
        C2<T> *xd = (dst == 0 ? a.x0 : a.x1) + off;
        const C2<T> *P = a.p + off, *Q = a.q + off, *M = a.zm + off, *CP = a.zc + off;
        C2<T> *R = a.r + off, *Z = a.z + off;
        const ColGeo<T> cg = col_geo(g, i, j);
        const int bx = i + g.nx * j, by = g.nXe + i + (g.nx + 1) * j, bz = g.nXe + g.nYe + i + (g.nx + 1) * j;
        const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
        for (int comp = 0; comp < 3; comp++) {
            const bool has = comp == 0 ? cg.hasX : comp == 1 ? cg.hasY : true;
            if (!has) continue;
            const bool lin = comp == 0 ? cg.intX : comp == 1 ? cg.intY : cg.intZ;
            const int base = comp == 0 ? bx : comp == 1 ? by : bz, sk = comp == 0 ? sxk : comp == 1 ? syk : szk;
            const int kmax = comp == 2 ? g.nz - 1 : g.nz;
            const T w = comp == 0 ? cg.dxi * cg.delYj : cg.dyj * cg.delXi;
            C2<T> yprev = mk<T>(0, 0);
            for (int k = 0; k <= kmax; k++) {
                const int e = base + sk * k;
                xd[e] = cadd(xs[e], cmul(al, P[e]));
                const C2<T> rr = csub(R[e], cmul(al, Q[e]));
                R[e] = rr;
                v[2] += (double)rr.x * rr.x + (double)rr.y * rr.y;
                C2<T> zz = mk<T>(0, 0);
                if (comp == 2) {
                    if (lin) { zz = cmul(rr, M[e]); acc_bil(v, rr, zz); }
                } else if (lin && k >= 1 && k <= g.nz - 1) {
                    const T lo = -w * plane_geo(g, k).rdzkm1;
                    zz = cmul(csub(rr, cscale(yprev, k > 1 ? lo : T(0))), M[e]);
                    yprev = zz;
                }
                Z[e] = zz;
            }
            if (comp < 2 && lin) zl_backward(g, base, sk, CP, R, Z, v);
        }
    }
    double tot[4];
    if (block_reduce_last<4>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        const double rnorm = sqrt(tot[2]);
        st.iter += 1;
        st.xcur = dst;
        st.first = 0;
        st.rnorm = rnorm;
        rerr[st.iter - 1] = rnorm / st.bnorm;
        if (!isfinite(rnorm)) { st.status = KS_NAN; return; }
        if (rnorm < st.btol) { st.status = KS_CONVERGED; st.xbest = dst; return; }
        if (rnorm < st.rnormin) { st.rnormin = rnorm; st.xbest = dst; st.imin = st.iter; }
        if (st.iter >= st.maxit) { st.status = KS_MAXIT; return; }
        const cd rho_new = {tot[0], tot[1]};
        if (!cd_finite(rho_new)) { st.status = KS_NAN; return; }
        if (cd_zero(rho_new)) { st.status = KS_BREAKDOWN; return; }
        st.beta = cd_div(rho_new, st.rho);
        st.rho = rho_new;
    }
}

// ---------------------------------------------------------------------------
// BiCGStab stencil kernels in column-marching form (KArgs; flat elementwise
// kernels do the vector updates).  blockIdx.z chunks the node planes; the
// reduction counts (x, z) blocks per right-hand side.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ void kb_range(const Geo<T> &g, int &k0, int &k1)
{
    const int kc = (g.nz + 1 + gridDim.z - 1) / gridDim.z;
    k0 = blockIdx.z * kc;
    k1 = min(k0 + kc, g.nz + 1);
}
template <typename T> __device__ __forceinline__ const C2<T> *kb_phi(const KArgs<T> &a, int r)
{
    return a.gd ? a.phi + (size_t)r * a.g.nN : nullptr;
}

// start of a call: r = b - A x0, rt = r; |b|^2, |r|^2
template <typename T> __global__ void __launch_bounds__(kThreads) kcb_init(KArgs<T> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    BicgState &st = a.st[r];
    int i, j;
    double v[2] = {0.0, 0.0};
    if (col_of(a.cmap, a.g.nx, a.g.ny, i, j)) {
        const size_t off = (size_t)r * a.stride;
        int k0, k1;
        kb_range(a.g, k0, k1);
        const C2<T> *b = a.b + off;
        C2<T> *R = a.r + off, *RT = a.rt + off;
        col_march(a.g, a.x0 + off, a.sigma, i, j, k0, k1, c_wmu<T>(a.ost, r, a.dsgn),
                  [&](int, int e, bool in, C2<T> ax, C2<T>, T) {
                      C2<T> res = mk<T>(0, 0);
                      if (in) {
                          const C2<T> bb = b[e];
                          res = csub(bb, ax);
                          v[0] += (double)bb.x * bb.x + (double)bb.y * bb.y;
                          v[1] += (double)res.x * res.x + (double)res.y * res.y;
                      }
                      R[e] = res;
                      RT[e] = res;
                  },
                  kb_phi(a, r));
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0)
        fin_init(st, tot, a.rerr + (size_t)r * a.rerr_stride, a.maxit, a.inner ? a.ost[r].tol_inner : a.ost[r].tol);
}

// v = A ph ; rtv = rt . v ; alpha = rho / rtv   (which = 0)
// t = A sh ; ts = t . s, tt = t . t ; omega     (which = 1)
template <typename T> __global__ void __launch_bounds__(kThreads) kcb_vt(KArgs<T> a, int which)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    int i, j;
    double v[3] = {0.0, 0.0, 0.0};
    if (col_of(a.cmap, a.g.nx, a.g.ny, i, j)) {
        const size_t off = (size_t)r * a.stride;
        int k0, k1;
        kb_range(a.g, k0, k1);
        const C2<T> *in = (which ? a.sh : a.ph) + off;
        const C2<T> *w = (which ? a.s : a.rt) + off;
        C2<T> *out = (which ? a.t : a.v) + off;
        col_march(a.g, in, a.sigma, i, j, k0, k1, c_wmu<T>(a.ost, r, a.dsgn),
                  [&](int, int e, bool inn, C2<T> y, C2<T>, T) {
                      if (!inn) {
                          y = mk<T>(0, 0);
                      } else if (which == 0) {
                          const C2<T> t = w[e];
                          v[0] += (double)t.x * y.x + (double)t.y * y.y;  // conj(rt) v
                          v[1] += (double)t.x * y.y - (double)t.y * y.x;
                      } else {
                          const C2<T> s = w[e];
                          v[0] += (double)y.x * s.x + (double)y.y * s.y;  // conj(t) s
                          v[1] += (double)y.x * s.y - (double)y.y * s.x;
                          v[2] += (double)y.x * y.x + (double)y.y * y.y;
                      }
                      out[e] = y;
                  },
                  kb_phi(a, r));
    }
    double tot[3];
    if (block_reduce_last<3>(v, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0) {
        if (which == 0) fin_v(st, tot);
        else fin_t(st, tot);
    }
}

// true FP64 residual r = b - A X (refinement loop); |r|^2 -> relres, scale
__global__ void __launch_bounds__(kThreads) kcb_res64(KArgs<double> a)
{
    const int r = blockIdx.y;
    OuterState &os = a.ost[r];
    if (!os.active) return;
    int i, j;
    double v[1] = {0.0};
    if (col_of(a.cmap, a.g.nx, a.g.ny, i, j)) {
        const size_t off = (size_t)r * a.stride;
        int k0, k1;
        kb_range(a.g, k0, k1);
        const double2 *b = a.b + off;
        double2 *R = a.r + off;
        col_march(a.g, a.x0 + off, a.sigma, i, j, k0, k1, c_wmu<double>(a.ost, r, a.dsgn),
                  [&](int, int e, bool in, double2 ax, double2, double) {
                      double2 res = make_double2(0, 0);
                      if (in) {
                          res = csub(b[e], ax);
                          v[0] += res.x * res.x + res.y * res.y;
                      }
                      R[e] = res;
                  },
                  kb_phi(a, r));
    }
    double tot[1];
    if (block_reduce_last<1>(v, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0)
        fin_res64(os, tot);
}

// inverse diagonal of A (curl-curl diagonal, grad-div diagonal, i*dterm) for
// the diagonal preconditioner, interior edges; zero on boundary edges
template <typename T> __global__ void __launch_bounds__(kThreads) kcb_jacobi(KArgs<T> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    int i, j;
    if (!col_of(a.cmap, a.g.nx, a.g.ny, i, j)) return;
    const Geo<T> &g = a.g;
    const size_t off = (size_t)r * a.stride;
    const T wmu = c_wmu<T>(a.ost, r, a.dsgn);
    const ColGeo<T> cg = col_geo(g, i, j);
    C2<T> *J = a.jinv + (a.padded ? (size_t)r * a.pl.len() : off);
    const int bx = i + g.nx * j, by = g.nXe + i + (g.nx + 1) * j, bz = g.nXe + g.nYe + i + (g.nx + 1) * j;
    const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
    const int bn = i + (g.nx + 1) * j, snj = g.nx + 1, snk = (g.nx + 1) * (g.ny + 1);
    int k0, k1;
    kb_range(g, k0, k1);
    for (int k = k0; k < k1; k++) {
        const PlaneGeo<T> pg = plane_geo(g, k);
        const bool kin = k >= 1 && k <= g.nz - 1;
        for (int comp = 0; comp < 3; comp++) {
            const bool has = comp == 0 ? cg.hasX : comp == 1 ? cg.hasY : k < g.nz;
            if (!has) continue;
            const int e = comp == 0 ? bx + sxk * k : comp == 1 ? by + syk * k : bz + szk * k;
            const bool in = comp == 0 ? (cg.intX && kin) : comp == 1 ? (cg.intY && kin) : cg.intZ;
            C2<T> m = mk<T>(0, 0);
            if (in) {
                const T sg = a.sigma[e];
                const T ve = comp == 0 ? cg.dxi * (cg.delYj * pg.delZk)
                           : comp == 1 ? cg.dyj * (cg.delXi * pg.delZk) : pg.dzk * (cg.delXi * cg.delYj);
                T dr = col_ccdiag(comp, cg, pg);
                if (a.gd) {
                    const int ns = bn + snk * k, ne = ns + (comp == 0 ? 1 : comp == 1 ? snj : snk);
                    const T dfa = comp == 0 ? cg.delYj * pg.delZk : comp == 1 ? cg.delXi * pg.delZk : cg.delXi * cg.delYj;
                    const T cs = a.gde[ns] ? sg : T(1), ce = a.gde[ne] ? sg : T(1);
                    dr += dfa * dfa * (a.gdw[ns] * cs + a.gdw[ne] * ce);
                }
                const T di = wmu * sg * ve;
                const T inv = T(1) / (dr * dr + di * di);
                m = mk<T>(dr * inv, -di * inv);
            }
            J[a.padded ? a.pl.idx(comp, i, j, k) : e] = m;
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int zchunks(int nz, int ntiles, int)
{
    // ~8 blocks per SM for one right-hand side (the blocks of converged ones
    // exit at once), chunks of >= 8 planes
    const int want = std::max(1, (148 * 8) / std::max(1, ntiles));
    return std::max(1, std::min(want, (nz + 1) / 8));
}

template <typename T> void launch_col_apply(const ColArgs<T> &a, const C2<T> *x, C2<T> *y, int neg, int nrhs,
                                            cudaStream_t s)
{
    counted(1);
    kc_apply<T><<<dim3(a.map.tiles, nrhs, zchunks(a.g.nz, a.map.tiles, nrhs)), kThreads, 0, s>>>(a, x, y, neg);
}
template <typename T> void launch_zl_setup(const ColArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kc_zl_setup<T><<<dim3(a.map.tiles, nrhs), kThreads, 0, s>>>(a);
}
template <typename T> void launch_cocg_start(const ColArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kc_cocg_start<T><<<dim3(a.map.tiles, nrhs), kThreads, 0, s>>>(a);
}
template <typename T> void launch_cocg_iter(const ColArgs<T> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev)
{
    counted(3);
    const int nE = a.g.nE;
    const int gp = std::min((nE + kThreads - 1) / kThreads, 148 * 16);
    kc_p<T><<<dim3(gp, nrhs), kThreads, 0, s>>>(a, nE);
    if (ev) cudaEventRecord(ev[0], s);
    kc_q<T><<<dim3(a.map.tiles, nrhs, zchunks(a.g.nz, a.map.tiles, nrhs)), kThreads, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[1], s);
    kc_xrz<T><<<dim3(a.map.tiles, nrhs), kThreads, 0, s>>>(a);
}
template <typename T> void launch_col_prec(const ColArgs<T> &a, const C2<T> *in, C2<T> *out, int nrhs, cudaStream_t s)
{
    counted(1);
    kc_prec<T><<<dim3(a.map.tiles, nrhs), kThreads, 0, s>>>(a, in, out);
}
template <typename T> void launch_colb_init(const KArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kcb_init<T><<<dim3(a.cmap.tiles, nrhs, zchunks(a.g.nz, a.cmap.tiles, nrhs)), kThreads, 0, s>>>(a);
}
template <typename T> void launch_colb_vt(const KArgs<T> &a, int which, int nrhs, cudaStream_t s)
{
    counted(1);
    kcb_vt<T><<<dim3(a.cmap.tiles, nrhs, zchunks(a.g.nz, a.cmap.tiles, nrhs)), kThreads, 0, s>>>(a, which);
}
void launch_colb_res64(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kcb_res64<<<dim3(a.cmap.tiles, nrhs, zchunks(a.g.nz, a.cmap.tiles, nrhs)), kThreads, 0, s>>>(a);
}
template <typename T> void launch_colb_jacobi(const KArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kcb_jacobi<T><<<dim3(a.cmap.tiles, nrhs, zchunks(a.g.nz, a.cmap.tiles, nrhs)), kThreads, 0, s>>>(a);
}
ColMapHost col_map(int nx, int ny)
{
    ColMapHost m;
    m.tiles_x = (nx + 1 + kColX - 1) / kColX;
    m.tiles = m.tiles_x * ((ny + 1 + kColY - 1) / kColY);
    return m;
}

#define INST(T)                                                                                                       \
    template void launch_col_apply<T>(const ColArgs<T> &, const C2<T> *, C2<T> *, int, int, cudaStream_t);            \
    template void launch_zl_setup<T>(const ColArgs<T> &, int, cudaStream_t);                                          \
    template void launch_cocg_start<T>(const ColArgs<T> &, int, cudaStream_t);                                        \
    template void launch_cocg_iter<T>(const ColArgs<T> &, int, cudaStream_t, cudaEvent_t *);                         \
    template void launch_col_prec<T>(const ColArgs<T> &, const C2<T> *, C2<T> *, int, cudaStream_t);          \
    template void launch_colb_init<T>(const KArgs<T> &, int, cudaStream_t);                                     \
    template void launch_colb_vt<T>(const KArgs<T> &, int, int, cudaStream_t);                                  \
    template void launch_colb_jacobi<T>(const KArgs<T> &, int, cudaStream_t);
INST(double)
INST(float)

}  // namespace mt3d

// kernels.cu -- CUDA kernels of the 3D-MT forward/adjoint solve (sm_100a).
//
// All kernels are batched over right-hand sides: blockIdx.y selects the
// right-hand side, blockIdx.x a contiguous chunk of edges (or nodes).  Every
// Krylov scalar lives in device memory (BicgState / PcgState); the last
// block of each right-hand side reduces the block partials in a fixed order
// and updates the scalars, so an iteration needs no host synchronisation and
// is bitwise reproducible.  A right-hand side whose state is not RUNNING is
// skipped by every block.
#include <atomic>

#include "common.cuh"
#include "finalize.cuh"
#include "kernels.h"

namespace mt3d {

std::atomic<long long> g_launch_count{0};
static inline void counted(int n) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

__device__ __forceinline__ int chunk_begin(int chunk) { return blockIdx.x * chunk + threadIdx.x; }

template <typename T> __device__ __forceinline__ T dterm_of(const Geo<T> &g, const EdgeIdx &q, T wmu, T sig)
{
    return wmu * sig * edge_volume(g, q);
}

// ph = v / d, d = V_E*ccdiag (+ GD_ee) + i*dterm (diagonal of A)
template <typename T>
__device__ __forceinline__ C2<T> jacobi(const Geo<T> &g, const EdgeIdx &q, T dterm, C2<T> v, T gdd = T(0))
{
    const T dr = cc_diag(g, q) + gdd, di = dterm;
    const T inv = T(1) / (dr * dr + di * di);
    return mk<T>((v.x * dr + v.y * di) * inv, (v.y * dr - v.x * di) * inv);
}

template <typename T> __device__ __forceinline__ T rhs_wmu(const KArgs<T> &a, int r)
{
    return (T)(a.dsgn * a.ost[r].omega * kMu0);
}

// ---------------------------------------------------------------------------
// grad-div term of the SP2 operator (GradDivSetup2,
// f90/3D_MT/FWD_SP2/modelOperator3D.f90:916-1008):
//   GD x = DFA . G phi,  phi_n = w_n sum_e G_en c_en DFA_e x_e
// with DFA the dual face area of an edge, G the edge-node incidence (-1 at
// the start node, +1 at the end node), c_en = sigma_e at earth nodes and 1 at
// air nodes, w_n = 1/(sigma_n V_n) (earth) or 1/V_n (air), 0 on the boundary.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T dual_face_area(const Geo<T> &g, const EdgeIdx &q)
{
    if (q.c == 0) return g.delY[q.j] * g.delZ[q.k];
    if (q.c == 1) return g.delX[q.i] * g.delZ[q.k];
    return g.delX[q.i] * g.delY[q.j];
}
template <typename T> __device__ __forceinline__ void edge_nodes(const Geo<T> &g, const EdgeIdx &q, int &ns, int &ne)
{
    ns = iN(g, q.i, q.j, q.k);
    ne = q.c == 0 ? iN(g, q.i + 1, q.j, q.k) : q.c == 1 ? iN(g, q.i, q.j + 1, q.k) : iN(g, q.i, q.j, q.k + 1);
}
// (GD x)_e from the node potentials phi of x
template <typename T>
__device__ __forceinline__ C2<T> gd_edge(const Geo<T> &g, const EdgeIdx &q, const C2<T> *__restrict__ phi)
{
    int ns, ne;
    edge_nodes(g, q, ns, ne);
    return cscale(csub(phi[ne], phi[ns]), dual_face_area(g, q));
}
// (GD^T x)_e from the potentials phi of mode 2 below: the transposed term
// scales each node's potential by the edge's own c_en (GD_e'e = DFA_e' sum_n
// G_e'n w_n G_en c_en DFA_e, so GD^T moves c_en to the outer side)
template <typename T>
__device__ __forceinline__ C2<T> gd_edge_t(const KArgs<T> &a, const EdgeIdx &q, T sig_e, const C2<T> *__restrict__ phi)
{
    int ns, ne;
    edge_nodes(a.g, q, ns, ne);
    const T cs = a.gde[ns] ? sig_e : T(1), ce = a.gde[ne] ? sig_e : T(1);
    return cscale(csub(cscale(phi[ne], ce), cscale(phi[ns], cs)), dual_face_area(a.g, q));
}
// GD_ee (diagonal of the grad-div term)
template <typename T>
__device__ __forceinline__ T gd_diag(const KArgs<T> &a, const EdgeIdx &q, T sig_e)
{
    int ns, ne;
    edge_nodes(a.g, q, ns, ne);
    const T dfa = dual_face_area(a.g, q);
    const T cs = a.gde[ns] ? sig_e : T(1), ce = a.gde[ne] ? sig_e : T(1);
    return dfa * dfa * (a.gdw[ns] * cs + a.gdw[ne] * ce);
}

// phi = W G^T (C DFA x) on interior nodes (mode 0: operator; mode 1: the
// source-correction operator V_E GD2 of GradDivSetup2, earth nodes only and
// c = 1; mode 2: the potentials of the transposed operator, W G^T DFA x with
// c = 1, which gd_edge_t completes).  For mode 1 the input is the source
// scaled per right-hand side by 1 / (i ISIGN omega mu0), divided by V_E for
// transposed problems.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gd_phi(KArgs<T> a, const C2<T> *x, C2<T> *phi, int mode)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active && mode != 1) return;
    const Geo<T> &g = a.g;
    const size_t eo = (size_t)r * a.stride, no = (size_t)r * g.nN;
    C2<T> scl = mk<T>(1, 0);
    bool dv = false;
    if (mode == 1) {
        if (!a.ost[r].has_src) return;
        // 1/(i*ISIGN*omega*mu0) = i/(omega*mu0) for ISIGN = -1
        scl = mk<T>(0, (T)(1.0 / (a.ost[r].omega * kMu0)));
        dv = a.ost[r].trans != 0;
    }
    for (int n = blockIdx.x * kThreads + threadIdx.x; n < g.nN; n += gridDim.x * kThreads) {
        const int i = n % (g.nx + 1), t = n / (g.nx + 1), j = t % (g.ny + 1), k = t / (g.ny + 1);
        C2<T> out = mk<T>(0, 0);
        const bool earth = a.gde[n];
        if (i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1 && k >= 1 && k <= g.nz - 1 && (mode != 1 || earth)) {
            const int e[6] = {iX(g, i - 1, j, k), iX(g, i, j, k), iY(g, i, j - 1, k),
                              iY(g, i, j, k), iZ(g, i, j, k - 1), iZ(g, i, j, k)};
            const T dfa[3] = {g.delY[j] * g.delZ[k], g.delX[i] * g.delZ[k], g.delX[i] * g.delY[j]};
            C2<T> acc = mk<T>(0, 0);
#pragma unroll
            for (int q = 0; q < 6; q++) {
                C2<T> v = x[eo + e[q]];
                T c = dfa[q >> 1];
                if (mode == 0 && earth) c *= a.sigma[e[q]];
                if (dv) {
                    const EdgeIdx qq = {q >> 1, (q == 0) ? i - 1 : i, (q == 2) ? j - 1 : j, (q == 4) ? k - 1 : k};
                    c /= edge_volume(g, qq);
                }
                v = cscale(v, c);
                acc = (q & 1) ? csub(acc, v) : cadd(acc, v);  // end node of the first, start of the second
            }
            out = cscale(acc, a.gdw[n]);
            if (mode == 1) out = cmul(out, scl);
        }
        phi[no + n] = out;
    }
}

// b += DFA G phi on interior edges (source correction of the SP2 right-hand side)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gd_add(KArgs<T> a, C2<T> *b, const C2<T> *phi)
{
    const int r = blockIdx.y;
    if (!a.ost[r].has_src) return;
    const Geo<T> &g = a.g;
    const size_t eo = (size_t)r * a.stride, no = (size_t)r * g.nN;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (!edge_interior(g, q)) continue;
        b[eo + e] = cadd(b[eo + e], gd_edge(g, q, phi + no));
    }
}

// ---------------------------------------------------------------------------
// operator apply: y = A x (interior; boundary of y set to zero); neg != 0
// negates.  use_gd = 1 adds the grad-div term GD x from the potentials in
// a.phi (mode 0), use_gd = 2 its transpose GD^T x (potentials of mode 2).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_apply(KArgs<T> a, const C2<T> *x, C2<T> *y, int neg, int use_gd)
{
    const int r = blockIdx.y;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        C2<T> out = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            const T sg = a.sigma[e];
            out = stencil(g, x + off, q, dterm_of(g, q, wmu, sg));
            if (use_gd == 1) out = cadd(out, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            if (use_gd == 2) out = cadd(out, gd_edge_t(a, q, sg, a.phi + (size_t)r * g.nN));
            if (neg) { out.x = -out.x; out.y = -out.y; }
        }
        y[off + e] = out;
    }
}

// ---------------------------------------------------------------------------
// BiCGStab (f90/3D_MT/FWD/solver.f90:346-555) with the diagonal preconditioner
// applied where M1solve/M2solve sit (right preconditioning).
// ---------------------------------------------------------------------------

// start of a call: r = b - A x, rt = r; |b|^2, |r|^2
template <typename T> __global__ void __launch_bounds__(kThreads) kb_init(KArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (!a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    const C2<T> *x = a.x0 + off;
    double v[2] = {0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        C2<T> res = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            C2<T> ax = stencil(g, x, q, dterm_of(g, q, wmu, a.sigma[e]));
            if (a.gd) ax = cadd(ax, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            C2<T> bb = a.b[off + e];
            res = csub(bb, ax);
            v[0] += (double)bb.x * bb.x + (double)bb.y * bb.y;
            v[1] += (double)res.x * res.x + (double)res.y * res.y;
        }
        a.r[off + e] = res;
        a.rt[off + e] = res;
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        fin_init(st, tot, a.rerr + (size_t)r * a.rerr_stride, a.maxit, a.inner ? a.ost[r].tol_inner : a.ost[r].tol);
    }
}

// p = r (first iteration) or p = r + beta (p - omega v); ph = M^-1 p
template <typename T> __global__ void __launch_bounds__(kThreads) kb_p(KArgs<T> a)
{
    const int r = blockIdx.y;
    const BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    const bool first = st.first, reset_rt = st.first && st.pad;
    const C2<T> beta = mk<T>((T)st.beta.re, (T)st.beta.im);
    const C2<T> om = mk<T>((T)st.omega.re, (T)st.omega.im);
    const int end = min((blockIdx.x + 1) * a.chunk, a.len);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        C2<T> rr = a.r[off + e];
        C2<T> p;
        if (first) {
            p = rr;
            if (reset_rt) a.rt[off + e] = rr;
        } else {
            C2<T> pv = csub(a.p[off + e], cmul(om, a.v[off + e]));
            p = cadd(rr, cmul(beta, pv));
        }
        a.p[off + e] = p;
        if (a.pc_ext) continue;
        if (a.jinv) {
            a.ph[off + e] = cmul(a.jinv[off + e], p);
            continue;
        }
        EdgeIdx q = edge_decode(g, e);
        C2<T> ph = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            const T sg = a.sigma[e];
            ph = jacobi(g, q, dterm_of(g, q, wmu, sg), p, a.gd ? gd_diag(a, q, sg) : T(0));
        }
        a.ph[off + e] = ph;
    }
}

// v = A ph; rtv = rt . v ; alpha = rho / rtv
template <typename T> __global__ void __launch_bounds__(kThreads) kb_v(KArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    double v[2] = {0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        C2<T> out = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            out = stencil(g, a.ph + off, q, dterm_of(g, q, wmu, a.sigma[e]));
            if (a.gd) out = cadd(out, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            C2<T> t = a.rt[off + e];
            v[0] += (double)t.x * out.x + (double)t.y * out.y;  // conj(rt)*v
            v[1] += (double)t.x * out.y - (double)t.y * out.x;
        }
        a.v[off + e] = out;
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        fin_v(st, tot);
    }
}

// s = r - alpha v ; sh = M^-1 s
template <typename T> __global__ void __launch_bounds__(kThreads) kb_s(KArgs<T> a)
{
    const int r = blockIdx.y;
    const BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    const C2<T> al = mk<T>((T)st.alpha.re, (T)st.alpha.im);
    const int end = min((blockIdx.x + 1) * a.chunk, a.len);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        C2<T> s = csub(a.r[off + e], cmul(al, a.v[off + e]));
        a.s[off + e] = s;
        if (a.pc_ext) continue;
        if (a.jinv) {
            a.sh[off + e] = cmul(a.jinv[off + e], s);
            continue;
        }
        EdgeIdx q = edge_decode(g, e);
        C2<T> sh = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            const T sg = a.sigma[e];
            sh = jacobi(g, q, dterm_of(g, q, wmu, sg), s, a.gd ? gd_diag(a, q, sg) : T(0));
        }
        a.sh[off + e] = sh;
    }
}

// t = A sh ; ts = t . s, tt = t . t ; omega = ts / tt
template <typename T> __global__ void __launch_bounds__(kThreads) kb_t(KArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const T wmu = rhs_wmu(a, r);
    double v[3] = {0.0, 0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        C2<T> out = mk<T>(0, 0);
        if (edge_interior(g, q)) {
            out = stencil(g, a.sh + off, q, dterm_of(g, q, wmu, a.sigma[e]));
            if (a.gd) out = cadd(out, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            C2<T> s = a.s[off + e];
            v[0] += (double)out.x * s.x + (double)out.y * s.y;  // conj(t)*s
            v[1] += (double)out.x * s.y - (double)out.y * s.x;
            v[2] += (double)out.x * out.x + (double)out.y * out.y;
        }
        a.t[off + e] = out;
    }
    double tot[3];
    if (block_reduce_last<3>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        fin_t(st, tot);
    }
}

// x += alpha ph + omega sh (into the buffer that does not hold the best
// iterate); r = s - omega t; |r|, rho = rt . r ; convergence, best iterate,
// beta for the next iteration
template <typename T> __global__ void __launch_bounds__(kThreads) kb_xr(KArgs<T> a)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<T> &g = a.g;
    const C2<T> al = mk<T>((T)st.alpha.re, (T)st.alpha.im);
    const C2<T> om = mk<T>((T)st.omega.re, (T)st.omega.im);
    const int cur = st.xcur, dst = (st.xcur == st.xbest) ? 1 - st.xcur : st.xcur;
    const C2<T> *xs = (cur == 0 ? a.x0 : a.x1) + off;
    C2<T> *xd = (dst == 0 ? a.x0 : a.x1) + off;
    double v[3] = {0.0, 0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, a.len);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        C2<T> xn = cadd(cadd(xs[e], cmul(al, a.ph[off + e])), cmul(om, a.sh[off + e]));
        xd[e] = xn;
        C2<T> rn = csub(a.s[off + e], cmul(om, a.t[off + e]));
        a.r[off + e] = rn;
        C2<T> t = a.rt[off + e];
        v[0] += (double)rn.x * rn.x + (double)rn.y * rn.y;
        v[1] += (double)t.x * rn.x + (double)t.y * rn.y;  // conj(rt)*r
        v[2] += (double)t.x * rn.y - (double)t.y * rn.x;
    }
    double tot[3];
    if (block_reduce_last<3>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        const double rnorm = sqrt(tot[0]);
        st.iter += 1;
        st.xcur = dst;
        st.first = 0;
        st.pad = 0;
        st.rnorm = rnorm;
        rerr[st.iter - 1] = rnorm / st.bnorm;
        if (!isfinite(rnorm)) { st.status = KS_NAN; return; }
        if (rnorm < st.btol) {
            st.status = KS_CONVERGED;
            st.xbest = dst;
            return;
        }
        if (rnorm < st.rnormin) {
            st.rnormin = rnorm;
            st.xbest = dst;
            st.imin = st.iter;
        }
        if (st.iter >= st.maxit) {
            st.status = KS_MAXIT;
            return;
        }
        if (a.restart > 0 && st.iter % a.restart == 0) {
            // restart towards steepest descent (cuBiCG, f90/3D_MT/FWD_SP2/solver.f90:1545-1573):
            // rt = r, rho = rt . r, p = r, omega = 1
            st.first = 1;
            st.pad = 1;
            st.rho = {tot[0], 0.0};
            st.omega = {1.0, 0.0};
            return;
        }
        cd rho_new = {tot[1], tot[2]};
        st.rho1 = st.rho;
        st.rho = rho_new;
        if (cd_zero(st.rho)) { st.status = KS_BREAKDOWN; return; }
        st.beta = cd_mul(cd_div(st.rho, st.rho1), cd_div(st.alpha, st.omega));
        if (cd_zero(st.beta)) st.status = KS_BREAKDOWN;
    }
}

// end of a call: bring the returned iterate (best iterate unless converged)
// into x0; zero solution for a zero right-hand side
template <typename T> __global__ void __launch_bounds__(kThreads) kb_finish(KArgs<T> a)
{
    const int r = blockIdx.y;
    const BicgState &st = a.st[r];
    if (!a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const int end = min((blockIdx.x + 1) * a.chunk, a.len);
    if (st.xbest == -1) {
        for (int e = chunk_begin(a.chunk); e < end; e += kThreads) a.x0[off + e] = mk<T>(0, 0);
    } else if (st.xbest == 1) {
        for (int e = chunk_begin(a.chunk); e < end; e += kThreads) a.x0[off + e] = a.x1[off + e];
    }
}

// ---------------------------------------------------------------------------
// QMR without look-ahead (f90/3D_MT/FWD/solver.f90:122-343, Barrett et al.'s
// template with the complex changes of the reference), FP64, with the
// diagonal preconditioner as M1 and M2 = I, so Z = WT, YT = Y and
// ZT = D^-H Z.  The vectors: R = r, VT = rt, Y = ph, V = v, WT = s, W = w,
// P = p, Q = q, PT = t, D = d, S = sh, x = x0.  Each right-hand side's scalars
// live in QmrState; the kernels run the reference's statements in order:
//   kq_vw   V = VT / RHO, W = WT / PSI, Y = Y / RHO, DELTA = (Z, Y)
//   kq_pq   P = Y + PDE P, Q = D^-H W + RDE Q
//   kq_pt   PT = A P, EPSIL = (Q, PT), BETA
//   kq_vt   VT = PT - BETA V, Y = D^-1 VT, RHO
//   kq_wt   WT = A^H Q - conj(BETA) W, PSI, THET, GAMM, ETA
//   kq_xr   D, S, x += D, R -= S, ||R||, iteration bookkeeping
// (A^H: the conjugate-transposed operator; in the grad-div formulation its
// grad-div part is GD^T, as Mult_Aii(adjt) forms it.)
// ---------------------------------------------------------------------------
__device__ inline cd cd_sqrt(cd z)
{
    // principal square root from |z|: sqrt((|z| + x)/2) + i sign(y) sqrt((|z| - x)/2)
    const double m = hypot(z.re, z.im);
    const double re = sqrt(0.5 * (m + z.re)), im = sqrt(fmax(0.0, 0.5 * (m - z.re)));
    return {re, z.im < 0.0 ? -im : im};
}
__device__ inline cd cd_add(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
__device__ inline cd cd_neg(cd a) { return {-a.re, -a.im}; }
__device__ inline cd cd_conj(cd a) { return {a.re, -a.im}; }
__device__ inline cd cd_real(double x) { return {x, 0.0}; }
__device__ __forceinline__ double2 cdm(cd c, double2 v) { return make_double2(c.re * v.x - c.im * v.y, c.re * v.y + c.im * v.x); }

// conj(a) b accumulated
template <int N> __device__ __forceinline__ void dotc_acc(double (&u)[N], int o, double2 a, double2 b)
{
    u[o] += a.x * b.x + a.y * b.y;
    u[o + 1] += a.x * b.y - a.y * b.x;
}

// D^-1 v (adj = 0) or D^-H v (adj = 1) at an interior edge
__device__ __forceinline__ double2 qmr_jac(const KArgs<double> &a, const EdgeIdx &q, int r, int e, double2 v, int adj)
{
    const double wmu = rhs_wmu(a, r), sg = a.sigma[e];
    const double dt = dterm_of(a.g, q, wmu, sg);
    return jacobi(a.g, q, adj ? -dt : dt, v, a.gd ? gd_diag(a, q, sg) : 0.0);
}

// R = b - A x, VT = R, Y = D^-1 R, WT = R; ||b||, ||R||, RHO = ||Y||, PSI = ||R||
__global__ void __launch_bounds__(kThreads) kq_init(KArgs<double> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double wmu = rhs_wmu(a, r);
    double u[4] = {0.0, 0.0, 0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        double2 res = make_double2(0.0, 0.0), y = res;
        if (edge_interior(g, q)) {
            double2 ax = stencil(g, a.x0 + off, q, dterm_of(g, q, wmu, a.sigma[e]));
            if (a.gd) ax = cadd(ax, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            const double2 bb = a.b[off + e];
            res = csub(bb, ax);
            y = qmr_jac(a, q, r, e, res, 0);
            u[0] += bb.x * bb.x + bb.y * bb.y;
            u[1] += res.x * res.x + res.y * res.y;
            u[2] += y.x * y.x + y.y * y.y;
        }
        a.r[off + e] = res;
        a.rt[off + e] = res;
        a.s[off + e] = res;
        a.ph[off + e] = y;
    }
    double tot[4];
    if (block_reduce_last<4>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        QmrState &st = a.qst[r];
        st = QmrState{};
        st.maxit = a.maxit;
        st.tol = a.ost[r].tol;
        st.bnorm = sqrt(tot[0]);
        const double rnorm = sqrt(tot[1]);
        st.iter = 1;
        st.rho = cd_real(sqrt(tot[2]));
        st.psi = cd_real(rnorm);
        st.gamm = cd_real(1.0);
        st.eta = cd_real(-1.0);
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        if (!isfinite(st.bnorm)) {
            st.status = KS_NAN;
        } else if (st.bnorm == 0.0) {
            st.status = KS_CONVERGED;
            st.zero = 1;
            rerr[0] = 0.0;
        } else {
            rerr[0] = rnorm / st.bnorm;
            st.status = (rerr[0] > st.tol && st.iter < st.maxit) ? KS_RUNNING : KS_CONVERGED;
            if (st.status == KS_RUNNING && (cd_zero(st.rho) || cd_zero(st.psi))) st.status = KS_BREAKDOWN;
        }
    }
}

__global__ void __launch_bounds__(kThreads) kq_vw(KArgs<double> a)
{
    const int r = blockIdx.y;
    QmrState &st = a.qst[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const cd ri = cd_div(cd_real(1.0), st.rho), pi = cd_div(cd_real(1.0), st.psi);
    double u[2] = {0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        const double2 v = cdm(ri, a.rt[off + e]), w = cdm(pi, a.s[off + e]), y = cdm(ri, a.ph[off + e]);
        a.v[off + e] = v;
        a.w[off + e] = w;
        a.ph[off + e] = y;
        dotc_acc(u, 0, w, y);  // DELTA = (Z, Y), Z = W
    }
    double tot[2];
    if (block_reduce_last<2>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        st.delta = {tot[0], tot[1]};
        if (!cd_finite(st.delta)) { st.status = KS_NAN; return; }
        if (cd_zero(st.delta)) { st.status = KS_BREAKDOWN; return; }
        if (st.iter > 1) {
            const cd de = cd_div(st.delta, st.epsil);
            st.pde = cd_neg(cd_mul(st.psi, de));
            st.rde = cd_neg(cd_mul(st.rho, cd_conj(de)));
        }
    }
}

__global__ void __launch_bounds__(kThreads) kq_pq(KArgs<double> a)
{
    const int r = blockIdx.y;
    const QmrState &st = a.qst[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const bool first = st.iter == 1;
    const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        const EdgeIdx q = edge_decode(a.g, e);
        double2 zt = make_double2(0.0, 0.0);
        if (edge_interior(a.g, q)) zt = qmr_jac(a, q, r, e, a.w[off + e], 1);
        const double2 y = a.ph[off + e];
        if (first) {
            a.p[off + e] = y;
            a.q[off + e] = zt;
        } else {
            a.p[off + e] = cadd(y, cdm(st.pde, a.p[off + e]));
            a.q[off + e] = cadd(zt, cdm(st.rde, a.q[off + e]));
        }
    }
}

// PT = A P (which = 0): EPSIL = (Q, PT), BETA; WT = A^H Q - conj(BETA) W
// (which = 1): PSI and the rotation scalars
__global__ void __launch_bounds__(kThreads) kq_apply(KArgs<double> a, int which)
{
    const int r = blockIdx.y;
    QmrState &st = a.qst[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double wmu = (which ? 1.0 : -1.0) * a.ost[r].omega * kMu0;
    const double2 *x = (which ? a.q : a.p) + off;
    const double2 *phi = a.phi + (size_t)r * g.nN;
    const cd cb = cd_conj(st.beta);
    double u[2] = {0.0, 0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        double2 out = make_double2(0.0, 0.0);
        if (edge_interior(g, q)) {
            const double sg = a.sigma[e];
            out = stencil(g, x, q, dterm_of(g, q, wmu, sg));
            if (a.gd) out = cadd(out, which ? gd_edge_t(a, q, sg, phi) : gd_edge(g, q, phi));
            if (which == 0) {
                dotc_acc(u, 0, a.q[off + e], out);
            } else {
                out = csub(out, cdm(cb, a.w[off + e]));
                u[0] += out.x * out.x + out.y * out.y;
            }
        }
        (which ? a.s : a.t)[off + e] = out;
    }
    double tot[2];
    if (block_reduce_last<2>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        if (which == 0) {
            st.epsil = {tot[0], tot[1]};
            if (!cd_finite(st.epsil)) { st.status = KS_NAN; return; }
            if (cd_zero(st.epsil)) { st.status = KS_BREAKDOWN; return; }
            st.beta = cd_div(st.epsil, st.delta);
            if (cd_zero(st.beta)) st.status = KS_BREAKDOWN;
        } else {
            st.psi = cd_real(sqrt(tot[0]));
            if (st.iter > 1) st.thet1 = st.thet;
            st.thet = cd_div(st.rho, cd_mul(st.gamm, cd_real(hypot(st.beta.re, st.beta.im))));
            st.gamm1 = st.gamm;
            st.gamm = cd_div(cd_real(1.0), cd_sqrt(cd_add(cd_real(1.0), cd_mul(st.thet, st.thet))));
            if (cd_zero(st.gamm) || !cd_finite(st.gamm)) { st.status = cd_zero(st.gamm) ? KS_MAXIT : KS_NAN; return; }
            // ETA = -ETA RHO1 GAMM^2 / (BETA GAMM1^2)
            const cd num = cd_mul(cd_neg(st.eta), cd_mul(st.rho1, cd_mul(st.gamm, st.gamm)));
            st.eta = cd_div(num, cd_mul(st.beta, cd_mul(st.gamm1, st.gamm1)));
            st.tm2 = cd_mul(cd_mul(st.thet1, st.thet1), cd_mul(st.gamm, st.gamm));
        }
    }
}

// VT = PT - BETA V, Y = D^-1 VT, RHO = ||Y||
__global__ void __launch_bounds__(kThreads) kq_vt(KArgs<double> a)
{
    const int r = blockIdx.y;
    QmrState &st = a.qst[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    double u[1] = {0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        const EdgeIdx q = edge_decode(a.g, e);
        const double2 vt = csub(a.t[off + e], cdm(st.beta, a.v[off + e]));
        double2 y = make_double2(0.0, 0.0);
        if (edge_interior(a.g, q)) y = qmr_jac(a, q, r, e, vt, 0);
        a.rt[off + e] = vt;
        a.ph[off + e] = y;
        u[0] += y.x * y.x + y.y * y.y;
    }
    double tot[1];
    if (block_reduce_last<1>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        st.rho1 = st.rho;
        st.rho = cd_real(sqrt(tot[0]));
    }
}

// D = ETA P (+ TM2 D), S = ETA PT (+ TM2 S), x += D, R -= S; ||R||
__global__ void __launch_bounds__(kThreads) kq_xr(KArgs<double> a)
{
    const int r = blockIdx.y;
    QmrState &st = a.qst[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride;
    const bool first = st.iter == 1;
    double u[1] = {0.0};
    const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        double2 d = cdm(st.eta, a.p[off + e]), sv = cdm(st.eta, a.t[off + e]);
        if (!first) {
            d = cadd(d, cdm(st.tm2, a.d[off + e]));
            sv = cadd(sv, cdm(st.tm2, a.sh[off + e]));
        }
        a.d[off + e] = d;
        a.sh[off + e] = sv;
        a.x0[off + e] = cadd(a.x0[off + e], d);
        const double2 rn = csub(a.r[off + e], sv);
        a.r[off + e] = rn;
        u[0] += rn.x * rn.x + rn.y * rn.y;
    }
    double tot[1];
    if (block_reduce_last<1>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        const double rnorm = sqrt(tot[0]);
        st.iter += 1;
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        rerr[st.iter - 1] = rnorm / st.bnorm;
        if (!isfinite(rnorm)) { st.status = KS_NAN; return; }
        if (!(rerr[st.iter - 1] > st.tol)) { st.status = KS_CONVERGED; return; }
        if (st.iter >= st.maxit) { st.status = KS_MAXIT; return; }
        if (cd_zero(st.rho) || cd_zero(st.psi)) st.status = KS_BREAKDOWN;
    }
}

// end of a QMR call: x = 0 for a zero right-hand side; the statuses in the
// BicgState the outer loop reads (iter = the reference's niter; the last
// iterate is the returned one)
__global__ void __launch_bounds__(kThreads) kq_finish(KArgs<double> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    const QmrState &st = a.qst[r];
    const size_t off = (size_t)r * a.stride;
    if (st.zero) {
        const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
        for (int e = chunk_begin(a.chunk); e < end; e += kThreads) a.x0[off + e] = make_double2(0.0, 0.0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        BicgState &b = a.st[r];
        b.status = st.status == KS_CONVERGED ? KS_CONVERGED : st.status == KS_RUNNING ? KS_MAXIT : st.status;
        b.iter = st.iter;
        b.imin = st.iter;
        b.xbest = 0;
        b.xcur = 0;
    }
}

// ---------------------------------------------------------------------------
// divergence correction (SdivCorr, f90/3D_MT/FWD/EMsolve3D.f90:403-492) with
// PCG (f90/3D_MT/FWD/solver.f90:40-118) on DivCgrad and a diagonal
// preconditioner, FP64 throughout.
// ---------------------------------------------------------------------------

// DivC (f90/3D_MT/FWD/modelOperator3D.f90:1817-1925) at interior node (i,j,k)
__device__ __forceinline__ double2 divc_node(const DArgs &a, const double2 *E, int i, int j, int k)
{
    const Geo<double> &g = a.g;
    const double *s = a.sigma;
    const double rx = 1.0 / g.delX[i], ry = 1.0 / g.delY[j], rz = 1.0 / g.delZ[k];
    const int kz = k + 1;  // 1-based iz
    const int ex = iX(g, i, j, k), exm = iX(g, i - 1, j, k);
    const int ey = iY(g, i, j, k), eym = iY(g, i, j - 1, k);
    const int ez = iZ(g, i, j, k), ezm = iZ(g, i, j, k - 1);
    double2 o;
    if (kz <= g.nzAir) {
        const double sa = kSigmaAir;
        o.x = sa * (E[ex].x - E[exm].x) * rx + sa * (E[ey].x - E[eym].x) * ry + sa * (E[ez].x - E[ezm].x) * rz;
        o.y = sa * (E[ex].y - E[exm].y) * rx + sa * (E[ey].y - E[eym].y) * ry + sa * (E[ez].y - E[ezm].y) * rz;
    } else {
        const double szm = (kz == g.nzAir + 1) ? kSigmaAir : s[ezm];
        o.x = (s[ex] * E[ex].x - s[exm] * E[exm].x) * rx + (s[ey] * E[ey].x - s[eym] * E[eym].x) * ry +
              (s[ez] * E[ez].x - szm * E[ezm].x) * rz;
        o.y = (s[ex] * E[ex].y - s[exm] * E[exm].y) * rx + (s[ey] * E[ey].y - s[eym] * E[eym].y) * ry +
              (s[ez] * E[ez].y - szm * E[ezm].y) * rz;
    }
    return o;
}

__device__ __forceinline__ bool node_interior(const Geo<double> &g, int i, int j, int k)
{
    return i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1 && k >= 1 && k <= g.nz - 1;
}
__device__ __forceinline__ void node_decode(const Geo<double> &g, int n, int &i, int &j, int &k)
{
    i = n % (g.nx + 1);
    int t = n / (g.nx + 1);
    j = t % (g.ny + 1);
    k = t / (g.ny + 1);
}

// phiRHS = V_N (DivC(E) - phi0); x = 0; r = b; divJ_before, ||b||, delta = r . M^-1 r
__global__ void __launch_bounds__(kThreads) kd_rhs(DArgs a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].dc_run) return;
    const size_t off = (size_t)r * a.stride;
    const size_t eoff = (size_t)r * a.estride;
    const Geo<double> &g = a.g;
    double v[4] = {0, 0, 0, 0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nN);
    for (int n = chunk_begin(a.chunk); n < end; n += kThreads) {
        int i, j, k;
        node_decode(g, n, i, j, k);
        double2 b = make_double2(0, 0);
        if (node_interior(g, i, j, k)) {
            double2 d = divc_node(a, a.E + eoff, i, j, k);
            if (a.phi0 && a.ost[r].has_src) {
                double2 p0 = a.phi0[off + n];
                d.x -= p0.x;
                d.y -= p0.y;
            }
            v[0] += d.x * d.x + d.y * d.y;
            const double vn = g.delX[i] * g.delY[j] * g.delZ[k];
            b = make_double2(vn * d.x, vn * d.y);
            v[1] += b.x * b.x + b.y * b.y;
            const double rc = 1.0 / a.coef[6 * (size_t)g.nN + n];
            v[2] += (b.x * b.x + b.y * b.y) * rc;  // conj(r)*(r/c): real
        }
        a.pr[off + n] = b;
        a.px[off + n] = make_double2(0, 0);
        a.pp[off + n] = make_double2(0, 0);
    }
    double tot[4];
    if (block_reduce_last<4>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        PcgState &st = a.pst[r];
        OuterState &os = a.ost[r];
        os.divJ[0] = sqrt(tot[0]);
        st.bnorm = sqrt(tot[1]);
        st.rnorm = st.bnorm;
        st.iter = 1;
        st.maxit = a.maxit;
        st.tol = a.tol;
        st.delta = {tot[2], 0.0};
        st.deltaOld = {1.0, 0.0};
        st.beta = {0.0, 0.0};
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        const double rel = st.rnorm / st.bnorm;  // NaN for a zero right-hand side, as in the reference
        rerr[0] = rel;
        st.status = (rel > st.tol && st.iter < st.maxit) ? KS_RUNNING : KS_CONVERGED;
    }
}

// p = M^-1 r + beta p
__global__ void __launch_bounds__(kThreads) kd_p(DArgs a)
{
    const int r = blockIdx.y;
    const PcgState &st = a.pst[r];
    if (!a.ost[r].dc_run || st.status != KS_RUNNING) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double2 be = make_double2(st.beta.re, st.beta.im);
    const int end = min((blockIdx.x + 1) * a.chunk, g.nN);
    for (int n = chunk_begin(a.chunk); n < end; n += kThreads) {
        int i, j, k;
        node_decode(g, n, i, j, k);
        if (!node_interior(g, i, j, k)) continue;
        const double rc = 1.0 / a.coef[6 * (size_t)g.nN + n];
        double2 rr = a.pr[off + n];
        double2 p = a.pp[off + n];
        double2 s = make_double2(rr.x * rc, rr.y * rc);
        a.pp[off + n] = cadd(s, cmul(be, p));
    }
}

// q = DivCgrad p (f90/3D_MT/FWD/modelOperator3D.f90:1760-1810); alpha = delta / (p . q)
__global__ void __launch_bounds__(kThreads) kd_q(DArgs a)
{
    const int r = blockIdx.y;
    PcgState &st = a.pst[r];
    if (!a.ost[r].dc_run || st.status != KS_RUNNING) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double2 *p = a.pp + off;
    double v[2] = {0, 0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nN);
    const int sx = 1, sy = g.nx + 1, sz = (g.nx + 1) * (g.ny + 1);
    for (int n = chunk_begin(a.chunk); n < end; n += kThreads) {
        int i, j, k;
        node_decode(g, n, i, j, k);
        double2 q = make_double2(0, 0);
        if (node_interior(g, i, j, k)) {
            const size_t N = (size_t)g.nN;
            const double c0 = a.coef[n], c1 = a.coef[N + n], c2 = a.coef[2 * N + n], c3 = a.coef[3 * N + n];
            const double c4 = a.coef[4 * N + n], c5 = a.coef[5 * N + n], c6 = a.coef[6 * N + n];
            const double2 pc = p[n];
            q.x = p[n + sx].x * c1 + p[n - sx].x * c0 + p[n + sy].x * c3 + p[n - sy].x * c2 + p[n + sz].x * c5 +
                  p[n - sz].x * c4 + pc.x * c6;
            q.y = p[n + sx].y * c1 + p[n - sx].y * c0 + p[n + sy].y * c3 + p[n - sy].y * c2 + p[n + sz].y * c5 +
                  p[n - sz].y * c4 + pc.y * c6;
            v[0] += pc.x * q.x + pc.y * q.y;  // conj(p)*q
            v[1] += pc.x * q.y - pc.y * q.x;
        }
        a.pq[off + n] = q;
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        cd pq = {tot[0], tot[1]};
        st.alpha = cd_div(st.delta, pq);
        if (!cd_finite(st.alpha)) st.status = KS_NAN;
    }
}

// x += alpha p; r -= alpha q; rerr; delta_new = r . M^-1 r; beta
__global__ void __launch_bounds__(kThreads) kd_xr(DArgs a)
{
    const int r = blockIdx.y;
    PcgState &st = a.pst[r];
    if (!a.ost[r].dc_run || st.status != KS_RUNNING) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double2 al = make_double2(st.alpha.re, st.alpha.im);
    double v[2] = {0, 0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nN);
    for (int n = chunk_begin(a.chunk); n < end; n += kThreads) {
        int i, j, k;
        node_decode(g, n, i, j, k);
        if (!node_interior(g, i, j, k)) continue;
        a.px[off + n] = cadd(a.px[off + n], cmul(al, a.pp[off + n]));
        double2 rr = csub(a.pr[off + n], cmul(al, a.pq[off + n]));
        a.pr[off + n] = rr;
        const double m2 = rr.x * rr.x + rr.y * rr.y;
        v[0] += m2;
        v[1] += m2 / a.coef[6 * (size_t)g.nN + n];
    }
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        st.iter += 1;
        st.rnorm = sqrt(tot[0]);
        const double rel = st.rnorm / st.bnorm;
        rerr[st.iter - 1] = rel;
        st.deltaOld = st.delta;
        st.delta = {tot[1], 0.0};
        st.beta = cd_div(st.delta, st.deltaOld);
        if (!isfinite(rel)) st.status = KS_NAN;
        else if (!(rel > st.tol && st.iter < st.maxit)) st.status = KS_CONVERGED;
    }
}

// E -= Grad(phi) on interior edges (Grad, f90/FIELDS/FiniteDiff3D/sg_diff_oper.f90:98-200)
__global__ void __launch_bounds__(kThreads) kd_grad(DArgs a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].dc_run) return;
    const size_t off = (size_t)r * a.stride;
    const size_t eoff = (size_t)r * a.estride;
    const Geo<double> &g = a.g;
    const double2 *phi = a.px + off;
    double2 *E = a.E + eoff;
    const int end = min((blockIdx.x + 1) * a.echunk, g.nE);
    for (int e = chunk_begin(a.echunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (!edge_interior(g, q)) continue;
        double2 gr;
        if (q.c == 0) {
            const double2 a1 = phi[iN(g, q.i + 1, q.j, q.k)], a0 = phi[iN(g, q.i, q.j, q.k)];
            gr = make_double2((a1.x - a0.x) / g.dx[q.i], (a1.y - a0.y) / g.dx[q.i]);
        } else if (q.c == 1) {
            const double2 a1 = phi[iN(g, q.i, q.j + 1, q.k)], a0 = phi[iN(g, q.i, q.j, q.k)];
            gr = make_double2((a1.x - a0.x) / g.dy[q.j], (a1.y - a0.y) / g.dy[q.j]);
        } else {
            const double2 a1 = phi[iN(g, q.i, q.j, q.k + 1)], a0 = phi[iN(g, q.i, q.j, q.k)];
            gr = make_double2((a1.x - a0.x) / g.dz[q.k], (a1.y - a0.y) / g.dz[q.k]);
        }
        E[e] = csub(E[e], gr);
    }
}

// divJ after the correction: ||DivC(E) - phi0||
__global__ void __launch_bounds__(kThreads) kd_divj(DArgs a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].dc_run) return;
    const size_t off = (size_t)r * a.stride;
    const size_t eoff = (size_t)r * a.estride;
    const Geo<double> &g = a.g;
    double v[1] = {0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nN);
    for (int n = chunk_begin(a.chunk); n < end; n += kThreads) {
        int i, j, k;
        node_decode(g, n, i, j, k);
        if (!node_interior(g, i, j, k)) continue;
        double2 d = divc_node(a, a.E + eoff, i, j, k);
        if (a.phi0 && a.ost[r].has_src) {
            d.x -= a.phi0[off + n].x;
            d.y -= a.phi0[off + n].y;
        }
        v[0] += d.x * d.x + d.y * d.y;
    }
    double tot[1];
    if (block_reduce_last<1>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        a.ost[r].divJ[1] = sqrt(tot[0]);
    }
}

// ---------------------------------------------------------------------------
// right-hand sides, post-processing, precision glue
// ---------------------------------------------------------------------------

// keep only the boundary entries of v (interior set to zero)
__global__ void __launch_bounds__(kThreads) k_keep_boundary(Geo<double> g, double2 *v, size_t stride)
{
    const size_t off = (size_t)blockIdx.y * stride;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (edge_interior(g, q)) v[off + e] = make_double2(0, 0);
    }
}

// keep only the interior entries of v (boundary set to zero)
__global__ void __launch_bounds__(kThreads) k_keep_interior(Geo<double> g, double2 *v, size_t stride)
{
    const size_t off = (size_t)blockIdx.y * stride;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (!edge_interior(g, q)) v[off + e] = make_double2(0, 0);
    }
}

// b += w * src on interior edges: w = V_E for a forward source, 1 for the
// (already V_E-weighted) adjoint source of the transposed problem
// (f90/3D_MT/FWD/EMsolve3D.f90:166-183, 202-218)
__global__ void __launch_bounds__(kThreads) k_add_src(Geo<double> g, double2 *b, const double2 *src, size_t stride,
                                                       const OuterState *ost)
{
    const int r = blockIdx.y;
    if (!ost[r].has_src) return;
    const bool tr = ost[r].trans != 0;
    const size_t off = (size_t)r * stride;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (!edge_interior(g, q)) continue;
        const double w = tr ? 1.0 : edge_volume(g, q);
        b[off + e] = cadd(b[off + e], make_double2(w * src[off + e].x, w * src[off + e].y));
    }
}

// phi0 = Div(w * src) / (i ISIGN mu0 omega) on interior nodes, w = 1/V_E when
// divide_ve (transposed problem) else 1 (Div, sg_diff_oper.f90:26-93)
__global__ void __launch_bounds__(kThreads) k_phi0(Geo<double> g, const double2 *src, size_t estride, double2 *phi0,
                                                    size_t nstride, const OuterState *ost)
{
    const int r = blockIdx.y;
    const size_t off = (size_t)r * nstride, eoff = (size_t)r * estride;
    const OuterState &os = ost[r];
    if (!os.has_src) return;
    const bool dv = os.trans != 0;
    // 1 / (i * ISIGN * mu0 * omega) = i / (mu0 * omega) for ISIGN = -1
    const double inv = 1.0 / (kMu0 * os.omega);
    for (int n = blockIdx.x * kThreads + threadIdx.x; n < g.nN; n += gridDim.x * kThreads) {
        int i = n % (g.nx + 1), t = n / (g.nx + 1), j = t % (g.ny + 1), k = t / (g.ny + 1);
        double2 out = make_double2(0, 0);
        if (i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1 && k >= 1 && k <= g.nz - 1) {
            auto val = [&](int e, const EdgeIdx &q) {
                double2 s = src[eoff + e];
                if (!edge_interior(g, q)) return make_double2(0, 0);
                if (dv) {
                    double ve = edge_volume(g, q);
                    s.x /= ve;
                    s.y /= ve;
                }
                return s;
            };
            EdgeIdx q;
            q = {0, i, j, k}; double2 ex = val(iX(g, i, j, k), q);
            q = {0, i - 1, j, k}; double2 exm = val(iX(g, i - 1, j, k), q);
            q = {1, i, j, k}; double2 ey = val(iY(g, i, j, k), q);
            q = {1, i, j - 1, k}; double2 eym = val(iY(g, i, j - 1, k), q);
            q = {2, i, j, k}; double2 ez = val(iZ(g, i, j, k), q);
            q = {2, i, j, k - 1}; double2 ezm = val(iZ(g, i, j, k - 1), q);
            double2 d;
            d.x = (ex.x - exm.x) / g.delX[i] + (ey.x - eym.x) / g.delY[j] + (ez.x - ezm.x) / g.delZ[k];
            d.y = (ex.y - exm.y) / g.delX[i] + (ey.y - eym.y) / g.delY[j] + (ez.y - ezm.y) / g.delZ[k];
            // d * i * inv
            out = make_double2(-d.y * inv, d.x * inv);
        }
        phi0[off + n] = out;
    }
}

// true FP64 residual of the mixed path: r64 = b - A X; |r64|^2 -> relres,
// convergence test and the scale of the FP32 right-hand side
__global__ void __launch_bounds__(kThreads) km_res64(KArgs<double> a, double tol_unused)
{
    const int r = blockIdx.y;
    OuterState &os = a.ost[r];
    if (!os.active) return;
    const size_t off = (size_t)r * a.stride;
    const Geo<double> &g = a.g;
    const double wmu = rhs_wmu(a, r);
    double v[1] = {0};
    const int end = min((blockIdx.x + 1) * a.chunk, g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        EdgeIdx q = edge_decode(g, e);
        double2 res = make_double2(0, 0);
        if (edge_interior(g, q)) {
            double2 ax = stencil(g, a.x0 + off, q, dterm_of(g, q, wmu, a.sigma[e]));
            if (a.gd) ax = cadd(ax, gd_edge(g, q, a.phi + (size_t)r * g.nN));
            res = csub(a.b[off + e], ax);
            v[0] += res.x * res.x + res.y * res.y;
        }
        a.r[off + e] = res;
    }
    double tot[1];
    if (block_reduce_last<1>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        fin_res64(os, tot);
    }
}

// FP32 right-hand side of the correction equation: b32 = r64 * scale, x32 = 0
__global__ void __launch_bounds__(kThreads) km_cast(const OuterState *ost, int nE, size_t stride, const double2 *r64,
                                                     float2 *b32, float2 *x32)
{
    const int r = blockIdx.y;
    if (!ost[r].active) return;
    const size_t off = (size_t)r * stride;
    const double sc = ost[r].scale;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < nE; e += gridDim.x * kThreads) {
        double2 v = r64[off + e];
        b32[off + e] = make_float2((float)(v.x * sc), (float)(v.y * sc));
        x32[off + e] = make_float2(0.f, 0.f);
    }
}

// X += d32 / scale
__global__ void __launch_bounds__(kThreads) km_update(const OuterState *ost, int nE, size_t stride, const float2 *d32,
                                                       double2 *X)
{
    const int r = blockIdx.y;
    if (!ost[r].active) return;
    const size_t off = (size_t)r * stride;
    const double inv = ost[r].scale > 0.0 ? 1.0 / ost[r].scale : 0.0;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < nE; e += gridDim.x * kThreads) {
        float2 d = d32[off + e];
        double2 x = X[off + e];
        X[off + e] = make_double2(x.x + (double)d.x * inv, x.y + (double)d.y * inv);
    }
}

// b32 = r64 * scale and x32 = 0 on the padded layout (the padding keeps the
// zeros it was allocated with)
__global__ void __launch_bounds__(kThreads) km_cast_p(Geo<double> g, const OuterState *ost, size_t stride64,
                                                      const double2 *r64, PadLayout pl, float2 *b32, float2 *x32)
{
    const int r = blockIdx.y;
    if (!ost[r].active) return;
    const size_t off = (size_t)r * stride64, offp = (size_t)r * pl.len();
    const double sc = ost[r].scale;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        const EdgeIdx q = edge_decode(g, e);
        const int pe = pl.idx(q.c, q.i, q.j, q.k);
        const double2 v = r64[off + e];
        b32[offp + pe] = make_float2((float)(v.x * sc), (float)(v.y * sc));
        x32[offp + pe] = make_float2(0.f, 0.f);
    }
}

// X += d32 / scale, d32 on the padded layout
__global__ void __launch_bounds__(kThreads) km_update_p(Geo<double> g, const OuterState *ost, size_t stride64,
                                                        PadLayout pl, const float2 *d32, double2 *X)
{
    const int r = blockIdx.y;
    if (!ost[r].active) return;
    const size_t off = (size_t)r * stride64, offp = (size_t)r * pl.len();
    const double inv = ost[r].scale > 0.0 ? 1.0 / ost[r].scale : 0.0;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        const EdgeIdx q = edge_decode(g, e);
        const float2 d = d32[offp + pl.idx(q.c, q.i, q.j, q.k)];
        const double2 x = X[off + e];
        X[off + e] = make_double2(x.x + (double)d.x * inv, x.y + (double)d.y * inv);
    }
}

// an edge array (sigma) and a node array (signed weights) in FP32 on the
// padded layout; the destinations are zeroed first by the caller
__global__ void __launch_bounds__(kThreads) k_to_padded(Geo<double> g, const double *src, PadLayout pl, float *dst)
{
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        const EdgeIdx q = edge_decode(g, e);
        dst[pl.idx(q.c, q.i, q.j, q.k)] = (float)src[e];
    }
}
__global__ void __launch_bounds__(kThreads) k_nodes_to_padded(Geo<double> g, const double *src, PadLayout pl,
                                                              float *dst)
{
    for (int n = blockIdx.x * kThreads + threadIdx.x; n < g.nN; n += gridDim.x * kThreads) {
        const int i = n % (g.nx + 1), t = n / (g.nx + 1), j = t % (g.ny + 1), k = t / (g.ny + 1);
        dst[pl.idx(0, i, j, k)] = (float)src[n];
    }
}

// ||b||^2 per right-hand side (FP64 interior system)
__global__ void __launch_bounds__(kThreads) k_norm_b(KArgs<double> a)
{
    const int r = blockIdx.y;
    const size_t off = (size_t)r * a.stride;
    double v[1] = {0};
    const int end = min((blockIdx.x + 1) * a.chunk, a.g.nE);
    for (int e = chunk_begin(a.chunk); e < end; e += kThreads) {
        double2 b = a.b[off + e];
        v[0] += b.x * b.x + b.y * b.y;
    }
    double tot[1];
    if (block_reduce_last<1>(v, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0)
        a.ost[r].bnorm64 = sqrt(tot[0]);
}

// Post-processing of FWDsolve3D (f90/3D_MT/FWD/EMsolve3D.f90:356-385):
// forward: boundary = bc (or 0); transposed: e = V_E e and boundary =
// bc - AdjtBC(e) (or -AdjtBC(e)), AdjtBC (f90/3D_MT/FWD/modelOperator3D.f90:
// 920-1057) with the face precedence of copy_bcvector.  Step 1 scales the
// interior of transposed solutions by V_E.
__global__ void __launch_bounds__(kThreads) k_post_scale(Geo<double> g, double2 *E, size_t stride, const OuterState *ost)
{
    const int r = blockIdx.y;
    if (!ost[r].trans) return;
    const size_t off = (size_t)r * stride;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (!edge_interior(g, q)) continue;
        E[off + e] = cscale(E[off + e], edge_volume(g, q));
    }
}

__device__ double2 adjt_bc_value(const Geo<double> &g, const double2 *E, const EdgeIdx &q)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz, i = q.i, j = q.j, k = q.k;
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz, *dX = g.delX, *dY = g.delY, *dZ = g.delZ;
    double2 z = make_double2(0, 0);
    // a*E[iu] + b*E[iv] + c*E[iw]; a zero coefficient skips its load, so only
    // interior entries are read while the boundary entries are rewritten
    auto lin3i = [&](double a, int iu, double b, int iv, double c, int iw) {
        double2 u = a != 0.0 ? E[iu] : z, v = b != 0.0 ? E[iv] : z, w = E[iw];
        return make_double2(a * u.x + b * v.x + c * w.x, a * u.y + b * v.y + c * w.y);
    };
    if (q.c == 0) {  // Ex
        if (k == 0 || k == nz) {
            if (j == 0 || j == ny) return z;
            if (k == 0) {
                double a1 = (i >= 1 && i <= nx - 1) ? 1.0 / (dX[i] * dz[0]) : 0.0;
                double a2 = (i <= nx - 2) ? 1.0 / (dX[i + 1] * dz[0]) : 0.0;
                return lin3i(-a1, iZ(g, i, j, 0), a2, iZ(g, i + 1, j, 0), -1.0 / (dZ[1] * dz[0]), iX(g, i, j, 1));
            } else {
                double a1 = (i >= 1 && i <= nx - 1) ? 1.0 / (dX[i] * dz[nz - 1]) : 0.0;
                double a2 = (i <= nx - 2) ? 1.0 / (dX[i + 1] * dz[nz - 1]) : 0.0;
                return lin3i(a1, iZ(g, i, j, nz - 1), -a2, iZ(g, i + 1, j, nz - 1), -1.0 / (dZ[nz - 1] * dz[nz - 1]),
                            iX(g, i, j, nz - 1));
            }
        }
        if (j == 0) {
            double a1 = (i >= 1 && i <= nx - 1) ? 1.0 / (dX[i] * dy[0]) : 0.0;
            double a2 = (i <= nx - 2) ? 1.0 / (dX[i + 1] * dy[0]) : 0.0;
            return lin3i(-a1, iY(g, i, 0, k), a2, iY(g, i + 1, 0, k), -1.0 / (dY[1] * dy[0]), iX(g, i, 1, k));
        } else {
            double a1 = (i >= 1 && i <= nx - 1) ? 1.0 / (dX[i] * dy[ny - 1]) : 0.0;
            double a2 = (i <= nx - 2) ? 1.0 / (dX[i + 1] * dy[ny - 1]) : 0.0;
            return lin3i(a1, iY(g, i, ny - 1, k), -a2, iY(g, i + 1, ny - 1, k), -1.0 / (dY[ny - 1] * dy[ny - 1]),
                        iX(g, i, ny - 1, k));
        }
    } else if (q.c == 1) {  // Ey
        if (k == 0 || k == nz) {
            if (i == 0 || i == nx) return z;
            if (k == 0) {
                double a1 = (j >= 1 && j <= ny - 1) ? 1.0 / (dY[j] * dz[0]) : 0.0;
                double a2 = (j <= ny - 2) ? 1.0 / (dY[j + 1] * dz[0]) : 0.0;
                return lin3i(-a1, iZ(g, i, j, 0), a2, iZ(g, i, j + 1, 0), -1.0 / (dZ[1] * dz[0]), iY(g, i, j, 1));
            } else {
                double a1 = (j >= 1 && j <= ny - 1) ? 1.0 / (dY[j] * dz[nz - 1]) : 0.0;
                double a2 = (j <= ny - 2) ? 1.0 / (dY[j + 1] * dz[nz - 1]) : 0.0;
                return lin3i(a1, iZ(g, i, j, nz - 1), -a2, iZ(g, i, j + 1, nz - 1), -1.0 / (dZ[nz - 1] * dz[nz - 1]),
                            iY(g, i, j, nz - 1));
            }
        }
        if (i == 0) {
            double a1 = (j >= 1 && j <= ny - 1) ? 1.0 / (dY[j] * dx[0]) : 0.0;
            double a2 = (j <= ny - 2) ? 1.0 / (dY[j + 1] * dx[0]) : 0.0;
            return lin3i(-a1, iX(g, 0, j, k), a2, iX(g, 0, j + 1, k), -1.0 / (dX[1] * dx[0]), iY(g, 1, j, k));
        } else {
            double a1 = (j >= 1 && j <= ny - 1) ? 1.0 / (dY[j] * dx[nx - 1]) : 0.0;
            double a2 = (j <= ny - 2) ? 1.0 / (dY[j + 1] * dx[nx - 1]) : 0.0;
            return lin3i(a1, iX(g, nx - 1, j, k), -a2, iX(g, nx - 1, j + 1, k), -1.0 / (dX[nx - 1] * dx[nx - 1]),
                        iY(g, nx - 1, j, k));
        }
    } else {  // Ez
        if (i == 0 || i == nx) {
            if (j == 0 || j == ny) return z;
            if (i == 0) {
                double a1 = (k >= 1 && k <= nz - 1) ? 1.0 / (dZ[k] * dx[0]) : 0.0;
                double a2 = (k <= nz - 2) ? 1.0 / (dZ[k + 1] * dx[0]) : 0.0;
                return lin3i(-a1, iX(g, 0, j, k), a2, iX(g, 0, j, k + 1), -1.0 / (dX[1] * dx[0]), iZ(g, 1, j, k));
            } else {
                double a1 = (k >= 1 && k <= nz - 1) ? 1.0 / (dZ[k] * dx[nx - 1]) : 0.0;
                double a2 = (k <= nz - 2) ? 1.0 / (dZ[k + 1] * dx[nx - 1]) : 0.0;
                return lin3i(a1, iX(g, nx - 1, j, k), -a2, iX(g, nx - 1, j, k + 1), -1.0 / (dX[nx - 1] * dx[nx - 1]),
                            iZ(g, nx - 1, j, k));
            }
        }
        if (j == 0) {
            double a1 = (k >= 1 && k <= nz - 1) ? 1.0 / (dZ[k] * dy[0]) : 0.0;
            double a2 = (k <= nz - 2) ? 1.0 / (dZ[k + 1] * dy[0]) : 0.0;
            return lin3i(-a1, iY(g, i, 0, k), a2, iY(g, i, 0, k + 1), -1.0 / (dY[1] * dy[0]), iZ(g, i, 1, k));
        } else {
            double a1 = (k >= 1 && k <= nz - 1) ? 1.0 / (dZ[k] * dy[ny - 1]) : 0.0;
            double a2 = (k <= nz - 2) ? 1.0 / (dZ[k + 1] * dy[ny - 1]) : 0.0;
            return lin3i(a1, iY(g, i, ny - 1, k), -a2, iY(g, i, ny - 1, k + 1), -1.0 / (dY[ny - 1] * dy[ny - 1]),
                        iZ(g, i, ny - 1, k));
        }
    }
}

// boundary entries of the returned field (bc is the uploaded boundary data,
// may be null; has_bc per right-hand side)
__global__ void __launch_bounds__(kThreads) k_post_boundary(Geo<double> g, double2 *E, const double2 *bc, size_t stride,
                                                             const OuterState *ost)
{
    const int r = blockIdx.y;
    const size_t off = (size_t)r * stride;
    const bool tr = ost[r].trans != 0;
    const bool hb = bc != nullptr && ost[r].has_bc;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        EdgeIdx q = edge_decode(g, e);
        if (edge_interior(g, q)) continue;
        double2 v = hb ? bc[off + e] : make_double2(0, 0);
        if (tr) v = csub(v, adjt_bc_value(g, E + off, q));
        E[off + e] = v;
    }
}

// PmultT + dEdgeToModelParam (f90/3D_MT/SolverSens.f90:63-116,
// f90/3D_MT/modelParam/ModelMap.inc:302-374), gathered per earth cell: each
// cell sums Re(i*mu0*omega*sum_pol e0*eadj)/V_E_ghost over its 12 edges with
// the Edge2Cell weights (1/4, 1/2 or 1 by the number of cells sharing the
// edge), then multiplies by V_C and exp(m0).
__device__ __forceinline__ int edge_ncells(const Geo<double> &g, int c, int i, int j, int k)
{
    int a = 2, b = 2;
    if (c == 0) { a = (j == 0 || j == g.ny) ? 1 : 2; b = (k == 0 || k == g.nz) ? 1 : 2; }
    if (c == 1) { a = (i == 0 || i == g.nx) ? 1 : 2; b = (k == 0 || k == g.nz) ? 1 : 2; }
    if (c == 2) { a = (i == 0 || i == g.nx) ? 1 : 2; b = (j == 0 || j == g.ny) ? 1 : 2; }
    return a * b;
}
__device__ __forceinline__ double cellvol(const Geo<double> &g, int i, int j, int k)
{
    return g.dx[i] * g.dy[j] * g.dz[k];
}
// V_E_ghost = sum of the adjacent cell volumes / their number (Cell2Edge of V_C)
__device__ double edge_vghost(const Geo<double> &g, int c, int i, int j, int k)
{
    double s = 0.0;
    int n = 0;
    for (int a = -1; a <= 0; a++)
        for (int b = -1; b <= 0; b++) {
            int ci = i, cj = j, ck = k;
            if (c == 0) { cj = j + a; ck = k + b; }
            if (c == 1) { ci = i + a; ck = k + b; }
            if (c == 2) { ci = i + a; cj = j + b; }
            if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny || ck < 0 || ck >= g.nz) continue;
            s += cellvol(g, ci, cj, ck);
            n++;
        }
    return s / n;
}

__global__ void __launch_bounds__(kThreads) k_pmult_t(Geo<double> g, int npol, const double2 *e0, const double2 *ea,
                                                       double omega, const double *m0, double *dm)
{
    const int nEarth = g.nx * g.ny * (g.nz - g.nzAir);
    const double w = kMu0 * omega;  // -ISIGN*mu0*omega with ISIGN = -1: factor i*w
    for (int c = blockIdx.x * kThreads + threadIdx.x; c < nEarth; c += gridDim.x * kThreads) {
        const int i = c % g.nx, t = c / g.nx, j = t % g.ny, k = t / g.ny + g.nzAir;
        double acc = 0.0;
        auto edge = [&](int comp, int ei, int ej, int ek, int idx) {
            double re = 0.0;
            for (int p = 0; p < npol; p++) {
                double2 a = e0[(size_t)p * g.nE + idx], b = ea[(size_t)p * g.nE + idx];
                // Re(i*w*a*b) = -w * Im(a*b)
                re += -w * (a.x * b.y + a.y * b.x);
            }
            return re / edge_vghost(g, comp, ei, ej, ek) / edge_ncells(g, comp, ei, ej, ek);
        };
        for (int b = 0; b <= 1; b++)
            for (int a = 0; a <= 1; a++) {
                acc += edge(0, i, j + a, k + b, iX(g, i, j + a, k + b));
                acc += edge(1, i + a, j, k + b, iY(g, i + a, j, k + b));
                acc += edge(2, i + a, j + b, k, iZ(g, i + a, j + b, k));
            }
        dm[c] = (acc * cellvol(g, i, j, k)) * exp(m0[c]);
    }
}

// flags[r] |= 1 when vector r has a non-zero (or NaN) entry
__global__ void __launch_bounds__(kThreads) k_nonzero(const double2 *v, size_t stride, int n, int *flags)
{
    const int r = blockIdx.y;
    bool nz = false;
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < n; e += gridDim.x * kThreads) {
        const double2 a = v[(size_t)r * stride + e];
        nz = nz || (a.x != 0.0) || (a.y != 0.0);
    }
    if (__syncthreads_or(nz) && threadIdx.x == 0) atomicOr(&flags[r], 1);
}

// ---------------------------------------------------------------------------
// gather / scatter between interior vectors (EDGEi order) and full vectors
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_scatter_interior(int nEi, const int *edgei, const double2 *vi, double2 *vf)
{
    for (int n = blockIdx.x * kThreads + threadIdx.x; n < nEi; n += gridDim.x * kThreads) vf[edgei[n]] = vi[n];
}
__global__ void __launch_bounds__(kThreads) k_gather_interior(int nEi, const int *edgei, const double2 *vf, double2 *vi)
{
    for (int n = blockIdx.x * kThreads + threadIdx.x; n < nEi; n += gridDim.x * kThreads) vi[n] = vf[edgei[n]];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t preload_apply_kernels()
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_apply<double>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_gd_phi<double>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_scatter_interior);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_gather_interior);
    return e;
}
template <typename T>
void launch_apply(const KArgs<T> &a, const C2<T> *x, C2<T> *y, int neg, int nrhs, cudaStream_t s, int use_gd)
{
    counted(1);
    if (use_gd) launch_gd_phi(a, x, a.phi, use_gd == 2 ? 2 : 0, nrhs, s);
    k_apply<T><<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a, x, y, neg, use_gd);
}
template <typename T> void launch_gd_phi(const KArgs<T> &a, const C2<T> *x, C2<T> *phi, int mode, int nrhs, cudaStream_t s)
{
    counted(1);
    const int gn = (int)std::min<long>((a.g.nN + kThreads - 1) / kThreads, 148L * 16);
    k_gd_phi<T><<<dim3(gn, nrhs), kThreads, 0, s>>>(a, x, phi, mode);
}
template <typename T> void launch_gd_add(const KArgs<T> &a, C2<T> *b, const C2<T> *phi, int nrhs, cudaStream_t s)
{
    counted(1);
    const int ge = (int)std::min<long>((a.g.nE + kThreads - 1) / kThreads, 148L * 16);
    k_gd_add<T><<<dim3(ge, nrhs), kThreads, 0, s>>>(a, b, phi);
}
template void launch_gd_phi<double>(const KArgs<double> &, const double2 *, double2 *, int, int, cudaStream_t);
template void launch_gd_phi<float>(const KArgs<float> &, const float2 *, float2 *, int, int, cudaStream_t);
template void launch_gd_add<double>(const KArgs<double> &, double2 *, const double2 *, int, cudaStream_t);
template <typename T> void launch_bicg_init(const KArgs<T> &a, int nrhs, cudaStream_t s)
{
    if (a.jinv) launch_colb_jacobi(a, nrhs, s);
    if (a.colstencil == 3) {
        if constexpr (sizeof(T) == 4) launch_tma_init(a, a.tma, nrhs, s);
        return;
    }
    if (a.colstencil == 2) {
        launch_stage_init(a, nrhs, s);
        return;
    }
    if (a.gd) launch_gd_phi(a, a.x0, a.phi, 0, nrhs, s);
    if (a.colstencil) {
        launch_colb_init(a, nrhs, s);
    } else {
        counted(1);
        kb_init<T><<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
    }
}
template <typename T>
void launch_bicg_iter(const KArgs<T> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev, const ColArgs<T> *pc)
{
    counted(a.colstencil ? 3 : 5);
    dim3 grid(a.nblk, nrhs);
    const bool staged = a.colstencil >= 2;
    kb_p<T><<<grid, kThreads, 0, s>>>(a);
    if (pc) launch_col_prec(*pc, a.p, a.ph, nrhs, s);
    if (a.gd && !staged) launch_gd_phi(a, a.ph, a.phi, 0, nrhs, s);
    if (ev) cudaEventRecord(ev[0], s);
    if (a.colstencil == 3) {
        if constexpr (sizeof(T) == 4) launch_tma_vt(a, a.tma, 0, nrhs, s);
    } else if (staged) launch_stage_vt(a, 0, nrhs, s);
    else if (a.colstencil) launch_colb_vt(a, 0, nrhs, s);
    else kb_v<T><<<grid, kThreads, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[1], s);
    kb_s<T><<<grid, kThreads, 0, s>>>(a);
    if (pc) launch_col_prec(*pc, a.s, a.sh, nrhs, s);
    if (a.gd && !staged) launch_gd_phi(a, a.sh, a.phi, 0, nrhs, s);
    if (ev) cudaEventRecord(ev[2], s);
    if (a.colstencil == 3) {
        if constexpr (sizeof(T) == 4) launch_tma_vt(a, a.tma, 1, nrhs, s);
    } else if (staged) launch_stage_vt(a, 1, nrhs, s);
    else if (a.colstencil) launch_colb_vt(a, 1, nrhs, s);
    else kb_t<T><<<grid, kThreads, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[3], s);
    kb_xr<T><<<grid, kThreads, 0, s>>>(a);
}
template <typename T> void launch_bicg_finish(const KArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kb_finish<T><<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}
void launch_qmr_init(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    if (a.gd) launch_gd_phi(a, a.x0, a.phi, 0, nrhs, s);
    counted(1);
    kq_init<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}
void launch_qmr_iter(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    const dim3 grid(a.nblk, nrhs);
    counted(6);
    kq_vw<<<grid, kThreads, 0, s>>>(a);
    kq_pq<<<grid, kThreads, 0, s>>>(a);
    if (a.gd) launch_gd_phi(a, a.p, a.phi, 0, nrhs, s);
    kq_apply<<<grid, kThreads, 0, s>>>(a, 0);
    kq_vt<<<grid, kThreads, 0, s>>>(a);
    if (a.gd) launch_gd_phi(a, a.q, a.phi, 2, nrhs, s);
    kq_apply<<<grid, kThreads, 0, s>>>(a, 1);
    kq_xr<<<grid, kThreads, 0, s>>>(a);
}
void launch_qmr_finish(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kq_finish<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}

template void launch_apply<double>(const KArgs<double> &, const double2 *, double2 *, int, int, cudaStream_t, int);
template void launch_apply<float>(const KArgs<float> &, const float2 *, float2 *, int, int, cudaStream_t, int);
template void launch_bicg_init<double>(const KArgs<double> &, int, cudaStream_t);
template void launch_bicg_init<float>(const KArgs<float> &, int, cudaStream_t);
template void launch_bicg_iter<double>(const KArgs<double> &, int, cudaStream_t, cudaEvent_t *, const ColArgs<double> *);
template void launch_bicg_iter<float>(const KArgs<float> &, int, cudaStream_t, cudaEvent_t *, const ColArgs<float> *);
template void launch_bicg_finish<double>(const KArgs<double> &, int, cudaStream_t);
template void launch_bicg_finish<float>(const KArgs<float> &, int, cudaStream_t);

void launch_norm_b(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    k_norm_b<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}
void launch_res64(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    if (a.colstencil == 2) {
        launch_stage_res64(a, nrhs, s);
        return;
    }
    if (a.gd) launch_gd_phi(a, a.x0, a.phi, 0, nrhs, s);
    if (a.colstencil) {
        launch_colb_res64(a, nrhs, s);
    } else {
        counted(1);
        km_res64<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a, 0.0);
    }
}
static int grid_for(long n) { return (int)std::min<long>((n + kThreads - 1) / kThreads, 148L * 16); }
void launch_cast(const OuterState *ost, int nE, size_t stride, const double2 *r64, float2 *b32, float2 *x32, int nrhs,
                 cudaStream_t s)
{
    counted(1);
    km_cast<<<dim3(grid_for(nE), nrhs), kThreads, 0, s>>>(ost, nE, stride, r64, b32, x32);
}
void launch_cast_padded(const Geo<double> &g, const OuterState *ost, size_t stride64, const double2 *r64,
                        PadLayout pl, float2 *b32, float2 *x32, int nrhs, cudaStream_t s)
{
    counted(1);
    km_cast_p<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, ost, stride64, r64, pl, b32, x32);
}
void launch_update_padded(const Geo<double> &g, const OuterState *ost, size_t stride64, PadLayout pl,
                          const float2 *d32, double2 *X, int nrhs, cudaStream_t s)
{
    counted(1);
    km_update_p<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, ost, stride64, pl, d32, X);
}
void launch_to_padded(const Geo<double> &g, const double *src, PadLayout pl, float *dst, cudaStream_t s)
{
    counted(1);
    k_to_padded<<<grid_for(g.nE), kThreads, 0, s>>>(g, src, pl, dst);
}
void launch_nodes_to_padded(const Geo<double> &g, const double *src, PadLayout pl, float *dst, cudaStream_t s)
{
    counted(1);
    k_nodes_to_padded<<<grid_for(g.nN), kThreads, 0, s>>>(g, src, pl, dst);
}
void launch_update(const OuterState *ost, int nE, size_t stride, const float2 *d32, double2 *X, int nrhs, cudaStream_t s)
{
    counted(1);
    km_update<<<dim3(grid_for(nE), nrhs), kThreads, 0, s>>>(ost, nE, stride, d32, X);
}
void launch_divcorr_start(const DArgs &a, int nrhs, cudaStream_t s)
{
    counted(1);
    kd_rhs<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}
void launch_divcorr_iter(const DArgs &a, int nrhs, cudaStream_t s)
{
    counted(3);
    dim3 grid(a.nblk, nrhs);
    kd_p<<<grid, kThreads, 0, s>>>(a);
    kd_q<<<grid, kThreads, 0, s>>>(a);
    kd_xr<<<grid, kThreads, 0, s>>>(a);
}
void launch_divcorr_finish(const DArgs &a, int nrhs, cudaStream_t s)
{
    counted(2);
    kd_grad<<<dim3(a.enblk, nrhs), kThreads, 0, s>>>(a);
    kd_divj<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}
void launch_keep_boundary(const Geo<double> &g, double2 *v, size_t stride, int nrhs, cudaStream_t s)
{
    counted(1);
    k_keep_boundary<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, v, stride);
}
void launch_keep_interior(const Geo<double> &g, double2 *v, size_t stride, int nrhs, cudaStream_t s)
{
    counted(1);
    k_keep_interior<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, v, stride);
}
void launch_add_src(const Geo<double> &g, double2 *b, const double2 *src, size_t stride, const OuterState *ost, int nrhs,
                    cudaStream_t s)
{
    counted(1);
    k_add_src<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, b, src, stride, ost);
}
void launch_phi0(const Geo<double> &g, const double2 *src, size_t estride, double2 *phi0, size_t nstride,
                 const OuterState *ost, int nrhs, cudaStream_t s)
{
    counted(1);
    k_phi0<<<dim3(grid_for(g.nN), nrhs), kThreads, 0, s>>>(g, src, estride, phi0, nstride, ost);
}
void launch_post(const Geo<double> &g, double2 *E, const double2 *bc, size_t stride, const OuterState *ost, int nrhs,
                 cudaStream_t s)
{
    counted(2);
    k_post_scale<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, E, stride, ost);
    k_post_boundary<<<dim3(grid_for(g.nE), nrhs), kThreads, 0, s>>>(g, E, bc, stride, ost);
}
void launch_pmult_t(const Geo<double> &g, int npol, const double2 *e0, const double2 *ea, double omega, const double *m0,
                    double *dm, cudaStream_t s)
{
    counted(1);
    const int nEarth = g.nx * g.ny * (g.nz - g.nzAir);
    k_pmult_t<<<grid_for(nEarth), kThreads, 0, s>>>(g, npol, e0, ea, omega, m0, dm);
}
void launch_nonzero(const double2 *v, size_t stride, int n, int *flags, int nrhs, cudaStream_t s)
{
    counted(1);
    k_nonzero<<<dim3(grid_for(n), nrhs), kThreads, 0, s>>>(v, stride, n, flags);
}
void launch_scatter_interior(int nEi, const int *edgei, const double2 *vi, double2 *vf, cudaStream_t s)
{
    counted(1);
    k_scatter_interior<<<grid_for(nEi), kThreads, 0, s>>>(nEi, edgei, vi, vf);
}
void launch_gather_interior(int nEi, const int *edgei, const double2 *vf, double2 *vi, cudaStream_t s)
{
    counted(1);
    k_gather_interior<<<grid_for(nEi), kThreads, 0, s>>>(nEi, edgei, vf, vi);
}

}  // namespace mt3d

// common.cuh -- shared device definitions of the 3D-MT solver kernels.
//
// Storage (HBM): every field is a full edge vector in ModEM's getCVector order
// (x-edges (nx, ny+1, nz+1), then y-edges (nx+1, ny, nz+1), then z-edges
// (nx+1, ny+1, nz), each x fastest), complex interleaved (double2 / float2).
// A batch of right-hand sides is nrhs such vectors back to back.  Boundary
// entries of Krylov vectors are kept at zero so the stencil needs no branches
// on its neighbours.  Node scalars (div correction) are (nx+1, ny+1, nz+1).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mt3d {

// f90/UTILS/math_constants.f90:12-19
constexpr double kPiRef = 3.14159265357898;
constexpr double kMu0 = kPiRef * 0.0000004;
constexpr double kSigmaAir = (double)1.0e-10f;  // single-precision literal in the reference

constexpr int kThreads = 256;
constexpr int kMaxParts = 4;  // doubles reduced per kernel (two complex numbers)
constexpr int kMaxBatch = 65535;  // right-hand sides per solve call (the launch grids' y extent)

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
template <typename T> struct cplx_of;
template <> struct cplx_of<double> { using type = double2; };
template <> struct cplx_of<float> { using type = float2; };
template <typename T> using C2 = typename cplx_of<T>::type;

template <typename T> __host__ __device__ inline C2<T> mk(T re, T im) { C2<T> c; c.x = re; c.y = im; return c; }
template <typename C> __host__ __device__ inline C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __host__ __device__ inline C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __host__ __device__ inline C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename C, typename T> __host__ __device__ inline C cscale(C a, T s) { a.x *= s; a.y *= s; return a; }

struct cd {  // host/device complex double scalar (solver state)
    double re, im;
};
__host__ __device__ inline cd cd_mul(cd a, cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__host__ __device__ inline cd cd_div(cd a, cd b)
{
    // Smith's algorithm (avoids overflow in |b|^2)
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, den = b.re + b.im * r;
        return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    } else {
        double r = b.re / b.im, den = b.re * r + b.im;
        return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
    }
}
__host__ __device__ inline bool cd_zero(cd a) { return a.re == 0.0 && a.im == 0.0; }
__host__ __device__ inline bool cd_finite(cd a) { return isfinite(a.re) && isfinite(a.im); }

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
template <typename T> struct Geo {
    int nx, ny, nz, nzAir;
    int nXe, nYe, nZe, nE, nN;
    // 0-based 1-D tables: cell widths d*, node-centred widths del*, reciprocals
    const T *dx, *dy, *dz, *delX, *delY, *delZ, *rdx, *rdy, *rdz;
};

// component and (i, j, k) of a flat edge index
struct EdgeIdx {
    int c, i, j, k;
};
template <typename T> __device__ __forceinline__ EdgeIdx edge_decode(const Geo<T> &g, int e)
{
    EdgeIdx r;
    if (e < g.nXe) {
        r.c = 0;
        r.i = e % g.nx;
        int t = e / g.nx;
        r.j = t % (g.ny + 1);
        r.k = t / (g.ny + 1);
    } else if (e < g.nXe + g.nYe) {
        int e2 = e - g.nXe;
        r.c = 1;
        r.i = e2 % (g.nx + 1);
        int t = e2 / (g.nx + 1);
        r.j = t % g.ny;
        r.k = t / g.ny;
    } else {
        int e3 = e - g.nXe - g.nYe;
        r.c = 2;
        r.i = e3 % (g.nx + 1);
        int t = e3 / (g.nx + 1);
        r.j = t % (g.ny + 1);
        r.k = t / (g.ny + 1);
    }
    return r;
}
template <typename T> __device__ __forceinline__ bool edge_interior(const Geo<T> &g, const EdgeIdx &q)
{
    if (q.c == 0) return q.j >= 1 && q.j <= g.ny - 1 && q.k >= 1 && q.k <= g.nz - 1;
    if (q.c == 1) return q.i >= 1 && q.i <= g.nx - 1 && q.k >= 1 && q.k <= g.nz - 1;
    return q.i >= 1 && q.i <= g.nx - 1 && q.j >= 1 && q.j <= g.ny - 1;
}
template <typename T> __device__ __forceinline__ int iX(const Geo<T> &g, int i, int j, int k)
{
    return i + g.nx * (j + (g.ny + 1) * k);
}
template <typename T> __device__ __forceinline__ int iY(const Geo<T> &g, int i, int j, int k)
{
    return g.nXe + i + (g.nx + 1) * (j + g.ny * k);
}
template <typename T> __device__ __forceinline__ int iZ(const Geo<T> &g, int i, int j, int k)
{
    return g.nXe + g.nYe + i + (g.nx + 1) * (j + (g.ny + 1) * k);
}
template <typename T> __device__ __forceinline__ int iN(const Geo<T> &g, int i, int j, int k)
{
    return i + (g.nx + 1) * (j + (g.ny + 1) * k);
}

// Edge volume V_E (EdgeVolume, f90/3D_MT/GridCalc.f90:44-90)
template <typename T> __device__ __forceinline__ T edge_volume(const Geo<T> &g, const EdgeIdx &q)
{
    if (q.c == 0) return g.dx[q.i] * (g.delY[q.j] * g.delZ[q.k]);
    if (q.c == 1) return g.dy[q.j] * (g.delX[q.i] * g.delZ[q.k]);
    return g.dz[q.k] * (g.delX[q.i] * g.delY[q.j]);
}

// V_E times the diagonal of the curl-curl operator (V_E*xXO, V_E*yYO, V_E*zZO
// of CurlcurleSetUp, f90/3D_MT/FWD/modelOperator3D.f90:430-494), interior edges.
template <typename T> __device__ __forceinline__ T cc_diag(const Geo<T> &g, const EdgeIdx &q)
{
    if (q.c == 0)
        return g.dx[q.i] * g.delZ[q.k] * (g.rdy[q.j] + g.rdy[q.j - 1]) +
               g.dx[q.i] * g.delY[q.j] * (g.rdz[q.k] + g.rdz[q.k - 1]);
    if (q.c == 1)
        return g.dy[q.j] * g.delX[q.i] * (g.rdz[q.k] + g.rdz[q.k - 1]) +
               g.dy[q.j] * g.delZ[q.k] * (g.rdx[q.i] + g.rdx[q.i - 1]);
    return g.dz[q.k] * g.delY[q.j] * (g.rdx[q.i] + g.rdx[q.i - 1]) +
           g.dz[q.k] * g.delX[q.i] * (g.rdy[q.j] + g.rdy[q.j - 1]);
}

// (A x)_e for an interior edge: V_E (curl curl x) + i*dsgn*omega*mu0*sigma*V_E*x_e,
// the Maxwell stencil of f90/3D_MT/FWD/modelOperator3D.f90:692-800 multiplied
// through by V_E (MultA_N, :879-918).  Multiplying the coefficient tables of
// CurlcurleSetUp by V_E leaves node-centred widths as the cross-term weights
// and differences of the same-component neighbours scaled by 1/d; the terms
// are grouped as differences (fluxes) to limit cancellation in FP32.
// dsgn = ISIGN = -1 for A, +1 for the conjugate-transposed operator.
template <typename T>
__device__ __forceinline__ C2<T> stencil(const Geo<T> &g, const C2<T> *__restrict__ x, const EdgeIdx &q, T wmusig_ve)
{
    using C = C2<T>;
    const int i = q.i, j = q.j, k = q.k;
    C acc;
    if (q.c == 0) {
        const int e = iX(g, i, j, k);
        const C x0 = x[e];
        const C yy = csub(cadd(csub(x[iY(g, i + 1, j, k)], x[iY(g, i, j, k)]), x[iY(g, i, j - 1, k)]), x[iY(g, i + 1, j - 1, k)]);
        const C zz = csub(cadd(csub(x[iZ(g, i + 1, j, k)], x[iZ(g, i, j, k)]), x[iZ(g, i, j, k - 1)]), x[iZ(g, i + 1, j, k - 1)]);
        const C fyp = cscale(csub(x[iX(g, i, j + 1, k)], x0), g.rdy[j]);
        const C fym = cscale(csub(x0, x[iX(g, i, j - 1, k)]), g.rdy[j - 1]);
        const C fzp = cscale(csub(x[iX(g, i, j, k + 1)], x0), g.rdz[k]);
        const C fzm = cscale(csub(x0, x[iX(g, i, j, k - 1)]), g.rdz[k - 1]);
        const T wy = g.dx[i] * g.delZ[k], wz = g.dx[i] * g.delY[j];
        acc = cadd(cscale(yy, g.delZ[k]), cscale(zz, g.delY[j]));
        acc = csub(acc, cscale(csub(fyp, fym), wy));
        acc = csub(acc, cscale(csub(fzp, fzm), wz));
        acc.x -= wmusig_ve * x0.y;  // + i*dterm*x0, dterm = dsgn*omega*mu0*sigma*V_E
        acc.y += wmusig_ve * x0.x;
    } else if (q.c == 1) {
        const int e = iY(g, i, j, k);
        const C x0 = x[e];
        const C zz = csub(cadd(csub(x[iZ(g, i, j + 1, k)], x[iZ(g, i, j, k)]), x[iZ(g, i, j, k - 1)]), x[iZ(g, i, j + 1, k - 1)]);
        const C xx = csub(cadd(csub(x[iX(g, i, j + 1, k)], x[iX(g, i, j, k)]), x[iX(g, i - 1, j, k)]), x[iX(g, i - 1, j + 1, k)]);
        const C fzp = cscale(csub(x[iY(g, i, j, k + 1)], x0), g.rdz[k]);
        const C fzm = cscale(csub(x0, x[iY(g, i, j, k - 1)]), g.rdz[k - 1]);
        const C fxp = cscale(csub(x[iY(g, i + 1, j, k)], x0), g.rdx[i]);
        const C fxm = cscale(csub(x0, x[iY(g, i - 1, j, k)]), g.rdx[i - 1]);
        const T wz = g.dy[j] * g.delX[i], wx = g.dy[j] * g.delZ[k];
        acc = cadd(cscale(zz, g.delX[i]), cscale(xx, g.delZ[k]));
        acc = csub(acc, cscale(csub(fzp, fzm), wz));
        acc = csub(acc, cscale(csub(fxp, fxm), wx));
        acc.x -= wmusig_ve * x0.y;
        acc.y += wmusig_ve * x0.x;
    } else {
        const int e = iZ(g, i, j, k);
        const C x0 = x[e];
        const C xx = csub(cadd(csub(x[iX(g, i, j, k + 1)], x[iX(g, i, j, k)]), x[iX(g, i - 1, j, k)]), x[iX(g, i - 1, j, k + 1)]);
        const C yy = csub(cadd(csub(x[iY(g, i, j, k + 1)], x[iY(g, i, j, k)]), x[iY(g, i, j - 1, k)]), x[iY(g, i, j - 1, k + 1)]);
        const C fxp = cscale(csub(x[iZ(g, i + 1, j, k)], x0), g.rdx[i]);
        const C fxm = cscale(csub(x0, x[iZ(g, i - 1, j, k)]), g.rdx[i - 1]);
        const C fyp = cscale(csub(x[iZ(g, i, j + 1, k)], x0), g.rdy[j]);
        const C fym = cscale(csub(x0, x[iZ(g, i, j - 1, k)]), g.rdy[j - 1]);
        const T wx = g.dz[k] * g.delY[j], wy = g.dz[k] * g.delX[i];
        acc = cadd(cscale(xx, g.delY[j]), cscale(yy, g.delX[i]));
        acc = csub(acc, cscale(csub(fxp, fxm), wx));
        acc = csub(acc, cscale(csub(fyp, fym), wy));
        acc.x -= wmusig_ve * x0.y;
        acc.y += wmusig_ve * x0.x;
    }
    return acc;
}

// ---------------------------------------------------------------------------
// device-side solver state (one per right-hand side)
// ---------------------------------------------------------------------------
enum KStatus : int { KS_IDLE = 0, KS_RUNNING = 1, KS_CONVERGED = 2, KS_BREAKDOWN = 3, KS_MAXIT = 4, KS_NAN = 5 };

struct BicgState {
    cd rho, rho1, alpha, omega, beta;
    double bnorm, btol, rnorm, rnormin;
    double rn2;  // fused FP32 iteration: ||s - omega t||^2 from the inner products of t = A sh
    int iter;    // iterations completed in this call
    int maxit;
    int status;  // KStatus
    int xcur, xbest, imin;
    int first;   // 1 until the first iteration of the call has formed p
    int pad;
};

// QMR without look-ahead (f90/3D_MT/FWD/solver.f90:122-343), one per
// right-hand side; the names are the reference's
struct QmrState {
    cd rho, rho1, psi, delta, epsil, beta, eta, thet, thet1, gamm, gamm1, tm2, pde, rde;
    double bnorm, tol;
    int iter;    // the reference's counter (1 before the first iteration)
    int maxit;
    int status;  // KStatus
    int zero;    // zero right-hand side: zero solution
};

struct PcgState {
    cd delta, deltaOld, alpha, beta;
    double bnorm, rnorm, tol;
    int iter;  // the reference's counter i (starts at 1)
    int maxit;
    int status;
    int pad;
};

// per right-hand side control and diagnostics of the outer (divergence
// correction) loop, FWDsolve3D
struct OuterState {
    double omega;        // angular frequency
    double tol;          // target relative residual (tolEMfwd / tolEMadj)
    double tol_inner;    // mixed: relative tolerance of the FP32 correction solve
    double bnorm64;      // ||b|| of the FP64 interior system
    double relres;       // last true relative residual ||b - A x|| / ||b||
    double scale;        // mixed: 1/||r64|| used to normalise the FP32 right-hand side
    double divJ[2];      // last divergence before/after
    int active;          // still iterating
    int converged;
    int failed;
    int nDivCor;
    int nIterTotal;
    int trans;
    int dc_run;          // run a divergence correction in this cycle
    int has_src;
    int has_bc;
    int pad;
};

// ---------------------------------------------------------------------------
// block reduction of up to kMaxParts doubles; the last block of a right-hand
// side finalises.  Deterministic: partials are summed in block-index order.
// ---------------------------------------------------------------------------
template <int N> __device__ __forceinline__ void warp_sum(double (&v)[N])
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int n = 0; n < N; n++) v[n] += __shfl_xor_sync(0xffffffffu, v[n], o);
}

// Reduce v over the block, write this block's partial, and return true in
// the (single) last block of this right-hand side, whose thread 0 then holds
// the total in `tot`.  `parts` is [nrhs][nblk][N]; `cnt` one counter per rhs.
// As block_reduce_last below, for blocks of NT threads, with its shared
// scratch (N * NT / 32 doubles and one flag) supplied by the caller, e.g.
// part of a ring buffer the block no longer reads.
template <int N, int NT = kThreads>
__device__ __forceinline__ bool block_reduce_last_in(double (&v)[N], double *__restrict__ parts, unsigned *cnt,
                                                     int rhs, int blk, int nblk, double (&tot)[N], double *scratch,
                                                     int *flag)
{
    double(*sm)[NT / 32] = reinterpret_cast<double(*)[NT / 32]>(scratch);
    int &s_last = *flag;
    warp_sum<N>(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int n = 0; n < N; n++) sm[n][w] = v[n];
    __syncthreads();
    if (threadIdx.x == 0) {
        double *p = parts + ((size_t)rhs * nblk + blk) * N;
#pragma unroll
        for (int n = 0; n < N; n++) {
            double s = 0.0;
            for (int q = 0; q < NT / 32; q++) s += sm[n][q];
            p[n] = s;
        }
        __threadfence();
        unsigned t = atomicAdd(&cnt[rhs], 1u);
        s_last = (t == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double acc[N];
#pragma unroll
    for (int n = 0; n < N; n++) acc[n] = 0.0;
    const volatile double *pp = parts + (size_t)rhs * nblk * N;
    for (int b = threadIdx.x; b < nblk; b += NT)
#pragma unroll
        for (int n = 0; n < N; n++) acc[n] += pp[(size_t)b * N + n];
    warp_sum<N>(acc);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int n = 0; n < N; n++) sm[n][w] = acc[n];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int n = 0; n < N; n++) {
            double s = 0.0;
            for (int q = 0; q < NT / 32; q++) s += sm[n][q];
            tot[n] = s;
        }
        cnt[rhs] = 0u;
    }
    return true;
}

template <int N>
__device__ __forceinline__ bool block_reduce_last(double (&v)[N], double *__restrict__ parts, unsigned *cnt, int rhs,
                                                  int blk, int nblk, double (&tot)[N])
{
    __shared__ double sm[N][kThreads / 32];
    __shared__ bool s_last;
    warp_sum<N>(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int n = 0; n < N; n++) sm[n][w] = v[n];
    __syncthreads();
    if (threadIdx.x == 0) {
        double* p = parts + ((size_t)rhs * nblk + blk) * N;
#pragma unroll
        for (int n = 0; n < N; n++) {
            double s = 0.0;
            for (int q = 0; q < kThreads / 32; q++) s += sm[n][q];
            p[n] = s;
        }
        __threadfence();
        unsigned t = atomicAdd(&cnt[rhs], 1u);
        s_last = (t == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double acc[N];
#pragma unroll
    for (int n = 0; n < N; n++) acc[n] = 0.0;
    const volatile double *pp = parts + (size_t)rhs * nblk * N;
    for (int b = threadIdx.x; b < nblk; b += kThreads)
#pragma unroll
        for (int n = 0; n < N; n++) acc[n] += pp[(size_t)b * N + n];
    warp_sum<N>(acc);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int n = 0; n < N; n++) sm[n][w] = acc[n];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int n = 0; n < N; n++) {
            double s = 0.0;
            for (int q = 0; q < kThreads / 32; q++) s += sm[n][q];
            tot[n] = s;
        }
        cnt[rhs] = 0u;
    }
    return true;
}

}  // namespace mt3d

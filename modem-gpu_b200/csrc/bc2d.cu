// bc2d.cu -- boundary conditions and first guess of the 3-D forward problem
// from 2-D TE solutions on the slices of the model (BC_x0_WS,
// f90/3D_MT/FWD/boundary_ws.f90:21-168, through ComputeBC,
// f90/3D_MT/FWD/modelOperator3D.f90:268-293).
//
// imode = 2: one 2-D problem per x-slice (horizontal axis y), field on the
// x-edges; imode = 1: one per y-slice (horizontal axis x), field on the
// y-edges.  Per slice (nh horizontal cells, nz vertical cells, air on top):
//   k_bc1d    the 1-D TE columns of SetBound2D_TE (Fwd1D_TE,
//             f90/3D_MT/FWD/Mod2d/WSfwd1Dmod.f90:70-126): both side columns
//             in full and, for every interior column, the bottom value of the
//             column with the area-averaged conductivity; one thread per
//             column, tridiagonal elimination (the 1-D matrix is diagonally
//             dominant, so no pivoting is needed);
//   k_bc_coef the operator coefficients and right-hand side per unknown;
//   k_bc2d    the 2-D TE system of SetupA_TE / FormAII / MulAibWithXb /
//             Fwd2DsolveTE (WSfwd2Dmod.f90:32-127, 325-418; FwdTEmod.f90:
//             104-157): (nh-1)(nz-1) interior nodes, bandwidth m = nz-1.  One
//             block per slice runs Gaussian elimination on the band with the
//             right-hand side carried along.  The active (m+1) x (m+1) window
//             lives in shared memory as a circular buffer; each step writes
//             the finished row of U out and loads the one new row and column
//             of A, which no earlier step has touched;
//   k_bc_back the back substitution, one warp per slice.  The matrix is column diagonally dominant
//             (the off-diagonal entries are real and sum to minus the real
//             part of the diagonal), so elimination without row exchanges is
//             stable; the reference's LAPACK band LU agrees with it to
//             rounding.
// The output is the full edge vector E0 with the tangential field of the
// bottom face zero (boundary_ws.f90:155-156): its boundary entries are the
// BC, its interior entries the first guess.
#include <algorithm>
#include <atomic>
#include <cmath>

#include "kernels.h"
#include "solver.h"

namespace mt3d {

extern std::atomic<long long> g_launch_count;

namespace {

__device__ __forceinline__ double2 c2(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 cm(double2 a, double2 b)
{
    return c2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a / b by Smith's algorithm
__device__ __forceinline__ double2 cdv(double2 a, double2 b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return c2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    }
    const double r = b.x / b.y, den = b.x * r + b.y;
    return c2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}

struct Slice {
    const BcArgs &a;
    int s;
    __device__ Slice(const BcArgs &a_, int s_) : a(a_), s(s_) {}
    // conductivity of cell (h, k) of the slice, the air at SIGMA_AIR
    __device__ double ccon(int h, int k) const
    {
        if (k < a.nza) return kSigmaAir;
        const long long c = a.imode == 2 ? s + (long long)a.nx * (h + (long long)a.ny * k)
                                         : h + (long long)a.nx * (s + (long long)a.ny * k);
        return a.sigC[c];
    }
    // flat edge index of node (h, k) of the slice
    __device__ long long edge(int h, int k) const
    {
        return a.imode == 2 ? s + (long long)a.nx * (h + (long long)(a.ny + 1) * k)
                            : a.nXe + h + (long long)(a.nx + 1) * (s + (long long)a.ny * k);
    }
};

}  // namespace

// 1-D TE columns.  Thread (slice, col): col 0 and col nh are the side
// columns (cells 0 and nh-1), solved in full into side[slice][0 / 1][0..nz];
// 1 <= col < nh averages cells col-1 and col and keeps the bottom node only.
__global__ void k_bc1d(BcArgs a)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)a.nslice * (a.nh + 1)) return;
    const int s = (int)(t / (a.nh + 1)), col = (int)(t % (a.nh + 1));
    const Slice sl(a, s);
    const int nz = a.nz;
    const int side = col == 0 ? 0 : (col == a.nh ? 1 : -1);
    auto s1d = [&](int k) -> double {
        if (k < a.nza) return kSigmaAir;
        if (col == 0) return sl.ccon(0, k);
        if (col == a.nh) return sl.ccon(a.nh - 1, k);
        return (sl.ccon(col - 1, k) * a.dh[col - 1] + sl.ccon(col, k) * a.dh[col]) / (a.dh[col - 1] + a.dh[col]);
    };
    const double sb = s1d(nz - 1);
    const double skd = sqrt(2.0 / (sb * a.omue));
    auto dz1 = [&](int k) -> double { return k < nz ? a.dz[k] : skd; };
    auto s1 = [&](int k) -> double { return k < nz ? s1d(k) : sb; };
    double2 *cp = side >= 0 ? a.cpr + ((size_t)s * 2 + side) * nz : nullptr;
    double2 *xs = side >= 0 ? a.side + ((size_t)s * 2 + side) * (nz + 1) : nullptr;
    // row j: ad_{j-1} x_{j-1} + ac_j x_j + ad_j x_{j+1} = r_j, r_0 = -au_0
    double2 cprev = c2(0, 0), dprev = c2(0, 0);
    double adprev = 0.0, sk = s1(0), dk = dz1(0);
    for (int j = 0; j < nz; j++) {
        const double sk1 = s1(j + 1), dk1 = dz1(j + 1);
        const double au = 2.0 / dk, ad = 2.0 / dk1;
        const double ss = sk1 * dk1 + sk * dk;
        const double2 ac = c2(-au - ad, a.omue * ss);
        const double2 den = c2(ac.x - adprev * cprev.x, ac.y - adprev * cprev.y);
        const double2 r = j == 0 ? c2(-au, 0.0) : c2(0.0, 0.0);
        const double2 cj = cdv(c2(ad, 0.0), den);
        const double2 dj = cdv(c2(r.x - adprev * dprev.x, r.y - adprev * dprev.y), den);
        if (side >= 0) {
            cp[j] = cj;
            xs[j + 1] = dj;
        }
        cprev = cj;
        dprev = dj;
        adprev = ad;
        sk = sk1;
        dk = dk1;
    }
    if (side < 0) {
        a.bottom[(size_t)s * (a.nh + 1) + col] = dprev;  // x at the bottom node = last d'
        return;
    }
    xs[0] = c2(1.0, 0.0);
    double2 xn = xs[nz];
    for (int j = nz - 2; j >= 0; j--) {
        const double2 d = xs[j + 1];
        xn = c2(d.x - (cp[j].x * xn.x - cp[j].y * xn.y), d.y - (cp[j].x * xn.y + cp[j].y * xn.x));
        xs[j + 1] = xn;
    }
}

namespace {
// 2-D operator of one slice: unknown r <-> node (iy, iz) = (r / m + 1, r % m + 1)
struct Op2d {
    const BcArgs &a;
    const Slice &sl;
    int m, n;
    __device__ Op2d(const BcArgs &a_, const Slice &sl_) : a(a_), sl(sl_), m(a_.nz - 1), n((a_.nh - 1) * (a_.nz - 1)) {}
    __device__ double cz(int iz) const { return a.dz[iz] + a.dz[iz - 1]; }
    __device__ double cy(int iy) const { return a.dh[iy] + a.dh[iy - 1]; }
    __device__ double2 diag(int r) const
    {
        const int iy = r / m + 1, iz = r % m + 1;
        const double s00 = sl.ccon(iy, iz), s10 = sl.ccon(iy, iz - 1), s01 = sl.ccon(iy - 1, iz),
                     s11 = sl.ccon(iy - 1, iz - 1);
        const double dzi = a.dz[iz], dzm = a.dz[iz - 1], dyi = a.dh[iy], dym = a.dh[iy - 1];
        const double s2d = (s00 * dzi * dyi + s01 * dzi * dym + s10 * dzm * dyi + s11 * dzm * dym) /
                           (dzi * dyi + dzi * dym + dzm * dyi + dzm * dym);
        const double czv = cz(iz), cyv = cy(iy);
        const double ar = 2.0 * czv / dyi, al = 2.0 * czv / dym, ad = 2.0 * cyv / dzi, au = 2.0 * cyv / dzm;
        return c2(-ar - al - ad - au, a.omue * (cyv * czv * s2d));
    }
    // A(r, r+1): vertical neighbour, none below the last interior row
    __device__ double zc(int r) const
    {
        const int iy = r / m + 1, iz = r % m + 1;
        return iz == m ? 0.0 : 2.0 * cy(iy) / a.dz[iz];
    }
    // A(r, r+m): horizontal neighbour, none right of the last interior column
    __device__ double yc(int r) const
    {
        const int iy = r / m + 1, iz = r % m + 1;
        return iy == a.nh - 1 ? 0.0 : 2.0 * cz(iz) / a.dh[iy];
    }
    __device__ double2 at(int r, int c) const
    {
        if (r >= n || c >= n) return c2(0, 0);
        const int d = c - r;
        if (d == 0) return diag(r);
        if (d == 1) return c2(zc(r), 0);
        if (d == -1) return c2(zc(c), 0);
        if (d == m) return c2(yc(r), 0);
        if (d == -m) return c2(yc(c), 0);
        return c2(0, 0);
    }
    // -A_ib x_b (MulAibWithXb)
    __device__ double2 rhs(int r, const double2 *left, const double2 *right, const double2 *bottom) const
    {
        if (r >= n) return c2(0, 0);
        const int iy = r / m + 1, iz = r % m + 1;
        double2 v = c2(0, 0);
        if (iy == 1) {
            const double b = 2.0 * cz(iz) / a.dh[0];
            v = c2(-(b * left[iz].x), -(b * left[iz].y));
        }
        if (iy == a.nh - 1) {
            const double b = 2.0 * cz(iz) / a.dh[a.nh - 1];
            v = c2(-(b * right[iz].x), -(b * right[iz].y));
        }
        if (iz == 1) v.x -= 2.0 * cy(iy) / a.dz[0];
        if (iz == m) {
            const double b = 2.0 * cy(iy) / a.dz[a.nz - 1];
            v = c2(v.x - b * bottom[iy].x, v.y - b * bottom[iy].y);
        }
        return v;
    }
};
}  // namespace

// Coefficients of the 2-D operators and right-hand sides of the slices of a
// launch chunk, one thread per unknown: the diagonal, A(r, r+1), A(r, r+m)
// and -A_ib x_b, so that the elimination reads them instead of forming them
// on its critical path.
__global__ void k_bc_coef(BcArgs a, int nslices)
{
    const int m = a.nz - 1, n = (a.nh - 1) * m;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= (long long)nslices * n) return;
    const int q = (int)(t / n), r = (int)(t % n), s = a.slice0 + q;
    const Slice sl(a, s);
    const Op2d op(a, sl);
    const double2 *left = a.side + (size_t)s * 2 * (a.nz + 1), *right = left + (a.nz + 1);
    const double2 *bottom = a.bottom + (size_t)s * (a.nh + 1);
    a.cd[t] = op.diag(r);
    a.czc[t] = op.zc(r);
    a.cyc[t] = op.yc(r);
    a.cb[t] = op.rhs(r, left, right, bottom);
}

// One block (32 x BY threads) per slice of the launch chunk.
__global__ void __launch_bounds__(1024) k_bc2d(BcArgs a, int smem_window)
{
    extern __shared__ double2 sm[];
    const int s = a.slice0 + blockIdx.x;
    const Slice sl(a, s);
    const Op2d op(a, sl);
    const int m = op.m, n = op.n, M = m + 1;
    double2 *W = smem_window ? sm : a.W + (size_t)blockIdx.x * M * M;
    double2 *rw = smem_window ? sm + (size_t)M * M : sm;  // right-hand side window
    double2 *U = a.U + (size_t)blockIdx.x * n * M;
    double2 *y = a.y + (size_t)blockIdx.x * n;
    const double2 *left = a.side + (size_t)s * 2 * (a.nz + 1), *right = left + (a.nz + 1);
    const double2 *bottom = a.bottom + (size_t)s * (a.nh + 1);
    const int tx = threadIdx.x, ty = threadIdx.y, nt = blockDim.x * blockDim.y, tid = ty * blockDim.x + tx;
    const double2 *cd = a.cd + (size_t)blockIdx.x * n, *cb = a.cb + (size_t)blockIdx.x * n;
    const double *czc = a.czc + (size_t)blockIdx.x * n, *cyc = a.cyc + (size_t)blockIdx.x * n;
    // A(r, c) of the slice from the coefficient arrays
    auto at = [&](int r, int c) -> double2 {
        if (r >= n || c >= n) return c2(0, 0);
        const int d = c - r;
        if (d == 0) return cd[r];
        if (d == 1) return c2(czc[r], 0);
        if (d == -1) return c2(czc[c], 0);
        if (d == m) return c2(cyc[r], 0);
        if (d == -m) return c2(cyc[c], 0);
        return c2(0, 0);
    };

    // boundary nodes of E0: side columns, 1 along the top; the bottom row stays zero
    for (int k = tid; k < a.nz; k += nt) {
        a.e0[sl.edge(0, k)] = left[k];
        a.e0[sl.edge(a.nh, k)] = right[k];
    }
    for (int h = 1 + tid; h < a.nh; h += nt) a.e0[sl.edge(h, 0)] = c2(1.0, 0.0);

    // window of step 0: rows and columns 0..m
    for (int q = tid; q < M * M; q += nt) {
        const int r = q / M, c = q % M;
        W[r * M + c] = at(r, c);
    }
    for (int r = tid; r < M; r += nt) rw[r] = r < n ? cb[r] : c2(0, 0);
    __syncthreads();

    for (int j = 0; j < n; j++) {
        const int s0 = j % M;
        // the row and column rn = j + M that enter at the end of this step hold
        // three nonzeros, A(rn, rn) and the symmetric pairs A(rn - 1, rn),
        // A(rn - m, rn); their loads are issued here, ahead of their use
        const int rn = j + M;
        const bool newrow = rn < n;
        const double2 nd = newrow ? cd[rn] : c2(0, 0), nb = newrow ? cb[rn] : c2(0, 0);
        const double nz1 = newrow ? czc[rn - 1] : 0.0, nym = newrow ? cyc[rn - m] : 0.0;
        const double2 piv = W[s0 * M + s0];
        const double2 rp = cdv(c2(1.0, 0.0), piv);
        // rows j+a, columns j+b, a, b = 1..m
        if (m <= 4 * (int)blockDim.y) {
            // up to four rows per thread: their multipliers in registers, each
            // entry of the pivot row read once per column
            int ras[4];
            double2 ls[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int ai = 1 + ty + q * blockDim.y;
                int ra = s0 + ai;
                if (ra >= M) ra -= M;
                ras[q] = ra;
                ls[q] = ai <= m ? cm(W[ra * M + s0], rp) : c2(0, 0);
            }
            for (int bi = 1 + tx; bi <= m; bi += blockDim.x) {
                int cb = s0 + bi;
                if (cb >= M) cb -= M;
                const double2 u = W[s0 * M + cb];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const double2 l = ls[q];
                    if (l.x == 0.0 && l.y == 0.0) continue;
                    double2 w = W[ras[q] * M + cb];
                    w.x -= l.x * u.x - l.y * u.y;
                    w.y -= l.x * u.y + l.y * u.x;
                    W[ras[q] * M + cb] = w;
                }
            }
            if (tx == 0) {
                const double2 r0 = rw[s0];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const double2 l = ls[q];
                    if (l.x == 0.0 && l.y == 0.0) continue;
                    double2 w = rw[ras[q]];
                    w.x -= l.x * r0.x - l.y * r0.y;
                    w.y -= l.x * r0.y + l.y * r0.x;
                    rw[ras[q]] = w;
                }
            }
        } else {
            for (int ai = 1 + ty; ai <= m; ai += blockDim.y) {
                int ra = s0 + ai;
                if (ra >= M) ra -= M;
                const double2 l = cm(W[ra * M + s0], rp);
                if (l.x == 0.0 && l.y == 0.0) continue;
                for (int bi = 1 + tx; bi <= m; bi += blockDim.x) {
                    int cb = s0 + bi;
                    if (cb >= M) cb -= M;
                    const double2 u = W[s0 * M + cb];
                    double2 w = W[ra * M + cb];
                    w.x -= l.x * u.x - l.y * u.y;
                    w.y -= l.x * u.y + l.y * u.x;
                    W[ra * M + cb] = w;
                }
                if (tx == 0) {
                    const double2 r0 = rw[s0];
                    double2 w = rw[ra];
                    w.x -= l.x * r0.x - l.y * r0.y;
                    w.y -= l.x * r0.y + l.y * r0.x;
                    rw[ra] = w;
                }
            }
        }
        // the finished row of U and of the reduced right-hand side
        for (int bi = tid; bi < M; bi += nt) {
            int cb = s0 + bi;
            if (cb >= M) cb -= M;
            U[(size_t)j * M + bi] = W[s0 * M + cb];
        }
        if (tid == 0) y[j] = rw[s0];
        __syncthreads();
        // slot s0 now takes row rn (columns j+1..j+M) and column rn (rows
        // j+1..j+M-1): column j+1 = rn - m, column rn - 1 and the diagonal
        for (int bi = 1 + tid; bi <= M; bi += nt) {
            int cb = s0 + bi;
            if (cb >= M) cb -= M;
            W[s0 * M + cb] = bi == M ? nd : c2(bi == 1 ? nym : bi == M - 1 ? nz1 : 0.0, 0.0);
        }
        for (int ai = 1 + tid; ai < M; ai += nt) {
            int ra = s0 + ai;
            if (ra >= M) ra -= M;
            W[ra * M + s0] = c2(ai == 1 ? nym : ai == M - 1 ? nz1 : 0.0, 0.0);
        }
        if (tid == 0) rw[s0] = nb;
        __syncthreads();
    }
}

// Back substitution, one warp per slice: x_j = (y_j - sum_b U[j][b] x_{j+b}) /
// U[j][0] from j = n-1 down.  Each lane holds up to kBackP entries of a U row
// (columns lane + 32 p), and the row of step j - 1 is loaded while step j is
// reduced, so the chain waits on shuffles and not on memory.  The last M
// values of x live in shared memory as a circular buffer.
constexpr int kBackP = 8;
__global__ void __launch_bounds__(32) k_bc_back(BcArgs a)
{
    extern __shared__ double2 xs[];
    const int q = blockIdx.x, s = a.slice0 + q;
    const int m = a.nz - 1, n = (a.nh - 1) * m, M = a.nz;
    const Slice sl(a, s);
    const double2 *U = a.U + (size_t)q * n * M, *y = a.y + (size_t)q * n;
    const int tx = threadIdx.x;
    double2 u[kBackP], un[kBackP];
    auto load = [&](int j, double2 *dst) {
#pragma unroll
        for (int p = 0; p < kBackP; p++) {
            const int bi = tx + 32 * p;
            dst[p] = bi < M ? U[(size_t)j * M + bi] : c2(0, 0);
        }
    };
    load(n - 1, u);
    double2 yj = y[n - 1];
    for (int j = n - 1; j >= 0; j--) {
        double2 yn = c2(0, 0);
        if (j > 0) {
            load(j - 1, un);
            yn = y[j - 1];
        }
        double2 acc = c2(0, 0);
#pragma unroll
        for (int p = 0; p < kBackP; p++) {
            const int bi = tx + 32 * p;
            if (bi >= 1 && bi < M && j + bi < n) {
                const double2 xv = xs[(j + bi) % M];
                acc.x += u[p].x * xv.x - u[p].y * xv.y;
                acc.y += u[p].x * xv.y + u[p].y * xv.x;
            }
        }
        for (int bi = tx + 32 * kBackP; bi < M && j + bi < n; bi += 32) {  // rows longer than 32 kBackP
            const double2 uv = U[(size_t)j * M + bi], xv = xs[(j + bi) % M];
            acc.x += uv.x * xv.x - uv.y * xv.y;
            acc.y += uv.x * xv.y + uv.y * xv.x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        const double2 dg = c2(__shfl_sync(0xffffffffu, u[0].x, 0), __shfl_sync(0xffffffffu, u[0].y, 0));
        const double2 xj = cdv(c2(yj.x - acc.x, yj.y - acc.y), dg);
        __syncwarp();
        if (tx == 0) {
            xs[j % M] = xj;
            a.e0[sl.edge(j / m + 1, j % m + 1)] = xj;
        }
        __syncwarp();
#pragma unroll
        for (int p = 0; p < kBackP; p++) u[p] = un[p];
        yj = yn;
    }
}

size_t bc_smem_bytes(int nz, bool window_in_smem)
{
    const size_t M = (size_t)nz;
    return (window_in_smem ? M * M + M : M) * sizeof(double2);
}

void launch_bc_coef(const BcArgs &a, int nslices, cudaStream_t s)
{
    g_launch_count.fetch_add(1, std::memory_order_relaxed);
    const long long nt = (long long)nslices * (a.nh - 1) * (a.nz - 1);
    k_bc_coef<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(a, nslices);
}

void launch_bc_back(const BcArgs &a, int nslices, cudaStream_t s)
{
    const size_t smem = (size_t)a.nz * sizeof(double2);
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_bc_back, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    g_launch_count.fetch_add(1, std::memory_order_relaxed);
    k_bc_back<<<nslices, 32, smem, s>>>(a);
}

void launch_bc1d(const BcArgs &a, cudaStream_t s)
{
    g_launch_count.fetch_add(1, std::memory_order_relaxed);
    const long long nt = (long long)a.nslice * (a.nh + 1);
    k_bc1d<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(a);
}

int launch_bc2d(const BcArgs &a, int nblocks, bool window_in_smem, cudaStream_t s)
{
    const size_t smem = bc_smem_bytes(a.nz, window_in_smem);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_bc2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
    }
    const int m = a.nz - 1;
    const dim3 block(32, m >= 64 ? 32 : 16);
    g_launch_count.fetch_add(1, std::memory_order_relaxed);
    k_bc2d<<<nblocks, block, smem, s>>>(a, window_in_smem ? 1 : 0);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// host side (ComputeBC)
// ---------------------------------------------------------------------------
int Solver::compute_bc(int imode, double om, double *e0, bool device)
{
    if (!cond_set) return fail(5, "mt3d_compute_bc: conductivity not set (call mt3d_update_cond)");
    if ((imode != 1 && imode != 2) || !e0 || !(om > 0) || !std::isfinite(om))
        return fail(5, "mt3d_compute_bc: invalid arguments");
    const int nh = imode == 2 ? ny : nx, nslice = imode == 2 ? nx : ny;
    if (nh < 3 || nz < 3) return fail(5, "mt3d_compute_bc: the slices need at least 3 x 3 cells");
    const int64_t nC = (int64_t)nx * ny * nz, nEarth = (int64_t)nx * ny * (nz - nzAir);
    const int m = nz - 1, M = nz;
    const int64_t n = (int64_t)(nh - 1) * m;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev_);
    const bool smem = bc_smem_bytes(nz, true) <= (size_t)optin;
    // per slice: U rows (n x M), reduced right-hand side (n), diagonal (n),
    // operator right-hand side (n), the two couplings (2n doubles = n double2),
    // the window when it is not in shared memory (M x M)
    const size_t per_slice = ((size_t)n * M + 4 * (size_t)n + (smem ? 0 : (size_t)M * M)) * sizeof(double2);
    const size_t cap = (size_t)8 << 30;
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(nslice, cap / per_slice));
    const size_t fixed = ((size_t)nslice * 2 * (nz + 1) + (size_t)nslice * 2 * nz + (size_t)nslice * (nh + 1));
    if (bcs_.alloc(fixed * sizeof(double2) + (size_t)chunk * per_slice) || (!device && bce_.alloc(nE * sizeof(double2))))
        return fail(8, "mt3d_compute_bc: out of device memory");
    BcArgs a{};
    a.imode = imode;
    a.nh = nh;
    a.nz = nz;
    a.nza = nzAir;
    a.nslice = nslice;
    a.nx = nx;
    a.ny = ny;
    a.nXe = g64_.nXe;
    // the 2-D code receives the period 2 pi / omega and forms 2 pi / period
    const double per = (2.0 * kPiRef) / om;
    a.omue = ((2.0 * kPiRef) / per) * kMu0;
    a.dh = imode == 2 ? g64_.dy : g64_.dx;
    a.dz = g64_.dz;
    a.sigC = setup_.as<double>() + nEarth + 2 * nC;
    double2 *p = bcs_.as<double2>();
    a.side = p; p += (size_t)nslice * 2 * (nz + 1);
    a.cpr = p; p += (size_t)nslice * 2 * nz;
    a.bottom = p; p += (size_t)nslice * (nh + 1);
    a.U = p; p += (size_t)chunk * n * M;
    a.y = p; p += (size_t)chunk * n;
    a.cd = p; p += (size_t)chunk * n;
    a.cb = p; p += (size_t)chunk * n;
    a.czc = reinterpret_cast<double *>(p);
    a.cyc = a.czc + (size_t)chunk * n;
    p += (size_t)chunk * n;
    a.W = smem ? nullptr : p;
    a.e0 = device ? reinterpret_cast<double2 *>(e0) : bce_.as<double2>();
    int rc;
    if ((rc = check(cudaMemsetAsync(a.e0, 0, nE * sizeof(double2), stream_), "mt3d_compute_bc"))) return rc;
    launch_bc1d(a, stream_);
    for (int s0 = 0; s0 < nslice; s0 += chunk) {
        a.slice0 = s0;
        launch_bc_coef(a, std::min(chunk, nslice - s0), stream_);
        if ((rc = check((cudaError_t)launch_bc2d(a, std::min(chunk, nslice - s0), smem, stream_), "mt3d_compute_bc")))
            return rc;
        launch_bc_back(a, std::min(chunk, nslice - s0), stream_);
    }
    if (!device &&
        (rc = check(cudaMemcpyAsync(e0, a.e0, nE * sizeof(double2), cudaMemcpyDeviceToHost, stream_), "copy E0")))
        return rc;
    return sync("mt3d_compute_bc");
}

}  // namespace mt3d

// stagekernels.cu -- BiCGStab stencil kernels on the shared-memory staged
// stencil (stagestencil.cuh): the start of a Krylov call (r = b - A x), the
// two operator applications of an iteration with their fused dot products,
// and the FP64 true residual of the refinement loop.  The grad-div potentials
// are formed inside these kernels, so no separate potential pass runs.
//
// Grid: blockIdx.x = tile of node columns, blockIdx.y = right-hand side,
// blockIdx.z = chunk of node planes.  The number of chunks is chosen per
// launch shape so that the blocks fill the resident slots of the GPU in as
// few, as full waves as possible (stage_chunks).
#include <algorithm>
#include <atomic>
#include <mutex>

#include "finalize.cuh"
#include "kernels.h"
#include "stagestencil.cuh"

namespace mt3d {

extern std::atomic<long long> g_launch_count;
static inline void counted(int n) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

template <typename T> __device__ __forceinline__ StageSmem<T> &stage_smem()
{
    extern __shared__ __align__(16) unsigned char stage_raw[];
    return *reinterpret_cast<StageSmem<T> *>(stage_raw);
}
__device__ __forceinline__ void stage_tile(const ColMap &m, int &i0, int &j0)
{
    i0 = (blockIdx.x % m.tiles_x) * kStX;
    j0 = (blockIdx.x / m.tiles_x) * kStY;
}
template <typename T> __device__ __forceinline__ void stage_range(const Geo<T> &g, int &k0, int &k1)
{
    const int kc = (g.nz + 1 + gridDim.z - 1) / gridDim.z;
    k0 = blockIdx.z * kc;
    k1 = min(k0 + kc, g.nz + 1);
}
template <typename T> __device__ __forceinline__ T stage_wmu(const KArgs<T> &a, int r)
{
    return (T)(a.dsgn * a.ost[r].omega * kMu0);
}

// start of a call: r = b - A x0, rt = r; |b|^2, |r|^2
template <typename T> __global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 4 : 2) kcs_init(KArgs<T> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    BicgState &st = a.st[r];
    int i0, j0, k0, k1;
    stage_tile(a.cmap, i0, j0);
    stage_range(a.g, k0, k1);
    const size_t off = (size_t)r * a.stride;
    const C2<T> *b = a.b + off;
    C2<T> *R = a.r + off, *RT = a.rt + off;
    double u[2] = {0.0, 0.0};
    stage_march(stage_smem<T>(), a.g, a.x0 + off, a.sigma, a.gd ? a.gdn : nullptr, b, stage_wmu(a, r), i0, j0, k0,
                k1, [&](int, int e, bool in, C2<T> ax, C2<T>, C2<T> bb) {
                    C2<T> res = mk<T>(0, 0);
                    if (in) {
                        res = csub(bb, ax);
                        u[0] += (double)bb.x * bb.x + (double)bb.y * bb.y;
                        u[1] += (double)res.x * res.x + (double)res.y * res.y;
                    }
                    R[e] = res;
                    RT[e] = res;
                });
    double v[2] = {u[0], u[1]};
    double tot[2];
    if (block_reduce_last<2>(v, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0)
        fin_init(st, tot, a.rerr + (size_t)r * a.rerr_stride, a.maxit, a.inner ? a.ost[r].tol_inner : a.ost[r].tol);
}

// v = A ph ; rtv = rt . v ; alpha = rho / rtv   (which = 0)
// t = A sh ; ts = t . s, tt = t . t ; omega     (which = 1)
template <typename T> __global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 4 : 2) kcs_vt(KArgs<T> a, int which)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    if (a.sweeps && threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.z == 0) atomicAdd(a.sweeps, 1ULL);
    int i0, j0, k0, k1;
    stage_tile(a.cmap, i0, j0);
    stage_range(a.g, k0, k1);
    const size_t off = (size_t)r * a.stride;
    const C2<T> *in = (which ? a.sh : a.ph) + off;
    const C2<T> *w = (which ? a.s : a.rt) + off;
    C2<T> *out = (which ? a.t : a.v) + off;
    // partial sums in double: the Krylov scalars of a converging iteration are
    // small differences of large sums, which FP32 sums lose at large grids
    double u[3] = {0.0, 0.0, 0.0};
    stage_march(stage_smem<T>(), a.g, in, a.sigma, a.gd ? a.gdn : nullptr, w, stage_wmu(a, r), i0, j0, k0, k1,
                [&](int, int e, bool inn, C2<T> y, C2<T>, C2<T> q) {
                    if (inn) {
                        if (which == 0) {
                            u[0] += (double)q.x * y.x + (double)q.y * y.y;  // conj(rt) v
                            u[1] += (double)q.x * y.y - (double)q.y * y.x;
                        } else {
                            u[0] += (double)y.x * q.x + (double)y.y * q.y;  // conj(t) s
                            u[1] += (double)y.x * q.y - (double)y.y * q.x;
                            u[2] += (double)y.x * y.x + (double)y.y * y.y;
                        }
                    }
                    out[e] = y;
                });
    double tot[3];
    if (block_reduce_last<3>(u, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0) {
        if (which == 0) fin_v(st, tot);
        else fin_t(st, tot);
    }
}

// true FP64 residual r = b - A X (refinement loop); |r|^2 -> relres, scale
__global__ void __launch_bounds__(kThreads) kcs_res64(KArgs<double> a)
{
    const int r = blockIdx.y;
    OuterState &os = a.ost[r];
    if (!os.active) return;
    int i0, j0, k0, k1;
    stage_tile(a.cmap, i0, j0);
    stage_range(a.g, k0, k1);
    const size_t off = (size_t)r * a.stride;
    const double2 *b = a.b + off;
    double2 *R = a.r + off;
    double v[1] = {0.0};
    stage_march(stage_smem<double>(), a.g, a.x0 + off, a.sigma, a.gd ? a.gdn : nullptr, b, stage_wmu(a, r), i0, j0,
                k0, k1, [&](int, int e, bool in, double2 ax, double2, double2 bb) {
                    double2 res = make_double2(0, 0);
                    if (in) {
                        res = csub(bb, ax);
                        v[0] += res.x * res.x + res.y * res.y;
                    }
                    R[e] = res;
                });
    double tot[1];
    if (block_reduce_last<1>(v, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0)
        fin_res64(os, tot);
}

// ---------------------------------------------------------------------------
// launch configuration
// ---------------------------------------------------------------------------
constexpr int kMaxDev = 64;

// opt a kernel into its dynamic shared memory once per device and return the
// number of blocks resident per SM
template <typename K> static int stage_setup(K kern, size_t smem, int slot)
{
    static std::mutex mu;
    static int occ[kMaxDev][8] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) dev = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (!occ[dev][slot]) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, kThreads, smem);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        occ[dev][slot] = std::max(1, n) * std::max(1, sms);
    }
    return occ[dev][slot];
}

// chunks of node planes: the count that minimises (waves of resident blocks)
// x (planes per chunk + the 3 planes of the prologue), chunks >= 8 planes.
// Sized for one right-hand side: the blocks of right-hand sides that have
// converged exit at once, and the last one left must still fill the GPU.
int stage_chunks(int nz, int tiles, int resident)
{
    const int planes = nz + 1;
    const long per = tiles;
    int best = 1;
    double best_t = 1e300;
    for (int c = 1; c <= std::max(1, planes / 8); c++) {
        const long waves = (per * c + resident - 1) / resident;
        const int len = (planes + c - 1) / c;
        const double t = (double)waves * (len + 3);
        if (t < best_t - 1e-9) { best_t = t; best = c; }
    }
    return best;
}

template <typename T> static dim3 stage_grid(const KArgs<T> &a, int nrhs, int resident)
{
    return dim3(a.cmap.tiles, nrhs, stage_chunks(a.g.nz, a.cmap.tiles, resident));
}

template <typename T> void launch_stage_init(const KArgs<T> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    const size_t sm = sizeof(StageSmem<T>);
    const int res = stage_setup(kcs_init<T>, sm, sizeof(T) == 8 ? 0 : 1);
    kcs_init<T><<<stage_grid(a, nrhs, res), kThreads, sm, s>>>(a);
}
template <typename T> void launch_stage_vt(const KArgs<T> &a, int which, int nrhs, cudaStream_t s)
{
    counted(1);
    const size_t sm = sizeof(StageSmem<T>);
    const int res = stage_setup(kcs_vt<T>, sm, sizeof(T) == 8 ? 2 : 3);
    kcs_vt<T><<<stage_grid(a, nrhs, res), kThreads, sm, s>>>(a, which);
}
void launch_stage_res64(const KArgs<double> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    const size_t sm = sizeof(StageSmem<double>);
    const int res = stage_setup(kcs_res64, sm, 4);
    kcs_res64<<<stage_grid(a, nrhs, res), kThreads, sm, s>>>(a);
}

template void launch_stage_init<double>(const KArgs<double> &, int, cudaStream_t);
template void launch_stage_init<float>(const KArgs<float> &, int, cudaStream_t);
template void launch_stage_vt<double>(const KArgs<double> &, int, int, cudaStream_t);
template void launch_stage_vt<float>(const KArgs<float> &, int, int, cudaStream_t);

}  // namespace mt3d

// tma.cuh -- shared pieces of the TMA-staged FP32 stencil kernels
// (tmakernels.cu, hatkernels.cu): tensor maps, tile and ring geometry, the
// shared-memory ring, mbarrier and tensor-copy wrappers, and the grad-div
// node potential formed from the staged planes.
//
// A block owns kTX x kTY node columns of one right-hand side and marches a
// chunk of node planes.  Per plane one thread issues the tensor copies of the
// fields (Ex, Ey, Ez over i0-2 .. i0+33, j0-1 .. j0+8: box 72 floats x 10 rows
// x 3 components), sigma (i0-4 .. i0+35, j0-1 .. j0+8) and the signed node
// weights (i0 .. i0+35, j0 .. j0+8) into rings in shared memory, completed on
// an mbarrier per field slot.  The x coordinates are the tile origin rounded
// down to a 16-byte boundary, as tensor copies require; coordinates outside a
// tensor read zeros.  No copy uses cluster multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "colstencil.cuh"
#include "kernels.h"

namespace mt3d {

struct TmaMaps {
    CUtensorMap x0, ph, sh;  // input vectors [nrhs][3][Pz][Py][2 Px] (float)
    CUtensorMap pw, sw;      // the polynomial preconditioner's intermediates (vectors p, s)
    CUtensorMap sig;         // sigma [3][Pz][Py][Px] (float)
    CUtensorMap node;        // signed node weights [Pz][Py][Px] (float)
    int ok;
};
struct alignas(64) TmaParams {
    CUtensorMap in, sig, node;
};

constexpr int kTX = 32, kTY = 8;
constexpr int kFW = 36;   // field tile columns (float2): i0-2 .. i0+33
constexpr int kSW = 40;   // sigma tile columns: i0-4 .. i0+35
constexpr int kNW = 36;   // node tile columns: i0 .. i0+35
constexpr int kFR = 10;   // field / sigma rows: j0-1 .. j0+8
constexpr int kNR = 9;    // node rows: j0 .. j0+8
constexpr int kPhX = kTX + 1, kPhN = (kTX + 1) * (kTY + 1);
constexpr unsigned kFBytes = 3 * kFR * kFW * 8;  // 8640
constexpr unsigned kSBytes = 3 * kFR * kSW * 4;  // 4800
constexpr unsigned kNBytes = kNR * kNW * 4;      // 1296
// ring slots, 128-byte aligned: the fields of four planes (k-1, k, k+1 in use,
// k+2 in flight), sigma of three (k, k+1, k+2) and the node weights of two
// (k+1, k+2), so that four blocks fit on an SM
constexpr unsigned kFSlot = 8704, kSSlot = 4864, kNSlot = 1408;
constexpr int kWaitLimit = 1 << 22;
constexpr int kMaxMultiGrids = 8;  // grids of one multi-grid batch
static_assert(kTX * kTY == kThreads, "one thread per node column");
static_assert(kFSlot % 128 == 0 && kSSlot % 128 == 0 && kNSlot % 128 == 0, "tensor-copy destinations 128-byte aligned");
static_assert(kFSlot >= kFBytes && kSSlot >= kSBytes && kNSlot >= kNBytes, "slot sizes");

struct TmaSmem {
    alignas(128) unsigned char fld[4][kFSlot];
    alignas(128) unsigned char sig[3][kSSlot];
    alignas(128) unsigned char nod[2][kNSlot];
    float2 phi[2][kPhN];
    unsigned long long mbar[4];
};
__device__ __forceinline__ int mod3(int p) { return ((p % 3) + 3) % 3; }

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned a, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned a, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned a, unsigned parity)
{
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    return done != 0;
}
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity, int limit)
{
    for (int it = 0; it < limit; it++)
        if (mbar_try(a, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap *m, int c0, int c1, int c2, int c3,
                                          unsigned mb)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mb)
        : "memory");
}
__device__ __forceinline__ void tma_load3(unsigned dst, const CUtensorMap *m, int c0, int c1, int c2, unsigned mb)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];\n" ::"r"(dst),
        "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(mb)
        : "memory");
}

// grad-div potential of node (ni, nj) of the tile (global i, j) at plane p:
// the sums of k_gd_phi (mode 0) in the same order, from the staged planes
__device__ __forceinline__ float2 tma_phi_node(const TmaSmem &sm, const Geo<float> &g, int i, int j, int p, int ni,
                                               int nj, float dX, float dY, float dZ)
{
    if (!(i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1 && p >= 1 && p <= g.nz - 1)) return make_float2(0, 0);
    const int sp = p & 3, sz = (p - 1) & 3;
    const float2 *F = reinterpret_cast<const float2 *>(sm.fld[sp]);
    const float2 *Fz = reinterpret_cast<const float2 *>(sm.fld[sz]) + 2 * kFR * kFW;
    const float *S = reinterpret_cast<const float *>(sm.sig[p % 3]);
    const float *Sz = reinterpret_cast<const float *>(sm.sig[(p - 1) % 3]) + 2 * kFR * kSW;
    const float wn = reinterpret_cast<const float *>(sm.nod[p & 1])[nj * kNW + ni];
    const int h = (nj + 1) * kFW + ni + 2, hs = (nj + 1) * kSW + ni + 4;
    const int cf = kFR * kFW, cs = kFR * kSW;
    const float dfa0 = dY * dZ, dfa1 = dX * dZ, dfa2 = dX * dY;
    float2 acc;
    if (wn < 0.f) {  // earth node: C = sigma_E
        acc = cscale(F[h - 1], dfa0 * S[hs - 1]);                       // Ex(i-1, j, p)
        acc = csub(acc, cscale(F[h], dfa0 * S[hs]));                     // Ex(i, j, p)
        acc = cadd(acc, cscale(F[cf + h - kFW], dfa1 * S[cs + hs - kSW]));  // Ey(i, j-1, p)
        acc = csub(acc, cscale(F[cf + h], dfa1 * S[cs + hs]));           // Ey(i, j, p)
        acc = cadd(acc, cscale(Fz[h], dfa2 * Sz[hs]));                   // Ez(i, j, p-1)
        acc = csub(acc, cscale(F[2 * cf + h], dfa2 * S[2 * cs + hs]));   // Ez(i, j, p)
        return cscale(acc, -wn);
    }
    acc = cscale(F[h - 1], dfa0);
    acc = csub(acc, cscale(F[h], dfa0));
    acc = cadd(acc, cscale(F[cf + h - kFW], dfa1));
    acc = csub(acc, cscale(F[cf + h], dfa1));
    acc = cadd(acc, cscale(Fz[h], dfa2));
    acc = csub(acc, cscale(F[2 * cf + h], dfa2));
    return cscale(acc, wn);
}

// tile (i0, j0) of column-tile bx, and node planes [k0, k1) of chunk bz of gz
__device__ __forceinline__ void tma_tile_at(const ColMap &m, int bx, int &i0, int &j0)
{
    i0 = (bx % m.tiles_x) * kTX;
    j0 = (bx / m.tiles_x) * kTY;
}
__device__ __forceinline__ void tma_range_at(int nz, int bz, int gz, int &k0, int &k1)
{
    const int kc = (nz + 1 + gz - 1) / gz;
    k0 = bz * kc;
    k1 = min(k0 + kc, nz + 1);
}
__device__ __forceinline__ void tma_tile(const ColMap &m, int &i0, int &j0) { tma_tile_at(m, blockIdx.x, i0, j0); }
__device__ __forceinline__ void tma_range(int nz, int &k0, int &k1) { tma_range_at(nz, blockIdx.z, gridDim.z, k0, k1); }
__device__ __forceinline__ TmaSmem &tma_smem()
{
    extern __shared__ __align__(128) unsigned char tma_raw[];
    return *reinterpret_cast<TmaSmem *>(tma_raw);
}

// the chunk count of stagekernels.cu, for the resident blocks of these
// kernels; `slot` identifies the kernel (its shared-memory attribute is set
// the first time its slot is seen), so every kernel needs its own slot
constexpr int kTmaSlots = 24;
// the fused stencil of hatkernels.cu: 128 threads, each on two node rows
// (ty and ty + 4) of the 32 x 8 tile
constexpr int kHatThreads = 128, kHatRows = kTY / 2;
static_assert(kHatThreads == kTX * kHatRows, "fused stencil thread layout");
template <typename K> inline int tma_resident(K kern, size_t smem, int slot, int threads = kThreads)
{
    static std::mutex mu;
    static int occ[64][kTmaSlots] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (!occ[dev][slot]) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        int n = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        occ[dev][slot] = std::max(1, n) * std::max(1, sms);
    }
    return occ[dev][slot];
}

}  // namespace mt3d

// noalloc.cu -- y = A x on caller-owned device vectors with no device
// allocation: the operator product of mt3d_mult_aii whose scratch (the two
// full-edge vectors, the grad-div node potentials and the per-call state)
// lives in one fixed, file-scope device array instead of the handle's
// workspace.
//
// The scratch is one array per device, shared by every handle on that
// device.  Its address is looked up once per device (cudaGetSymbolAddress,
// with that device current) when mt3d_create makes the first handle there:
// under CUDA's lazy module loading that look-up is what commits the array's
// 16 MiB, and the kernels this entry launches are loaded at the same time, so
// the entry itself takes no device memory, on its first call or later.  Two
// calls whose GPU work overlaps in time on one device (different streams,
// handles or host threads) use the same scratch and race; calls enqueued on
// one stream run one after the other and are safe.
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "solver.h"

namespace mt3d {

// 16 MiB: the state record plus (2 nE + nN) complex doubles, enough for
// grids up to about 52^3 cells (nE ~ 3 n^3, nN ~ n^3)
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr size_t kNoAllocStateBytes = 256;
static_assert(sizeof(OuterState) <= kNoAllocStateBytes, "state record does not fit its slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mutex;
static void *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// device address of the scratch on the current device (set-up on first use)
static int noalloc_scratch(int dev, void **ptr, std::string &err)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        err = "device ordinal out of range for the fixed scratch table";
        return 5;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            err = std::string("cudaGetSymbolAddress of the fixed scratch failed: ") + cudaGetErrorString(e);
            return 4;
        }
        g_noalloc_ptr[dev] = p;
    }
    *ptr = g_noalloc_ptr[dev];
    return 0;
}

// the per-call state record: all fields zero except omega and active
__global__ void k_noalloc_state(OuterState *st, double omega)
{
    OuterState s{};
    s.omega = omega;
    s.active = 1;
    *st = s;
}

// set-up at handle creation, with device `dev` current: the scratch address
// (committing the array) and the kernels of the entry (loading their modules)
int noalloc_prepare(int dev, std::string &err)
{
    void *p = nullptr;
    int rc = noalloc_scratch(dev, &p, err);
    if (rc) return rc;
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_noalloc_state);
    if (e == cudaSuccess) e = preload_apply_kernels();
    if (e != cudaSuccess) {
        cudaGetLastError();
        err = std::string("loading the operator kernels failed: ") + cudaGetErrorString(e);
        return 4;
    }
    return 0;
}

extern std::atomic<long long> g_launch_count;

static bool device_vector(const void *p, int dev)
{
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) return false;
    return at.type == cudaMemoryTypeManaged || at.device == dev;
}

int Solver::mult_aii_noalloc(int adjt, const double *x, double *y)
{
    const char *who = "mt3d_mult_aii_device_noalloc";
    if (!cond_set) return fail(5, std::string(who) + ": conductivity not set (call mt3d_update_cond)");
    if (!(omega > 0)) return fail(5, std::string(who) + ": frequency not set (call mt3d_update_freq)");
    if (!x || !y) return fail(5, std::string(who) + ": null vector");
    if ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15)
        return fail(5, std::string(who) + ": x and y must be 16-byte aligned");
    if (!device_vector(x, dev_) || !device_vector(y, dev_))
        return fail(5, std::string(who) + ": x and y must be device memory of the handle's device");
    const bool gd = ctl.formulation == 1;
    const size_t need = kNoAllocStateBytes + sizeof(double2) * (size_t)(2 * nE + (gd ? nN : 0));
    if (need > kNoAllocScratchBytes) {
        char buf[256];
        snprintf(buf, sizeof buf,
                 "%s: this grid needs %zu bytes of scratch, more than the fixed %zu-byte scratch (at most about "
                 "52^3 cells); use mt3d_mult_aii",
                 who, need, kNoAllocScratchBytes);
        return fail(5, buf);
    }
    void *base = nullptr;
    std::string err;
    int rc = noalloc_scratch(dev_, &base, err);
    if (rc) return fail(rc, std::string(who) + ": " + err);
    unsigned char *p = static_cast<unsigned char *>(base);
    OuterState *st = reinterpret_cast<OuterState *>(p);
    double2 *xf = reinterpret_cast<double2 *>(p + kNoAllocStateBytes);
    double2 *yf = xf + nE;
    double2 *phi = gd ? yf + nE : nullptr;
    // the boundary edges of xf must read as zero (the scatter writes only the
    // interior); yf and phi are written in full by their kernels
    if ((rc = check(cudaMemsetAsync(xf, 0, nE * sizeof(double2), stream_), who))) return rc;
    k_noalloc_state<<<1, 1, 0, stream_>>>(st, omega);
    g_launch_count.fetch_add(1, std::memory_order_relaxed);
    launch_scatter_interior((int)nEi, edgei_d_.as<int>(), reinterpret_cast<const double2 *>(x), xf, stream_);
    KArgs<double> a = kargs<double>(1, 0);
    a.ost = st;
    a.phi = phi;
    a.dsgn = adjt ? 1.0 : -1.0;
    launch_apply(a, xf, yf, 0, 1, stream_, gd ? (adjt ? 2 : 1) : 0);
    launch_gather_interior((int)nEi, edgei_d_.as<int>(), yf, reinterpret_cast<double2 *>(y), stream_);
    return check(cudaGetLastError(), who);
}

}  // namespace mt3d

// solver.cu -- host driver of the B200 3D-MT solve: operator set-up, the
// divergence-corrected Krylov loop of FWDsolve3D and the mixed-precision
// refinement.  Everything numeric runs in the kernels of kernels.cu; this
// file sequences launches on the handle's stream and reads back only the
// per-right-hand-side scalar state once per outer (divergence-correction)
// cycle.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>

#include "solver.h"

namespace mt3d {

std::atomic<long long> g_alloc_count{0};

int DevBuf::alloc(size_t bytes)
{
    if (bytes <= bytes_ && ptr_) return 0;
    release();
    if (bytes == 0) return 0;
    g_alloc_count.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaMalloc(&ptr_, bytes);
    if (e != cudaSuccess) {
        ptr_ = nullptr;
        return (int)e;
    }
    bytes_ = bytes;
    return 0;
}
void DevBuf::release()
{
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
}

Solver::~Solver()
{
    cudaSetDevice(dev_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (tma_) tma_maps_free(tma_);
    for (cudaEvent_t e : ev_) cudaEventDestroy(e);
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

int Solver::set_stream(void *s)
{
    if (stream_) cudaStreamSynchronize(stream_);
    stream_ = s ? (cudaStream_t)s : own_stream_;
    return 0;
}

int Solver::set_fused(int on)
{
    ctl.fused = on != 0;
    return 0;
}

int Solver::set_wait_limit(int polls)
{
    if (polls < 0) return fail(5, "mt3d_set_wait_limit: the limit must not be negative");
    wait_limit_ = polls;
    return 0;
}

int Solver::profile(int enable)
{
    if (stream_) cudaStreamSynchronize(stream_);
    prof_ = enable != 0;
    prof_launches_[0] = prof_launches_[1] = 0;
    prof_ms_[0] = prof_ms_[1] = 0.0;
    ev_used_ = 0;
    if (prof_) {
        if (prof_cnt_.alloc(2 * sizeof(unsigned long long))) return fail(8, "mt3d_profile: out of device memory");
        if (int rc = check(cudaMemset(prof_cnt_.as<void>(), 0, 2 * sizeof(unsigned long long)), "mt3d_profile"))
            return rc;
    }
    return 0;
}

cudaEvent_t *Solver::next_events(int n)
{
    if (!prof_) return nullptr;
    while (ev_.size() < ev_used_ + n) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        ev_.push_back(e);
    }
    ev_prec_.resize(ev_.size());
    for (int q = 0; q < n; q++) ev_prec_[ev_used_ + q] = prof_cur_;
    cudaEvent_t *p = &ev_[ev_used_];
    ev_used_ += n;
    return p;
}

// sum the elapsed time of the recorded (start, stop) pairs per precision; the
// stream must have been synchronised
void Solver::collect_events()
{
    for (size_t i = 0; i + 1 < ev_used_; i += 2) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ev_[i], ev_[i + 1]) == cudaSuccess) {
            prof_ms_[ev_prec_[i] ? 1 : 0] += ms;
            prof_launches_[ev_prec_[i] ? 1 : 0] += 1;
        } else {
            cudaGetLastError();
        }
    }
    ev_used_ = 0;
}

int Solver::kernel_time(int precision, int *launches, double *ms, int64_t *sweeps)
{
    if (precision != 0 && precision != 1) return fail(5, "mt3d_kernel_time: precision must be 0 or 1");
    if (stream_) cudaStreamSynchronize(stream_);
    collect_events();
    if (launches) *launches = prof_launches_[precision];
    if (ms) *ms = prof_ms_[precision];
    if (sweeps) {
        unsigned long long c[2] = {0, 0};
        if (prof_cnt_.bytes() >= sizeof c &&
            cudaMemcpy(c, prof_cnt_.as<void>(), sizeof c, cudaMemcpyDeviceToHost) != cudaSuccess)
            cudaGetLastError();
        *sweeps = (int64_t)c[precision];
    }
    return 0;
}

int Solver::fail(int code, const std::string &msg)
{
    last_error = msg;
    return code;
}

int Solver::check(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return 0;
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    last_error = buf;
    return e == cudaErrorMemoryAllocation ? 8 : 4;
}

int Solver::sync(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    return check(e, what);
}

static void deltas(const std::vector<double> &d, std::vector<double> &del)
{
    const size_t n = d.size();
    del.assign(n + 1, 0.0);
    del[0] = d[0];
    for (size_t i = 1; i < n; i++) del[i] = d[i - 1] + d[i];
    del[n] = d[n - 1];
    for (auto &v : del) v = v / 2.0;
}

int Solver::create(int dev, int nx_, int ny_, int nz_, int nzAir_, const double *dx, const double *dy, const double *dz)
{
    if (nx_ < 2 || ny_ < 2 || nz_ < 2 || nzAir_ < 0 || nzAir_ >= nz_ || !dx || !dy || !dz)
        return fail(5, "mt3d_create: invalid grid dimensions or null spacing arrays");
    nx = nx_; ny = ny_; nz = nz_; nzAir = nzAir_;
    const int64_t nX = (int64_t)nx * (ny + 1) * (nz + 1), nY = (int64_t)(nx + 1) * ny * (nz + 1),
                  nZ = (int64_t)(nx + 1) * (ny + 1) * nz;
    nE = nX + nY + nZ;
    nN = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    nEi = (int64_t)nx * (ny - 1) * (nz - 1) + (int64_t)(nx - 1) * ny * (nz - 1) + (int64_t)(nx - 1) * (ny - 1) * nz;
    if (nE >= (int64_t)1 << 31) return fail(5, "mt3d_create: grid too large (edge count must fit in int32)");
    for (int i = 0; i < nx; i++) if (!(dx[i] > 0)) return fail(5, "mt3d_create: dx must be positive");
    for (int i = 0; i < ny; i++) if (!(dy[i] > 0)) return fail(5, "mt3d_create: dy must be positive");
    for (int i = 0; i < nz; i++) if (!(dz[i] > 0)) return fail(5, "mt3d_create: dz must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(7, "mt3d_create: no CUDA device available");
    }
    if (dev < 0 || dev >= ndev) return fail(5, "mt3d_create: device id out of range");
    dev_ = dev;
    int rc;
    if ((rc = check(cudaSetDevice(dev_), "cudaSetDevice"))) return rc;
    // a blocking stream: ordered with the legacy default stream, so device
    // buffers a caller fills there (stream handle 0, as torch's default
    // stream reports itself, which mt3d_set_stream also reads as "the
    // handle's own stream") are complete before the handle's work reads them
    if ((rc = check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamDefault), "cudaStreamCreate"))) return rc;
    stream_ = own_stream_;

    pl_.Px = (nx + 1 + 3) / 4 * 4;
    pl_.Py = ny + 1;
    pl_.Pz = nz + 1;
    if (errf_.alloc(sizeof(int))) return fail(8, "mt3d_create: out of device memory");
    cudaMemset(errf_.as<void>(), 0, sizeof(int));
    dx_.assign(dx, dx + nx); dy_.assign(dy, dy + ny); dz_.assign(dz, dz + nz);
    deltas(dx_, delX_); deltas(dy_, delY_); deltas(dz_, delZ_);
    // tables: dx dy dz delX delY delZ rdx rdy rdz
    std::vector<double> t;
    auto app = [&](const std::vector<double> &v) { t.insert(t.end(), v.begin(), v.end()); };
    std::vector<double> rdx(nx), rdy(ny), rdz(nz);
    for (int i = 0; i < nx; i++) rdx[i] = 1.0 / dx_[i];
    for (int i = 0; i < ny; i++) rdy[i] = 1.0 / dy_[i];
    for (int i = 0; i < nz; i++) rdz[i] = 1.0 / dz_[i];
    app(dx_); app(dy_); app(dz_); app(delX_); app(delY_); app(delZ_); app(rdx); app(rdy); app(rdz);
    std::vector<float> tf(t.begin(), t.end());
    if (tab64_.alloc(t.size() * sizeof(double)) || tab32_.alloc(tf.size() * sizeof(float)))
        return fail(8, "mt3d_create: out of device memory");
    if ((rc = check(cudaMemcpy(tab64_.as<void>(), t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice), "copy tables")))
        return rc;
    if ((rc = check(cudaMemcpy(tab32_.as<void>(), tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice), "copy tables")))
        return rc;
    size_t o[10];
    o[0] = 0; o[1] = o[0] + nx; o[2] = o[1] + ny; o[3] = o[2] + nz; o[4] = o[3] + nx + 1; o[5] = o[4] + ny + 1;
    o[6] = o[5] + nz + 1; o[7] = o[6] + nx; o[8] = o[7] + ny; o[9] = o[8] + nz;
    auto fill = [&](auto &g, auto *base) {
        g.nx = nx; g.ny = ny; g.nz = nz; g.nzAir = nzAir;
        g.nXe = (int)nX; g.nYe = (int)nY; g.nZe = (int)nZ; g.nE = (int)nE; g.nN = (int)nN;
        g.dx = base + o[0]; g.dy = base + o[1]; g.dz = base + o[2];
        g.delX = base + o[3]; g.delY = base + o[4]; g.delZ = base + o[5];
        g.rdx = base + o[6]; g.rdy = base + o[7]; g.rdz = base + o[8];
    };
    fill(g64_, tab64_.as<double>());
    fill(g32_, tab32_.as<float>());

    // interior edge list (boundaryIndex, vecTranslate.f90:436-526), 0-based
    edgei.clear();
    edgei.reserve(nEi);
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i < nx; i++)
                if (j >= 1 && j <= ny - 1 && k >= 1 && k <= nz - 1) edgei.push_back(i + nx * (j + (ny + 1) * k));
    for (int k = 0; k <= nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i <= nx; i++)
                if (i >= 1 && i <= nx - 1 && k >= 1 && k <= nz - 1)
                    edgei.push_back((int)nX + i + (nx + 1) * (j + ny * k));
    for (int k = 0; k < nz; k++)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i <= nx; i++)
                if (i >= 1 && i <= nx - 1 && j >= 1 && j <= ny - 1)
                    edgei.push_back((int)(nX + nY) + i + (nx + 1) * (j + (ny + 1) * k));
    if ((int64_t)edgei.size() != nEi) return fail(5, "internal: interior edge count mismatch");
    if (edgei_d_.alloc(edgei.size() * sizeof(int32_t))) return fail(8, "mt3d_create: out of device memory");
    if ((rc = check(cudaMemcpy(edgei_d_.as<void>(), edgei.data(), edgei.size() * sizeof(int32_t), cudaMemcpyHostToDevice),
                    "copy edge list")))
        return rc;
    std::string err;
    if ((rc = noalloc_prepare(dev_, err))) return fail(rc, "mt3d_create: " + err);
    return 0;
}

// ---------------------------------------------------------------------------
// UpdateCond: ModelParamToEdge (LOGE, f90/3D_MT/modelParam/ModelMap.inc:88-188),
// the SP2 edge and node data (f90/3D_MT/FWD_SP2/modelOperator3D.f90:176-230,
// 916-1008, 1086-1130) and DivCorrSetUp (f90/3D_MT/FWD/modelOperator3D.f90:
// 1538-1672), built on the device from the model parameter
// ---------------------------------------------------------------------------
int Solver::update_cond(const double *m_earth, double airCond)
{
    if (!m_earth) return fail(5, "mt3d_update_cond: null model");
    const int64_t nEarth = (int64_t)nx * ny * (nz - nzAir), nC = (int64_t)nx * ny * nz;
    for (int64_t c = 0; c < nEarth; c++)
        if (!std::isfinite(m_earth[c])) return fail(3, "mt3d_update_cond: NaN/Inf in the model parameter");
    if (!std::isfinite(airCond)) return fail(3, "mt3d_update_cond: NaN/Inf air conductivity");
    int rc;
    if (sig64_.alloc(nE * sizeof(double)) || sig32_.alloc(nE * sizeof(float)) || coef_.alloc(7 * nN * sizeof(double)) ||
        sigs64_.alloc(nE * sizeof(double)) || sigs32_.alloc(nE * sizeof(float)) || gdw64_.alloc(nN * sizeof(double)) ||
        gdw32_.alloc(nN * sizeof(float)) || gde_.alloc(nN) || gdn64_.alloc(nN * sizeof(double)) ||
        gdn32_.alloc(nN * sizeof(float)) || setup_.alloc((nEarth + 3 * nC) * sizeof(double)))
        return fail(8, "mt3d_update_cond: out of device memory");
    double *m_d = setup_.as<double>(), *VC = m_d + nEarth, *CT = VC + nC, *sigC = CT + nC;
    if ((rc = check(cudaMemcpyAsync(m_d, m_earth, nEarth * sizeof(double), cudaMemcpyHostToDevice, stream_),
                    "copy model parameter")))
        return rc;
    launch_setup_cond(g64_, m_d, airCond, VC, CT, sigC, sig64_.as<double>(), sigs64_.as<double>(), gdw64_.as<double>(),
                      gde_.as<unsigned char>(), gdn64_.as<double>(), coef_.as<double>(), sig32_.as<float>(),
                      sigs32_.as<float>(), gdw32_.as<float>(), gdn32_.as<float>(), stream_);
    // sigma of both formulations and the signed node weights on the padded
    // layout (FP32), for the TMA-staged kernels
    const size_t pe = (size_t)pl_.len(), pn = (size_t)pl_.Px * pl_.Py * pl_.Pz;
    if (sigP32_.alloc(pe * sizeof(float)) || sigsP32_.alloc(pe * sizeof(float)) || gdnP32_.alloc(pn * sizeof(float)))
        return fail(8, "mt3d_update_cond: out of device memory");
    cudaMemsetAsync(sigP32_.as<void>(), 0, pe * sizeof(float), stream_);
    cudaMemsetAsync(sigsP32_.as<void>(), 0, pe * sizeof(float), stream_);
    cudaMemsetAsync(gdnP32_.as<void>(), 0, pn * sizeof(float), stream_);
    launch_to_padded(g64_, sig64_.as<double>(), pl_, sigP32_.as<float>(), stream_);
    launch_to_padded(g64_, sigs64_.as<double>(), pl_, sigsP32_.as<float>(), stream_);
    launch_nodes_to_padded(g64_, gdn64_.as<double>(), pl_, gdnP32_.as<float>(), stream_);
    tma_stale_ = true;
    if ((rc = sync("mt3d_update_cond"))) return rc;
    cond_set = true;
    return 0;
}

int Solver::get_cond(double *sigma_e, double *divcorr, double *node_w)
{
    if (!cond_set) return fail(5, "mt3d_get_cond: conductivity not set (call mt3d_update_cond)");
    int rc;
    if (sigma_e && (rc = check(cudaMemcpyAsync(sigma_e, sig64_.as<void>(), nE * sizeof(double), cudaMemcpyDeviceToHost,
                                               stream_), "copy sigma")))
        return rc;
    if (divcorr && (rc = check(cudaMemcpyAsync(divcorr, coef_.as<void>(), 7 * nN * sizeof(double),
                                               cudaMemcpyDeviceToHost, stream_), "copy div-corr coefficients")))
        return rc;
    if (node_w && (rc = check(cudaMemcpyAsync(node_w, gdn64_.as<void>(), nN * sizeof(double), cudaMemcpyDeviceToHost,
                                              stream_), "copy node weights")))
        return rc;
    return sync("mt3d_get_cond");
}

// tensor maps of the padded FP32 vectors, rebuilt after the workspace or the
// conductivity changed
int Solver::tma_ready()
{
    if (!tma_stale_) return 0;
    if (!tma_) tma_ = tma_maps_new();
    Workspace &w = ws_;
    if (tma_maps_build(tma_, w.f_x0.as<float2>(), w.f_ph.as<float2>(), w.f_sh.as<float2>(), w.f_p.as<float2>(),
                       w.f_s.as<float2>(),
                       (ctl.formulation == 1 ? sigsP32_ : sigP32_).as<float>(), gdnP32_.as<float>(), pl_, w.nrhs))
        return fail(4, "cuTensorMapEncodeTiled failed for the padded FP32 vectors");
    tma_stale_ = false;
    return 0;
}

// a bounded device-side wait gave up (MT3D_DEVICE_TIMEOUT)
int Solver::check_device_error(const char *what)
{
    int e = 0;
    cudaMemcpy(&e, errf_.as<void>(), sizeof(int), cudaMemcpyDeviceToHost);
    if (!e) return 0;
    cudaMemset(errf_.as<void>(), 0, sizeof(int));
    // the blocks that gave up skipped their reductions: clear the counters
    // of the last-block detection for the next call
    if (ws_.cnt.bytes()) cudaMemset(ws_.cnt.as<void>(), 0, ws_.cnt.bytes());
    return fail(6, std::string(what) + ": a bounded device-side wait gave up");
}

int Solver::update_freq(double w)
{
    if (!(w > 0.0) || !std::isfinite(w)) return fail(5, "mt3d_update_freq: omega must be positive and finite");
    omega = w;
    return 0;
}

// ---------------------------------------------------------------------------
// workspace and argument blocks
// ---------------------------------------------------------------------------
static int blocks_for(int64_t n, int &chunk)
{
    // contiguous chunks of >= 4 sweeps of the block; about 8 resident blocks
    // per SM for ONE right-hand side: the right-hand sides of a batch converge
    // at different iterations, the blocks of finished ones exit at once, and
    // the grid must still fill the GPU when a single right-hand side is left
    const int64_t target = 148LL * 8;
    int64_t per = (n + target - 1) / target;
    per = std::max<int64_t>(per, 4 * kThreads);
    per = (per + kThreads - 1) / kThreads * kThreads;
    chunk = (int)per;
    return (int)((n + per - 1) / per);
}

// FP64 Krylov vectors in a mixed-precision workspace (allocated when a
// right-hand side first falls back to FP64 cycles; kept with the workspace)
int Solver::ensure_fp64_krylov(int nrhs)
{
    Workspace &w = ws_;
    const size_t e64 = (size_t)nrhs * nE * sizeof(double2);
    if (w.r.bytes() >= e64) return 0;
    DevBuf *v64[] = {&w.x1, &w.r, &w.rt, &w.p, &w.v, &w.ph, &w.s, &w.sh, &w.t, &w.jinv64, &w.zm, &w.zc};
    int err = 0;
    for (int q = 0; q < 9; q++) err |= v64[q]->alloc(e64);
    if (ctl.solver == 1) err |= w.jinv64.alloc(e64);
    if (ctl.solver == 3) err |= w.zm.alloc(e64) | w.zc.alloc(e64);
    if (err) {
        for (DevBuf *d : v64) d->release();
        cudaGetLastError();
        return fail(8, "out of device memory for the FP64 Krylov vectors");
    }
    return 0;
}

int Solver::ensure_workspace(int nrhs, int precision)
{
    const int rlen = std::max(ctl.IterPerDivCor, 1) + 1, dlen = std::max(ctl.MaxIterDivCor, 1) + 1;
    if (ws_.nrhs >= nrhs && ws_.precision == precision && ws_.rlen == rlen && ws_.dlen == dlen &&
        ws_.solver == ctl.solver && ws_.formulation == ctl.formulation)
        return 0;
    tma_stale_ = true;
    Workspace &w = ws_;
    // FP32 vectors on the padded layout for the TMA-staged BiCGStab + diagonal path
    const bool padded = precision == 1 && ctl.solver == 1;
    const size_t e64 = (size_t)nrhs * nE * sizeof(double2),
                 e32 = (size_t)nrhs * (padded ? (size_t)pl_.len() : (size_t)nE) * sizeof(float2);
    const size_t n64 = (size_t)nrhs * nN * sizeof(double2);
    // release everything first so a precision change does not hold both sets
    DevBuf *all[] = {&w.qst, &w.b, &w.X, &w.x1, &w.r, &w.rt, &w.p, &w.v, &w.ph, &w.s, &w.sh, &w.t, &w.bc, &w.tmp,
                     &w.f_b, &w.f_x0, &w.f_x1, &w.f_r, &w.f_rt, &w.f_p, &w.f_v, &w.f_ph, &w.f_s, &w.f_sh, &w.f_t,
                     &w.px, &w.pr, &w.pp, &w.pq, &w.phi0, &w.zm, &w.zc, &w.f_zm, &w.f_zc, &w.phi64, &w.phi32, &w.jinv64, &w.jinv32};
    for (DevBuf *d : all) d->release();
    int err = 0;
    err |= w.b.alloc(e64) | w.X.alloc(e64) | w.bc.alloc(e64) | w.tmp.alloc(e64);
    if (precision == 0) {
        DevBuf *v64[] = {&w.x1, &w.r, &w.rt, &w.p, &w.v, &w.ph, &w.s, &w.sh, &w.t};
        for (DevBuf *d : v64) err |= d->alloc(e64);
        if (ctl.solver == 3 || ctl.solver == 4) err |= w.zm.alloc(e64) | w.zc.alloc(e64);
        if (ctl.solver == 1) err |= w.jinv64.alloc(e64);
    } else {
        DevBuf *v32[] = {&w.f_b, &w.f_x0, &w.f_x1, &w.f_r, &w.f_rt, &w.f_p, &w.f_v, &w.f_ph, &w.f_s, &w.f_sh, &w.f_t};
        for (DevBuf *d : v32) err |= d->alloc(e32);
        if (ctl.solver == 3) err |= w.f_zm.alloc(e32) | w.f_zc.alloc(e32);
        if (ctl.solver == 1) err |= w.jinv32.alloc(e32);
        if (!err && padded) {  // the padding entries must read as zero
            for (DevBuf *d : v32) cudaMemsetAsync(d->as<void>(), 0, e32, stream_);
            cudaMemsetAsync(w.jinv32.as<void>(), 0, e32, stream_);
        }
    }
    if (ctl.formulation == 0) {
        DevBuf *nv[] = {&w.px, &w.pr, &w.pp, &w.pq, &w.phi0};
        for (DevBuf *d : nv) err |= d->alloc(n64);
    } else {
        err |= w.phi64.alloc(n64);
        if (precision == 1) err |= w.phi32.alloc((size_t)nrhs * nN * sizeof(float2));
    }
    int c;
    const ColMapHost cm = col_map(nx, ny);
    const int nb = std::max({blocks_for(nE, c), blocks_for(nN, c), cm.tiles * std::max(1, (nz + 1) / 8),
                             1184});
    err |= w.bst.alloc(nrhs * sizeof(BicgState)) | w.pst.alloc(nrhs * sizeof(PcgState)) |
           w.ost.alloc(nrhs * sizeof(OuterState)) | w.qst.alloc(nrhs * sizeof(QmrState));
    err |= w.parts.alloc((size_t)nrhs * nb * kMaxParts * sizeof(double)) | w.cnt.alloc(3 * nrhs * sizeof(unsigned));
    err |= w.rerr.alloc((size_t)nrhs * rlen * sizeof(double));
    err |= w.dcrerr.alloc((size_t)nrhs * dlen * sizeof(double));
    if (err) {
        for (DevBuf *d : all) d->release();
        w.nrhs = 0;
        w.precision = -1;
        cudaGetLastError();
        return fail(8, "out of device memory for the solver workspace");
    }
    cudaMemsetAsync(w.cnt.as<void>(), 0, nrhs * sizeof(unsigned), stream_);
    w.nrhs = nrhs;
    w.precision = precision;
    w.rlen = rlen;
    w.dlen = dlen;
    w.solver = ctl.solver;
    w.formulation = ctl.formulation;
    w.padded = padded;
    return 0;
}

template <> KArgs<double> Solver::kargs<double>(int nrhs, int)
{
    KArgs<double> a{};
    Workspace &w = ws_;
    a.sweeps = prof_ ? prof_cnt_.as<unsigned long long>() + 0 : nullptr;
    a.g = g64_;
    a.sigma = sig64_.as<double>();
    a.ost = w.ost.as<OuterState>();
    a.st = w.bst.as<BicgState>();
    a.r = w.r.as<double2>(); a.rt = w.rt.as<double2>(); a.p = w.p.as<double2>(); a.v = w.v.as<double2>();
    a.ph = w.ph.as<double2>(); a.s = w.s.as<double2>(); a.sh = w.sh.as<double2>(); a.t = w.t.as<double2>();
    a.x0 = w.X.as<double2>(); a.x1 = w.x1.as<double2>();
    a.b = w.b.as<double2>();
    a.parts = w.parts.as<double>();
    a.cnt = w.cnt.as<unsigned>();
    a.rerr = w.rerr.as<double>();
    a.rerr_stride = ctl.IterPerDivCor + 1;
    a.stride = nE;
    a.nblk = blocks_for(nE, a.chunk);
    a.len = (int)nE;
    a.err = errf_.as<int>();
    a.maxit = ctl.IterPerDivCor;
    a.inner = 0;
    a.dsgn = -1.0;
    a.colstencil = 2;
    a.cmap = col_map(nx, ny);
    a.jinv = ctl.solver == 1 ? w.jinv64.as<double2>() : nullptr;
    a.qst = w.qst.as<QmrState>();
    a.q = w.zm.as<double2>();
    a.w = w.zc.as<double2>();
    a.d = w.x1.as<double2>();
    if (ctl.formulation == 1) {
        a.sigma = sigs64_.as<double>();
        a.gd = 1;
        a.gdw = gdw64_.as<double>();
        a.gde = gde_.as<unsigned char>();
        a.gdn = gdn64_.as<double>();
        a.phi = w.phi64.as<double2>();
        a.restart = ctl.restart;
    }
    return a;
}
template <> KArgs<float> Solver::kargs<float>(int nrhs, int)
{
    // zeroed as bytes: the captured FP32 cycle is keyed on the bytes of its
    // arguments, padding included
    KArgs<float> a;
    std::memset(&a, 0, sizeof a);
    Workspace &w = ws_;
    a.sweeps = prof_ ? prof_cnt_.as<unsigned long long>() + 1 : nullptr;
    a.g = g32_;
    a.sigma = sig32_.as<float>();
    a.ost = w.ost.as<OuterState>();
    a.st = w.bst.as<BicgState>();
    a.r = w.f_r.as<float2>(); a.rt = w.f_rt.as<float2>(); a.p = w.f_p.as<float2>(); a.v = w.f_v.as<float2>();
    a.ph = w.f_ph.as<float2>(); a.s = w.f_s.as<float2>(); a.sh = w.f_sh.as<float2>(); a.t = w.f_t.as<float2>();
    a.x0 = w.f_x0.as<float2>(); a.x1 = w.f_x1.as<float2>();
    a.b = w.f_b.as<float2>();
    a.parts = w.parts.as<double>();
    a.cnt = w.cnt.as<unsigned>();
    a.rerr = w.rerr.as<double>();
    a.rerr_stride = ctl.IterPerDivCor + 1;
    a.stride = nE;
    a.len = (int)nE;
    a.err = errf_.as<int>();
    a.wait_limit = wait_limit_;
    a.pc = (float)ctl.poly;
    if (w.padded) {
        // padded layout: the elementwise kernels sweep the padded length and
        // the stencil runs on the TMA-staged kernels
        a.padded = 1;
        a.pl = pl_;
        a.len = (int)pl_.len();
        a.stride = (size_t)pl_.len();
        a.tma = tma_;
    }
    a.nblk = blocks_for(a.len, a.chunk);
    a.maxit = ctl.IterPerDivCor;
    a.inner = 1;
    a.dsgn = -1.0;
    a.colstencil = w.padded ? 3 : 2;
    a.cmap = col_map(nx, ny);
    a.jinv = ctl.solver == 1 ? w.jinv32.as<float2>() : nullptr;
    if (ctl.formulation == 1) {
        a.sigma = sigs32_.as<float>();
        a.gd = 1;
        a.gdw = gdw32_.as<float>();
        a.gde = gde_.as<unsigned char>();
        a.gdn = gdn32_.as<float>();
        a.phi = w.phi32.as<float2>();
        a.restart = ctl.restart;
    }
    return a;
}

template <> ColArgs<double> Solver::cargs<double>()
{
    ColArgs<double> a{};
    Workspace &w = ws_;
    a.g = g64_;
    a.sigma = sig64_.as<double>();
    a.ost = w.ost.as<OuterState>();
    a.st = w.bst.as<BicgState>();
    a.map = col_map(nx, ny);
    a.r = w.r.as<double2>(); a.z = w.rt.as<double2>(); a.p = w.p.as<double2>(); a.q = w.v.as<double2>();
    a.x0 = w.X.as<double2>(); a.x1 = w.x1.as<double2>();
    a.zm = w.ph.as<double2>(); a.zc = w.s.as<double2>();
    a.parts = w.parts.as<double>();
    a.cnt = w.cnt.as<unsigned>();
    a.rerr = w.rerr.as<double>();
    a.rerr_stride = ctl.IterPerDivCor + 1;
    a.stride = nE;
    a.dsgn = -1.0;
    return a;
}
template <> ColArgs<float> Solver::cargs<float>()
{
    ColArgs<float> a{};
    Workspace &w = ws_;
    a.g = g32_;
    a.sigma = sig32_.as<float>();
    a.ost = w.ost.as<OuterState>();
    a.st = w.bst.as<BicgState>();
    a.map = col_map(nx, ny);
    a.r = w.f_r.as<float2>(); a.z = w.f_rt.as<float2>(); a.p = w.f_p.as<float2>(); a.q = w.f_v.as<float2>();
    a.x0 = w.f_x0.as<float2>(); a.x1 = w.f_x1.as<float2>();
    a.zm = w.f_ph.as<float2>(); a.zc = w.f_s.as<float2>();
    a.parts = w.parts.as<double>();
    a.cnt = w.cnt.as<unsigned>();
    a.rerr = w.rerr.as<double>();
    a.rerr_stride = ctl.IterPerDivCor + 1;
    a.stride = nE;
    a.dsgn = -1.0;
    return a;
}

DArgs Solver::dargs(int nrhs)
{
    DArgs a{};
    Workspace &w = ws_;
    a.g = g64_;
    a.sigma = sig64_.as<double>();
    a.coef = coef_.as<double>();
    a.ost = w.ost.as<OuterState>();
    a.pst = w.pst.as<PcgState>();
    a.E = w.X.as<double2>();
    a.phi0 = w.phi0.as<double2>();
    a.px = w.px.as<double2>(); a.pr = w.pr.as<double2>(); a.pp = w.pp.as<double2>(); a.pq = w.pq.as<double2>();
    a.parts = w.parts.as<double>();
    a.cnt = w.cnt.as<unsigned>();
    a.rerr = w.dcrerr.as<double>();
    a.rerr_stride = ctl.MaxIterDivCor + 1;
    a.stride = nN;
    a.estride = nE;
    a.nblk = blocks_for(nN, a.chunk);
    a.enblk = blocks_for(nE, a.echunk);
    a.maxit = ctl.MaxIterDivCor;
    a.tol = ctl.tolDivCor;
    return a;
}

int Solver::run_bicg(int nrhs, int precision, int maxit)
{
    prof_cur_ = precision;
    if (ctl.solver == 4) {  // QMR (FP64)
        KArgs<double> a = kargs<double>(nrhs, 0);
        a.maxit = maxit;
        launch_qmr_init(a, nrhs, stream_);
        for (int it = 1; it < maxit; it++) launch_qmr_iter(a, nrhs, stream_);
        launch_qmr_finish(a, nrhs, stream_);
        return check(cudaGetLastError(), "QMR launch");
    }
    if (ctl.solver == 2) {  // Bi-CG for the complex-symmetric system (COCG) with z-line preconditioner
        if (precision == 0) {
            KArgs<double> a = kargs<double>(nrhs, 0);
            a.maxit = maxit;
            ColArgs<double> c = cargs<double>();
            launch_bicg_init(a, nrhs, stream_);
            launch_zl_setup(c, nrhs, stream_);
            launch_cocg_start(c, nrhs, stream_);
            for (int it = 0; it < maxit; it++) launch_cocg_iter(c, nrhs, stream_, next_events(2));
            launch_bicg_finish(a, nrhs, stream_);
        } else {
            KArgs<float> a = kargs<float>(nrhs, 1);
            a.maxit = maxit;
            ColArgs<float> c = cargs<float>();
            launch_bicg_init(a, nrhs, stream_);
            launch_zl_setup(c, nrhs, stream_);
            launch_cocg_start(c, nrhs, stream_);
            for (int it = 0; it < maxit; it++) launch_cocg_iter(c, nrhs, stream_, next_events(2));
            launch_bicg_finish(a, nrhs, stream_);
        }
        return check(cudaGetLastError(), "Bi-CG launch");
    }
    const bool zl = ctl.solver == 3;  // BiCGStab with the z-line preconditioner
    if (precision == 0) {
        KArgs<double> a = kargs<double>(nrhs, 0);
        a.maxit = maxit;
        a.pc_ext = zl;
        ColArgs<double> c = cargs<double>();
        c.zm = ws_.zm.as<double2>();
        c.zc = ws_.zc.as<double2>();
        launch_bicg_init(a, nrhs, stream_);
        if (zl) launch_zl_setup(c, nrhs, stream_);
        for (int it = 0; it < maxit; it++) launch_bicg_iter(a, nrhs, stream_, next_events(4), zl ? &c : nullptr);
        launch_bicg_finish(a, nrhs, stream_);
    } else {
        KArgs<float> a = kargs<float>(nrhs, 1);
        a.maxit = maxit;
        a.pc_ext = zl;
        ColArgs<float> c = cargs<float>();
        c.zm = ws_.f_zm.as<float2>();
        c.zc = ws_.f_zc.as<float2>();
        launch_bicg_init(a, nrhs, stream_);
        if (zl) launch_zl_setup(c, nrhs, stream_);
        for (int it = 0; it < maxit; it++) launch_bicg_iter(a, nrhs, stream_, next_events(4), zl ? &c : nullptr);
        launch_bicg_finish(a, nrhs, stream_);
    }
    return check(cudaGetLastError(), "BiCG launch");
}

// one FP32 cycle of the fused BiCGStab (hatkernels.cu) on the normalised
// FP64 residual in tmp: x = 0, rh = D^-1 b, maxit iterations; the returned
// iterate ends in f_x0
int Solver::run_hat(int nrhs, int maxit)
{
    prof_cur_ = 1;
    KArgs<float> a = kargs<float>(nrhs, 1);
    a.maxit = maxit;
    launch_hat_cast(a, ws_.tmp.as<double2>(), nE, nrhs, stream_);
    if (prof_) {
        // timed launches, events around the operator kernels
        for (int it = 0; it < maxit; it++) launch_hat_iter(a, nrhs, stream_, next_events(4));
    } else {
        // the cycle as one CUDA graph, replayed while its arguments hold
        const cudaError_t e = hat_graph_run(hat_graph_, &a, &nrhs, nullptr, 0, maxit, stream_);
        if (e != cudaSuccess) return check(e, "fused BiCGStab graph");
    }
    launch_bicg_finish(a, nrhs, stream_);
    launch_hat_conv(a, nrhs, stream_);
    return check(cudaGetLastError(), "fused BiCGStab launch");
}

int Solver::run_hat_multi(const KArgs<float> *args, const int *nrhs, const int *zch, int ng, int maxit, cudaStream_t s)
{
    if (prof_) {
        for (int it = 0; it < maxit; it++)
            if (launch_hat_iter_multi(args, nrhs, zch, ng, s, fp32_events(4))) return 5;
        return 0;
    }
    return hat_graph_run(hat_graph_multi_, args, nrhs, zch, ng, maxit, s) == cudaSuccess ? 0 : 4;
}

KArgs<float> Solver::hat_args(int nrhs)
{
    KArgs<float> a = kargs<float>(nrhs, 1);
    a.maxit = ctl.IterPerDivCor;
    return a;
}

int Solver::set_poly(double c)
{
    if (!(c >= 0.0 && c <= 1.5)) return fail(5, "mt3d_set_poly: the coefficient must lie in [0, 1.5]");
    ctl.poly = c;
    return 0;
}
int Solver::hat_cycle_begin(int nrhs, KArgs<float> &a)
{
    a = hat_args(nrhs);
    launch_hat_cast(a, ws_.tmp.as<double2>(), nE, nrhs, stream_);
    return check(cudaGetLastError(), "fused BiCGStab start");
}
cudaEvent_t *Solver::fp32_events(int n)
{
    prof_cur_ = 1;
    return next_events(n);
}
int Solver::hat_cycle_end(int nrhs, const KArgs<float> &a)
{
    launch_bicg_finish(a, nrhs, stream_);
    launch_hat_conv(a, nrhs, stream_);
    return check(cudaGetLastError(), "fused BiCGStab end");
}

int Solver::run_divcorr(int nrhs)
{
    DArgs a = dargs(nrhs);
    launch_divcorr_start(a, nrhs, stream_);
    for (int it = 1; it < ctl.MaxIterDivCor; it++) launch_divcorr_iter(a, nrhs, stream_);
    launch_divcorr_finish(a, nrhs, stream_);
    return check(cudaGetLastError(), "divergence correction launch");
}

// ---------------------------------------------------------------------------
// y = A x on interior vectors
// ---------------------------------------------------------------------------
int Solver::mult_aii(int adjt, const double *x, double *y)
{
    if (!cond_set) return fail(5, "mt3d_mult_aii: conductivity not set (call mt3d_update_cond)");
    if (!(omega > 0)) return fail(5, "mt3d_mult_aii: frequency not set (call mt3d_update_freq)");
    if (!x || !y) return fail(5, "mt3d_mult_aii: null vector");
    int rc;
    if ((rc = ensure_workspace(1, ws_.precision < 0 ? 0 : ws_.precision))) return rc;
    OuterState os{};
    os.omega = omega;
    os.active = 1;
    if ((rc = check(cudaMemcpyAsync(ws_.ost.as<void>(), &os, sizeof os, cudaMemcpyHostToDevice, stream_), "copy state"))) return rc;
    double2 *xf = ws_.bc.as<double2>(), *yf = ws_.tmp.as<double2>(), *xi = ws_.b.as<double2>();
    cudaMemsetAsync(xf, 0, nE * sizeof(double2), stream_);
    cudaMemcpyAsync(xi, x, nEi * sizeof(double2), cudaMemcpyHostToDevice, stream_);
    launch_scatter_interior((int)nEi, edgei_d_.as<int>(), xi, xf, stream_);
    KArgs<double> a = kargs<double>(1, 0);
    a.dsgn = adjt ? 1.0 : -1.0;
    // grad-div formulation: the transposed product needs GD^T (GD is not symmetric)
    launch_apply(a, xf, yf, 0, 1, stream_, ctl.formulation == 1 ? (adjt ? 2 : 1) : 0);
    launch_gather_interior((int)nEi, edgei_d_.as<int>(), yf, xi, stream_);
    cudaMemcpyAsync(y, xi, nEi * sizeof(double2), cudaMemcpyDeviceToHost, stream_);
    return sync("mt3d_mult_aii");
}

// ---------------------------------------------------------------------------
// y = A x on full edge vectors through one internal operator kernel: 0 the
// flat FP64 apply, 1 the staged FP64 BiCGStab stencil (kcs_vt), 2 the
// TMA-staged FP32 BiCGStab stencil on the padded layout (kct_vt); 3: y =
// D^-1 A x through the fused FP32 iteration's stencil (kh_vt)
// ---------------------------------------------------------------------------
int Solver::apply_kernel(int kernel, const double *x, double *y)
{
    const char *who = "mt3d_apply_kernel";
    if (!cond_set) return fail(5, std::string(who) + ": conductivity not set (call mt3d_update_cond)");
    if (!(omega > 0)) return fail(5, std::string(who) + ": frequency not set (call mt3d_update_freq)");
    if (!x || !y || kernel < 0 || kernel > 3) return fail(5, std::string(who) + ": invalid arguments");
    if (kernel >= 2 && ctl.solver != 1)
        return fail(5, std::string(who) + ": the FP32 stencil belongs to the BiCGStab + diagonal solver");
    int rc;
    if ((rc = ensure_workspace(1, kernel >= 2 ? 1 : 0))) return rc;
    Workspace &w = ws_;
    OuterState os{};
    os.omega = omega;
    os.active = 1;
    os.scale = 1.0;
    BicgState bs{};
    bs.status = KS_RUNNING;
    cudaMemcpyAsync(w.ost.as<void>(), &os, sizeof os, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(w.bst.as<void>(), &bs, sizeof bs, cudaMemcpyHostToDevice, stream_);
    double2 *X = w.tmp.as<double2>(), *Y = w.bc.as<double2>();
    cudaMemcpyAsync(X, x, nE * sizeof(double2), cudaMemcpyHostToDevice, stream_);
    if (kernel == 0) {
        KArgs<double> a = kargs<double>(1, 0);
        launch_apply(a, X, Y, 0, 1, stream_, ctl.formulation == 1);
    } else if (kernel == 1) {
        KArgs<double> a = kargs<double>(1, 0);
        cudaMemcpyAsync(a.ph, X, nE * sizeof(double2), cudaMemcpyDeviceToDevice, stream_);
        launch_stage_vt(a, 0, 1, stream_);
        cudaMemcpyAsync(Y, a.v, nE * sizeof(double2), cudaMemcpyDeviceToDevice, stream_);
    } else {
        if ((rc = tma_ready())) return rc;
        // x to FP32 on the padded layout (scale 1), through the stencil, back
        launch_cast_padded(g64_, w.ost.as<OuterState>(), nE, X, pl_, w.f_ph.as<float2>(), w.f_x0.as<float2>(), 1,
                           stream_);
        KArgs<float> a = kargs<float>(1, 1);
        if (kernel == 2) launch_tma_vt(a, tma_, 0, 1, stream_);
        else launch_hat_apply(a, 1, stream_);
        cudaMemsetAsync(Y, 0, nE * sizeof(double2), stream_);
        launch_update_padded(g64_, w.ost.as<OuterState>(), nE, pl_, w.f_v.as<float2>(), Y, 1, stream_);
    }
    cudaMemcpyAsync(y, Y, nE * sizeof(double2), cudaMemcpyDeviceToHost, stream_);
    if ((rc = sync(who))) return rc;
    return check_device_error(who);
}

// ---------------------------------------------------------------------------
// one Krylov call on interior vectors (BICG / cuBiCG)
// ---------------------------------------------------------------------------
int Solver::bicg(const double *b, double *x, int maxit, double tol, int *niter, double *rerr, int *failed)
{
    if (!cond_set) return fail(5, "mt3d_bicg: conductivity not set (call mt3d_update_cond)");
    if (!(omega > 0)) return fail(5, "mt3d_bicg: frequency not set (call mt3d_update_freq)");
    if (!b || !x || maxit < 1 || !(tol > 0)) return fail(5, "mt3d_bicg: invalid arguments");
    const int keep = ctl.IterPerDivCor;
    ctl.IterPerDivCor = maxit;  // rerr rows of maxit+1 entries
    int rc = ensure_workspace(1, 0);
    ctl.IterPerDivCor = keep;
    if (rc) return rc;
    OuterState os{};
    os.omega = omega;
    os.tol = tol;
    os.active = 1;
    cudaMemcpyAsync(ws_.ost.as<void>(), &os, sizeof os, cudaMemcpyHostToDevice, stream_);
    double2 *xi = ws_.tmp.as<double2>();
    cudaMemsetAsync(ws_.b.as<void>(), 0, nE * sizeof(double2), stream_);
    cudaMemsetAsync(ws_.X.as<void>(), 0, nE * sizeof(double2), stream_);
    cudaMemcpyAsync(xi, b, nEi * sizeof(double2), cudaMemcpyHostToDevice, stream_);
    launch_scatter_interior((int)nEi, edgei_d_.as<int>(), xi, ws_.b.as<double2>(), stream_);
    cudaMemcpyAsync(xi, x, nEi * sizeof(double2), cudaMemcpyHostToDevice, stream_);
    launch_scatter_interior((int)nEi, edgei_d_.as<int>(), xi, ws_.X.as<double2>(), stream_);
    {
        KArgs<double> a = kargs<double>(1, 0);
        a.maxit = maxit;
        a.rerr_stride = maxit + 1;
        launch_bicg_init(a, 1, stream_);
        for (int it = 0; it < maxit; it++) launch_bicg_iter(a, 1, stream_);
        launch_bicg_finish(a, 1, stream_);
    }
    launch_gather_interior((int)nEi, edgei_d_.as<int>(), ws_.X.as<double2>(), xi, stream_);
    cudaMemcpyAsync(x, xi, nEi * sizeof(double2), cudaMemcpyDeviceToHost, stream_);
    BicgState st;
    cudaMemcpyAsync(&st, ws_.bst.as<void>(), sizeof st, cudaMemcpyDeviceToHost, stream_);
    std::vector<double> h(maxit + 1);
    cudaMemcpyAsync(h.data(), ws_.rerr.as<void>(), (maxit + 1) * sizeof(double), cudaMemcpyDeviceToHost, stream_);
    if ((rc = sync("mt3d_bicg"))) return rc;
    const bool conv = st.status == KS_CONVERGED;
    const int n = conv ? st.iter : maxit;
    if (!conv && st.imin > 0) h[maxit - 1] = h[st.imin - 1];
    if (!conv && st.imin == 0) h[maxit - 1] = h[0];
    if (niter) *niter = n;
    if (failed) *failed = (st.status == KS_BREAKDOWN || st.status == KS_NAN) ? 1 : 0;
    if (rerr) std::memcpy(rerr, h.data(), maxit * sizeof(double));
    if (st.status == KS_NAN) return fail(3, "mt3d_bicg: NaN in the right-hand side or iterates");
    if (st.status == KS_BREAKDOWN) return fail(2, "mt3d_bicg: BiCGStab breakdown");
    return conv ? 0 : 1;
}

// ---------------------------------------------------------------------------
// FWDsolve3D over a batch of right-hand sides
// ---------------------------------------------------------------------------
void Solver::push_state(SolveRun &run)
{
    cudaMemcpyAsync(ws_.ost.as<void>(), run.os.data(), run.nrhs * sizeof(OuterState), cudaMemcpyHostToDevice,
                    stream_);
}

// take over the device-written fields of the outer states
int Solver::pull_state(SolveRun &run)
{
    std::vector<OuterState> dv(run.nrhs);
    cudaMemcpyAsync(dv.data(), ws_.ost.as<void>(), run.nrhs * sizeof(OuterState), cudaMemcpyDeviceToHost, stream_);
    int rc = sync("fwdsolve");
    if (rc) return rc;
    for (int r = 0; r < run.nrhs; r++) {
        run.os[r].bnorm64 = dv[r].bnorm64;
        run.os[r].relres = dv[r].relres;
        run.os[r].scale = dv[r].scale;
        run.os[r].divJ[0] = dv[r].divJ[0];
        run.os[r].divJ[1] = dv[r].divJ[1];
    }
    return 0;
}

bool SolveRun::any_active() const
{
    for (auto &o : os)
        if (o.active) return true;
    return false;
}

int Solver::solve(int nrhs, const double *omegas, const int *trans, const double *bc, const double *src, double *e,
                  int *status, bool device)
{
    SolveRun run;
    int rc = solve_begin(run, nrhs, omegas, trans, bc, src, e, status, device);
    if (rc) return rc;
    while (!run.done) {
        if ((rc = solve_pre(run))) return rc;
        if (run.done) break;
        if ((rc = solve_fp32(run))) return rc;
        if ((rc = solve_post(run))) return rc;
    }
    return solve_end(run);
}

// ---------------------------------------------------------------------------
// FWDsolve3D over a batch of right-hand sides, in phases: set-up (RHS
// assembly, initial divergence correction), then per outer cycle the true
// residual and the decisions (solve_pre), the FP32 Krylov cycle (solve_fp32),
// the FP64 cycles and bookkeeping (solve_post), and the post-processing
// (solve_end).  A multi-grid batch runs the phases of several handles in
// lockstep, with the FP32 cycles of all grids in shared launches.
// ---------------------------------------------------------------------------
int Solver::solve_begin(SolveRun &run, int nrhs, const double *omegas, const int *trans, const double *bc,
                        const double *src, double *e, int *status, bool device)
{
    if (!cond_set) return fail(5, "fwdsolve: conductivity not set (call mt3d_update_cond)");
    // the kernels index the right-hand sides by the grid's y dimension
    if (nrhs > kMaxBatch) return fail(5, "fwdsolve: at most 65535 right-hand sides per call");
    if (nrhs < 1 || !omegas || !e) return fail(5, "fwdsolve: invalid arguments");
    for (int r = 0; r < nrhs; r++)
        if (!(omegas[r] > 0) || !std::isfinite(omegas[r])) return fail(5, "fwdsolve: omega must be positive and finite");
    const int prec = ctl.precision;
    int rc;
    if ((rc = ensure_workspace(nrhs, prec))) return rc;
    Workspace &w = ws_;
    run = SolveRun{};
    run.nrhs = nrhs;
    run.prec = prec;
    run.device = device;
    run.e = e;
    run.status = status;
    run.refine = prec == 1 || ctl.formulation == 1;  // loop driven by the true FP64 residual
    const size_t ebytes = nE * sizeof(double2);
    const cudaMemcpyKind in_kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (prof_) collect_events();
    double2 *B = w.b.as<double2>(), *X = w.X.as<double2>(), *BC = w.bc.as<double2>(), *TMP = w.tmp.as<double2>();
    // boundary data (kept for the post-processing) and initial guess
    std::vector<OuterState> &os = run.os;
    os.assign(nrhs, OuterState{});
    for (int r = 0; r < nrhs; r++) {
        os[r].omega = omegas[r];
        os[r].trans = trans ? (trans[r] != 0) : 0;
        os[r].active = 1;
    }
    push_state(run);
    cudaMemsetAsync(BC, 0, nrhs * ebytes, stream_);
    if (bc) cudaMemcpyAsync(BC, bc, nrhs * ebytes, in_kind, stream_);
    cudaMemcpyAsync(X, e, nrhs * ebytes, in_kind, stream_);
    launch_keep_interior(g64_, X, nE, nrhs, stream_);
    // forward right-hand side: b = -V_E A_IB bc (FWDsolve3D, f90/3D_MT/FWD/EMsolve3D.f90:186-200)
    cudaMemcpyAsync(TMP, BC, nrhs * ebytes, cudaMemcpyDeviceToDevice, stream_);
    for (int r = 0; r < nrhs; r++)
        if (os[r].trans) cudaMemsetAsync(TMP + (size_t)r * nE, 0, ebytes, stream_);
    launch_keep_boundary(g64_, TMP, nE, nrhs, stream_);
    {
        KArgs<double> a = kargs<double>(nrhs, 0);
        launch_apply(a, TMP, B, 1, nrhs, stream_);
    }
    // which right-hand sides carry non-zero boundary data / sources (found on
    // the device); the sources stay in TMP
    std::vector<int> flags(2 * nrhs, 0);
    int *dflags = w.cnt.as<int>() + nrhs;  // scratch after the reduction counters
    cudaMemsetAsync(dflags, 0, 2 * nrhs * sizeof(int), stream_);
    launch_nonzero(BC, nE, (int)nE, dflags, nrhs, stream_);
    if (src) {
        cudaMemcpyAsync(TMP, src, nrhs * ebytes, in_kind, stream_);
        launch_keep_interior(g64_, TMP, nE, nrhs, stream_);
        launch_nonzero(TMP, nE, (int)nE, dflags + nrhs, nrhs, stream_);
    }
    cudaMemcpyAsync(flags.data(), dflags, 2 * nrhs * sizeof(int), cudaMemcpyDeviceToHost, stream_);
    if ((rc = sync("fwdsolve input"))) return rc;
    bool any_src = false;
    for (int r = 0; r < nrhs; r++) {
        OuterState &o = os[r];
        o.has_bc = flags[r] != 0;
        o.has_src = flags[nrhs + r] != 0;
        o.tol = o.trans ? ctl.tolEMadj : (o.has_bc ? ctl.tolEMfwd : ctl.tolEMadj);
        any_src = any_src || o.has_src;
    }
    push_state(run);
    // sources: b += V_E src (forward) or b = src (transposed); phi0 for the
    // divergence correction, or the grad-div source correction of the SP2
    // right-hand side (f90/3D_MT/FWD_SP2/EMsolve3D.f90:215-228, 271-289)
    if (any_src) {
        launch_add_src(g64_, B, TMP, nE, w.ost.as<OuterState>(), nrhs, stream_);
        if (ctl.formulation == 0) {
            launch_phi0(g64_, TMP, nE, w.phi0.as<double2>(), nN, w.ost.as<OuterState>(), nrhs, stream_);
        } else {
            KArgs<double> a = kargs<double>(nrhs, 0);
            launch_gd_phi(a, TMP, a.phi, 1, nrhs, stream_);
            launch_gd_add(a, B, a.phi, nrhs, stream_);
        }
    }
    {
        KArgs<double> a = kargs<double>(nrhs, 0);
        launch_norm_b(a, nrhs, stream_);
    }
    // transposed problem without a source: zero solution (plus boundary
    // data), whatever the first guess (f90/3D_MT/FWD_SP2/EMsolve3D.f90:233-245)
    for (int r = 0; r < nrhs; r++)
        if (os[r].trans && !os[r].has_src) {
            cudaMemsetAsync(X + (size_t)r * nE, 0, ebytes, stream_);
            os[r].active = 0;
            os[r].converged = 1;
        }
    diag = Diag{};
    run.dg.assign(nrhs, Diag{});
    if ((rc = pull_state(run))) return rc;
    for (int r = 0; r < nrhs; r++) {
        if (!std::isfinite(os[r].bnorm64)) {
            os[r].active = 0;
            os[r].failed = 3;
        } else if (os[r].active && os[r].bnorm64 == 0.0) {
            // zero right-hand side (no boundary data, no source): zero
            // interior solution, reported as BICG reports b = 0 (one
            // iteration, relative residual 0; f90/3D_MT/FWD_SP2/
            // solver.f90:780-786)
            cudaMemsetAsync(X + (size_t)r * nE, 0, ebytes, stream_);
            os[r].active = 0;
            os[r].converged = 1;
            os[r].nIterTotal = 1;
            os[r].relres = 0.0;
            run.dg[r].EMrelErr.push_back(0.0);
        }
    }
    // initial divergence correction for a source term (EMsolve3D.f90:298-303)
    bool any_dc = false;
    for (int r = 0; r < nrhs; r++) {
        os[r].dc_run = ctl.formulation == 0 && os[r].active && os[r].has_src;
        if (os[r].dc_run) { os[r].nDivCor = 1; any_dc = true; }
    }
    push_state(run);
    if (any_dc) {
        if ((rc = run_divcorr(nrhs))) return rc;
        if ((rc = pull_state(run))) return rc;
        for (int r = 0; r < nrhs; r++)
            if (os[r].dc_run) { run.dg[r].divJ.push_back(os[r].divJ[0]); run.dg[r].divJ.push_back(os[r].divJ[1]); }
    }
    run.bs.assign(nrhs, BicgState{});
    run.rerr.assign((size_t)nrhs * (ctl.IterPerDivCor + 1), 0.0);
    // mixed precision: a right-hand side whose last FP32 cycle did not halve
    // its true FP64 residual continues with FP64 Krylov cycles (the FP32
    // operator's rounding can stop an FP32 solve from reducing a residual
    // that is already small relative to the field)
    run.prev_relres.assign(nrhs, std::numeric_limits<double>::infinity());
    run.hi.assign(nrhs, 0);
    // smallest relative residual of the last FP32 cycle's own iteration and
    // the number of FP32 cycles in a row that did not halve the true residual
    run.inner_best.assign(nrhs, 0.0);
    run.stalls.assign(nrhs, 0);
    run.done = !run.any_active();
    return 0;
}

// start of an outer cycle: the true FP64 residual r64 = b - A X (into tmp);
// converged right-hand sides leave the loop; the FP32 and FP64 groups of the
// mixed-precision cycle; the FP32 group marked active on the device
int Solver::solve_pre(SolveRun &run)
{
    Workspace &w = ws_;
    std::vector<OuterState> &os = run.os;
    const int nrhs = run.nrhs;
    int rc;
    run.n32 = run.n64 = false;
    if (!run.any_active()) {
        run.done = true;
        return 0;
    }
    if (run.refine) {
        for (auto &o : os) o.dc_run = 0;
        push_state(run);
        {
            KArgs<double> a = kargs<double>(nrhs, 0);
            a.r = w.tmp.as<double2>();
            launch_res64(a, nrhs, stream_);
        }
        if ((rc = pull_state(run))) return rc;
        bool work = false;
        for (int r = 0; r < nrhs; r++) {
            OuterState &o = os[r];
            if (!o.active) continue;
            if (!std::isfinite(o.relres)) { o.active = 0; o.failed = 3; continue; }
            if (o.relres <= o.tol) { o.active = 0; o.converged = 1; continue; }
            if (o.nDivCor >= ctl.MaxDivCor) { o.active = 0; o.failed = 1; continue; }
            o.tol_inner = o.tol * o.bnorm64 * o.scale;  // tol*||b|| relative to ||r64||
            // an FP32 cycle that did not halve the true residual: when its
            // own iteration converged well, the FP32 operator's rounding is
            // the limit and the right-hand side moves to FP64; when the
            // iteration itself stagnated, one more FP32 cycle restarts it
            // from the new residual first
            if (run.prec == 1 && !run.hi[r]) {
                if (o.relres > 0.5 * run.prev_relres[r]) {
                    if (run.inner_best[r] < 0.1 || ++run.stalls[r] >= 2) run.hi[r] = 1;
                } else {
                    run.stalls[r] = 0;
                }
            }
            run.prev_relres[r] = o.relres;
            work = true;
        }
        if (!work) {
            run.done = true;
            return 0;
        }
        push_state(run);
    }
    if (run.prec == 1) {
        // FP32 cycles on the normalised residual, FP64 cycles on (b, X) for
        // the right-hand sides that left FP32; each group runs with the
        // other group's right-hand sides marked inactive on the device
        for (int r = 0; r < nrhs; r++) {
            if (!os[r].active) continue;
            (run.hi[r] ? run.n64 : run.n32) = true;
        }
        run.grp = os;
        if (run.n32) {
            for (int r = 0; r < nrhs; r++) run.grp[r].active = os[r].active && !run.hi[r];
            cudaMemcpyAsync(w.ost.as<void>(), run.grp.data(), nrhs * sizeof(OuterState), cudaMemcpyHostToDevice,
                            stream_);
            if (w.padded && (rc = tma_ready())) return rc;
        }
    }
    return 0;
}

// whether this cycle's FP32 group runs the fused iteration (and so may share
// launches with other grids)
bool Solver::fp32_fused(const SolveRun &run) const
{
    return run.prec == 1 && run.n32 && ws_.padded && ctl.fused;
}

// the FP32 cycle of the FP32 group on this handle alone
int Solver::solve_fp32(SolveRun &run)
{
    Workspace &w = ws_;
    const int nrhs = run.nrhs;
    if (!(run.prec == 1 && run.n32)) return 0;
    if (fp32_fused(run)) return run_hat(nrhs, ctl.IterPerDivCor);
    if (w.padded) {
        launch_cast_padded(g64_, w.ost.as<OuterState>(), nE, w.tmp.as<double2>(), pl_, w.f_b.as<float2>(),
                           w.f_x0.as<float2>(), nrhs, stream_);
    } else {
        launch_cast(w.ost.as<OuterState>(), (int)nE, nE, w.tmp.as<double2>(), w.f_b.as<float2>(), w.f_x0.as<float2>(),
                    nrhs, stream_);
    }
    return run_bicg(nrhs, 1, ctl.IterPerDivCor);
}

// end of an outer cycle: the FP32 correction into X, the FP64 group (or the
// FP64 Krylov call), the Krylov states and histories, the divergence
// correction and the right-hand sides that finished
int Solver::solve_post(SolveRun &run)
{
    Workspace &w = ws_;
    std::vector<OuterState> &os = run.os;
    const int nrhs = run.nrhs, prec = run.prec;
    double2 *X = w.X.as<double2>();
    int rc;
    if (prec == 1) {
        if (run.n32) {
            if (w.padded)
                launch_update_padded(g64_, w.ost.as<OuterState>(), nE, pl_, w.f_x0.as<float2>(), X, nrhs, stream_);
            else
                launch_update(w.ost.as<OuterState>(), (int)nE, nE, w.f_x0.as<float2>(), X, nrhs, stream_);
        }
        if (run.n64) {
            if ((rc = ensure_fp64_krylov(nrhs))) return rc;
            for (int r = 0; r < nrhs; r++) run.grp[r].active = os[r].active && run.hi[r];
            cudaMemcpyAsync(w.ost.as<void>(), run.grp.data(), nrhs * sizeof(OuterState), cudaMemcpyHostToDevice,
                            stream_);
            if ((rc = run_bicg(nrhs, 0, ctl.IterPerDivCor))) return rc;
        }
        push_state(run);
    } else {
        // Krylov call: FP64 on (b, X)
        if ((rc = run_bicg(nrhs, prec, ctl.IterPerDivCor))) return rc;
    }
    std::vector<BicgState> &bs = run.bs;
    std::vector<double> &rerr = run.rerr;
    cudaMemcpyAsync(bs.data(), w.bst.as<void>(), nrhs * sizeof(BicgState), cudaMemcpyDeviceToHost, stream_);
    cudaMemcpyAsync(rerr.data(), w.rerr.as<void>(), rerr.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_);
    if ((rc = sync("fwdsolve Krylov cycle"))) return rc;
    if ((rc = check_device_error("fwdsolve Krylov cycle"))) return rc;
    if (prof_) collect_events();
    for (int r = 0; r < nrhs; r++) {
        OuterState &o = os[r];
        o.dc_run = 0;
        if (!o.active) continue;
        const BicgState &st = bs[r];
        const int maxit = ctl.IterPerDivCor;
        const bool conv = st.status == KS_CONVERGED;
        const int niter = conv ? st.iter : maxit;
        double *h = &rerr[(size_t)r * (maxit + 1)];
        if (!conv) h[maxit - 1] = st.imin > 0 ? h[st.imin - 1] : h[0];
        for (int k = 0; k < niter; k++) run.dg[r].EMrelErr.push_back(h[k]);
        if (prec == 1 && !run.hi[r]) {
            double best = 1.0;
            for (int k = 0; k < niter; k++) best = std::min(best, h[k]);
            run.inner_best[r] = best;
        }
        o.nIterTotal += niter;
        if (!run.refine) {
            if (conv) o.converged = 1;
            if (st.status == KS_BREAKDOWN || st.status == KS_NAN) o.failed = (st.status == KS_NAN) ? 3 : 2;
        } else if (st.status == KS_NAN) {
            o.failed = 3;
        }
        o.nDivCor += 1;
        if (o.nDivCor < ctl.MaxDivCor) {
            o.dc_run = ctl.formulation == 0;
        } else if (!run.refine) {
            if (!o.failed) o.failed = 1;
        }
    }
    push_state(run);
    bool dc = false;
    for (auto &o : os) dc = dc || o.dc_run;
    if (dc) {
        if ((rc = run_divcorr(nrhs))) return rc;
        if ((rc = pull_state(run))) return rc;
        for (int r = 0; r < nrhs; r++)
            if (os[r].dc_run) { run.dg[r].divJ.push_back(os[r].divJ[0]); run.dg[r].divJ.push_back(os[r].divJ[1]); }
    }
    for (int r = 0; r < nrhs; r++) {
        OuterState &o = os[r];
        o.dc_run = 0;
        if (!o.active) continue;
        if (!run.refine) {
            if (o.converged || o.failed) o.active = 0;
        } else if (o.failed == 3) {
            o.active = 0;
        }
    }
    // right-hand sides that finished in this cycle sit out the next one
    push_state(run);
    run.done = !run.any_active();
    return 0;
}

// true relative residual of the returned interior fields, post-processing,
// copy back and the statuses
int Solver::solve_end(SolveRun &run)
{
    Workspace &w = ws_;
    std::vector<OuterState> &os = run.os;
    const int nrhs = run.nrhs;
    double2 *X = w.X.as<double2>(), *BC = w.bc.as<double2>();
    int rc;
    for (auto &o : os) { o.active = 1; o.dc_run = 0; }
    push_state(run);
    {
        KArgs<double> a = kargs<double>(nrhs, 0);
        if (run.prec == 1) a.r = w.tmp.as<double2>();
        launch_res64(a, nrhs, stream_);
    }
    if ((rc = pull_state(run))) return rc;
    launch_post(g64_, X, BC, nE, w.ost.as<OuterState>(), nrhs, stream_);
    cudaMemcpyAsync(run.e, X, nrhs * nE * sizeof(double2),
                    run.device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream_);
    if ((rc = sync("fwdsolve copy back"))) return rc;
    if (prof_) collect_events();
    int worst = 0;
    for (int r = 0; r < nrhs; r++) {
        OuterState &o = os[r];
        int s = 0;
        if (o.failed == 3) s = 3;
        else if (o.failed == 2) s = 2;
        else if (!o.converged) s = 1;
        if (run.status) run.status[r] = s;
        worst = std::max(worst, s);
        run.dg[r].nIterTotal = o.nIterTotal;
        run.dg[r].nDivCor = o.nDivCor;
        run.dg[r].failed = s != 0;
        run.dg[r].final_relres = o.relres;
    }
    diag = run.dg[0];
    batch_niter.assign(nrhs, 0);
    batch_relres.assign(nrhs, 0.0);
    for (int r = 0; r < nrhs; r++) {
        batch_niter[r] = os[r].nIterTotal;
        batch_relres[r] = os[r].relres;
    }
    if (worst == 3) return fail(3, "fwdsolve: NaN/Inf in the right-hand side or iterates");
    if (worst == 2) return fail(2, "fwdsolve: BiCGStab breakdown");
    return worst;
}

int Solver::pmult_t(int npol, const double *e0, const double *eadj, const double *m0, double *dm)
{
    if (npol < 1 || !e0 || !eadj || !m0 || !dm) return fail(5, "mt3d_pmult_t: invalid arguments");
    if (!(omega > 0)) return fail(5, "mt3d_pmult_t: frequency not set (call mt3d_update_freq)");
    const size_t eb = (size_t)npol * nE * sizeof(double2);
    const int64_t nEarth = (int64_t)nx * ny * (nz - nzAir);
    DevBuf a, b, m, d;
    if (a.alloc(eb) || b.alloc(eb) || m.alloc(nEarth * sizeof(double)) || d.alloc(nEarth * sizeof(double)))
        return fail(8, "mt3d_pmult_t: out of device memory");
    cudaMemcpyAsync(a.as<void>(), e0, eb, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(b.as<void>(), eadj, eb, cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(m.as<void>(), m0, nEarth * sizeof(double), cudaMemcpyHostToDevice, stream_);
    launch_pmult_t(g64_, npol, a.as<double2>(), b.as<double2>(), omega, m.as<double>(), d.as<double>(), stream_);
    cudaMemcpyAsync(dm, d.as<void>(), nEarth * sizeof(double), cudaMemcpyDeviceToHost, stream_);
    return sync("mt3d_pmult_t");
}

}  // namespace mt3d

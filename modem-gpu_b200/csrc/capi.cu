// capi.cu -- extern "C" entry points of libmt3d.so (declared in include/mt3d.h).
// Each call validates its arguments, runs on the handle's device and
// returns an mt3d_status; exceptions never cross the boundary.
#include <atomic>
#include <cstring>
#include <new>
#include <string>

#include "../../include/mt3d.h"
#include "solver.h"

namespace mt3d {
extern std::atomic<long long> g_launch_count;
extern std::atomic<long long> g_alloc_count;
}

struct mt3d_solver {
    mt3d::Solver s;
    int device = 0;
};

namespace {
thread_local std::string g_create_error;

int guard_device(mt3d_handle h)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    if (cudaSetDevice(h->device) != cudaSuccess) {
        cudaGetLastError();
        h->s.last_error = "cudaSetDevice failed";
        return MT3D_CUDA_ERROR;
    }
    return 0;
}

template <typename F> int wrap(mt3d_handle h, F &&f)
{
    int rc = guard_device(h);
    if (rc) return rc;
    try {
        return f();
    } catch (const std::bad_alloc &) {
        h->s.last_error = "host out of memory";
        return MT3D_OUT_OF_MEMORY;
    } catch (...) {
        h->s.last_error = "unexpected exception";
        return MT3D_CUDA_ERROR;
    }
}
}  // namespace

extern "C" {

#ifndef MT3D_SRC_HASH
#define MT3D_SRC_HASH "unknown"
#endif
// the source hash of build.py follows "mt3d-src-"
const char *mt3d_version(void) { return "mt3d-b200 0.2 (sm_100a) mt3d-src-" MT3D_SRC_HASH; }

int mt3d_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int mt3d_create(int device_id, int nx, int ny, int nz, int nzAir, const double *dx, const double *dy, const double *dz,
                mt3d_handle *out)
{
    if (!out) return MT3D_INVALID_ARGUMENT;
    *out = nullptr;
    mt3d_solver *h = nullptr;
    try {
        h = new mt3d_solver();
    } catch (...) {
        g_create_error = "host out of memory";
        return MT3D_OUT_OF_MEMORY;
    }
    h->device = device_id;
    int rc = h->s.create(device_id, nx, ny, nz, nzAir, dx, dy, dz);
    if (rc) {
        g_create_error = h->s.last_error;
        delete h;
        return rc;
    }
    *out = h;
    return MT3D_OK;
}

int mt3d_destroy(mt3d_handle h)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    delete h;
    return MT3D_OK;
}

int mt3d_set_control(mt3d_handle h, int IterPerDivCor, int MaxDivCor, int MaxIterDivCor, double tolEMfwd,
                     double tolEMadj, double tolDivCor, int solver, int precision)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    if (IterPerDivCor < 1 || MaxDivCor < 1 || MaxIterDivCor < 1 || !(tolEMfwd > 0) || !(tolEMadj > 0) ||
        !(tolDivCor > 0)) {
        h->s.last_error = "mt3d_set_control: iteration counts must be >= 1 and tolerances > 0";
        return MT3D_INVALID_ARGUMENT;
    }
    if (solver != MT3D_SOLVER_BICG && solver != MT3D_SOLVER_COCG && solver != MT3D_SOLVER_BICG_ZLINE &&
        solver != MT3D_SOLVER_QMR) {
        h->s.last_error = "mt3d_set_control: unknown solver";
        return MT3D_INVALID_ARGUMENT;
    }
    if (solver == MT3D_SOLVER_QMR && precision != MT3D_PREC_FP64) {
        h->s.last_error = "mt3d_set_control: QMR runs in FP64 (MT3D_PREC_FP64)";
        return MT3D_INVALID_ARGUMENT;
    }
    if (precision != MT3D_PREC_FP64 && precision != MT3D_PREC_MIXED) {
        h->s.last_error = "mt3d_set_control: unknown precision mode";
        return MT3D_INVALID_ARGUMENT;
    }
    mt3d::Control &c = h->s.ctl;
    c.IterPerDivCor = IterPerDivCor;
    c.MaxDivCor = MaxDivCor;
    c.MaxIterDivCor = MaxIterDivCor;
    c.tolEMfwd = tolEMfwd;
    c.tolEMadj = tolEMadj;
    c.tolDivCor = tolDivCor;
    c.solver = solver;
    c.precision = precision;
    return MT3D_OK;
}

int mt3d_set_restart(mt3d_handle h, int restart)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    if (restart < 0) {
        h->s.last_error = "mt3d_set_restart: restart length must be >= 0";
        return MT3D_INVALID_ARGUMENT;
    }
    h->s.ctl.restart = restart;
    return MT3D_OK;
}

int mt3d_set_formulation(mt3d_handle h, int formulation)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    if (formulation != MT3D_FORM_CCDC && formulation != MT3D_FORM_CCGD) {
        h->s.last_error = "mt3d_set_formulation: unknown formulation";
        return MT3D_INVALID_ARGUMENT;
    }
    h->s.ctl.formulation = formulation;
    return MT3D_OK;
}

int mt3d_update_cond(mt3d_handle h, const double *m_earth, double airCond)
{
    return wrap(h, [&] { return h->s.update_cond(m_earth, airCond); });
}

int mt3d_get_cond(mt3d_handle h, double *sigma_e, double *divcorr, double *node_w)
{
    return wrap(h, [&] { return h->s.get_cond(sigma_e, divcorr, node_w); });
}

int mt3d_compute_bc(mt3d_handle h, int imode, double *e0)
{
    return wrap(h, [&] {
        if (!(h->s.omega > 0)) return h->s.fail(5, "mt3d_compute_bc: frequency not set (call mt3d_update_freq)");
        return h->s.compute_bc(imode, h->s.omega, e0, false);
    });
}

int mt3d_compute_bc_device(mt3d_handle h, int imode, double omega, void *e0)
{
    return wrap(h, [&] { return h->s.compute_bc(imode, omega, reinterpret_cast<double *>(e0), true); });
}

int mt3d_update_freq(mt3d_handle h, double omega)
{
    return wrap(h, [&] { return h->s.update_freq(omega); });
}

int mt3d_sizes(mt3d_handle h, int64_t *nE, int64_t *nEi, int64_t *nN)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    if (nE) *nE = h->s.nE;
    if (nEi) *nEi = h->s.nEi;
    if (nN) *nN = h->s.nN;
    return MT3D_OK;
}

int mt3d_interior_index(mt3d_handle h, int32_t *edgei)
{
    if (!h || !edgei) return MT3D_INVALID_ARGUMENT;
    for (size_t i = 0; i < h->s.edgei.size(); i++) edgei[i] = h->s.edgei[i] + 1;
    return MT3D_OK;
}

int mt3d_mult_aii(mt3d_handle h, int adjt, const double *x, double *y)
{
    return wrap(h, [&] { return h->s.mult_aii(adjt, x, y); });
}

int mt3d_mult_aii_device_noalloc(mt3d_handle h, int adjt, const double *x, double *y)
{
    return wrap(h, [&] { return h->s.mult_aii_noalloc(adjt, x, y); });
}

int mt3d_impedance(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin, const double *e1,
                   const double *e2, double *Z)
{
    return wrap(h, [&] { return h->s.impedance(omega, nsite, xyz, origin, e1, e2, Z, false); });
}

int mt3d_impedance_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                          const double *e1_dev, const double *e2_dev, double *Z)
{
    return wrap(h, [&] { return h->s.impedance(omega, nsite, xyz, origin, e1_dev, e2_dev, Z, true); });
}

int mt3d_lmult_t(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin, const double *e1,
                 const double *e2, const double *d, double *s1, double *s2)
{
    return wrap(h, [&] { return h->s.lmult_t(omega, nsite, xyz, origin, e1, e2, d, s1, s2, false); });
}

int mt3d_lmult_t_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                        const double *e1_dev, const double *e2_dev, const double *d, double *s1_dev, double *s2_dev)
{
    return wrap(h, [&] { return h->s.lmult_t(omega, nsite, xyz, origin, e1_dev, e2_dev, d, s1_dev, s2_dev, true); });
}

int mt3d_bicg(mt3d_handle h, const double *b, double *x, int maxit, double tol, int *niter, double *rerr, int *failed)
{
    return wrap(h, [&] { return h->s.bicg(b, x, maxit, tol, niter, rerr, failed); });
}

int mt3d_fwdsolve(mt3d_handle h, int trans, const double *bc, const double *src, double *e)
{
    return wrap(h, [&] {
        double om = h->s.omega;
        if (!(om > 0)) {
            h->s.last_error = "mt3d_fwdsolve: frequency not set (call mt3d_update_freq)";
            return (int)MT3D_INVALID_ARGUMENT;
        }
        int tr = trans ? 1 : 0, st = 0;
        return h->s.solve(1, &om, &tr, bc, src, e, &st);
    });
}

int mt3d_fwdsolve_batch(mt3d_handle h, int nrhs, const double *omegas, const int *trans, const double *bc,
                        const double *src, double *e, int *status)
{
    return wrap(h, [&] { return h->s.solve(nrhs, omegas, trans, bc, src, e, status); });
}

int mt3d_fwdsolve_batch_device(mt3d_handle h, int nrhs, const double *omegas, const int *trans, const double *bc_dev,
                               const double *src_dev, double *e_dev, int *status)
{
    return wrap(h, [&] { return h->s.solve(nrhs, omegas, trans, bc_dev, src_dev, e_dev, status, true); });
}

int mt3d_set_stream(mt3d_handle h, void *stream)
{
    return wrap(h, [&] { return h->s.set_stream(stream); });
}

int mt3d_jmult_t(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin, const double *e0,
                 const double *d, const double *m0_earth, double *dm, double *eadj)
{
    return wrap(h, [&] { return h->s.jmult_t(omega, nsite, xyz, origin, e0, d, m0_earth, dm, eadj, false); });
}

int mt3d_jmult_t_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                        const double *e0_dev, const double *d, const double *m0_earth, double *dm_dev,
                        double *eadj_dev)
{
    return wrap(h, [&] {
        return h->s.jmult_t(omega, nsite, xyz, origin, e0_dev, d, m0_earth, dm_dev, eadj_dev, true);
    });
}

static int fwdsolve_multi_entry(int nh, mt3d_handle *hs, const int *nrhs, const double *const *omegas,
                                const int *const *trans, const double *const *bc, const double *const *src,
                                double *const *e, int *const *status, const int *zchunks, bool device)
{
    if (nh < 1 || nh > 8 || !hs) {
        g_create_error = "mt3d_fwdsolve_multi: 1 to 8 handles";
        return MT3D_INVALID_ARGUMENT;
    }
    mt3d::Solver *ss[8];
    for (int i = 0; i < nh; i++) {
        if (!hs[i]) {
            g_create_error = "mt3d_fwdsolve_multi: null handle";
            return MT3D_INVALID_ARGUMENT;
        }
        ss[i] = &hs[i]->s;
    }
    const int rc0 = guard_device(hs[0]);
    if (rc0) return rc0;
    try {
        std::string err;
        const int rc = mt3d::fwdsolve_multi(nh, ss, nrhs, omegas, trans, bc, src, e, status, zchunks, device, err);
        if (rc) {
            g_create_error = err;
            hs[0]->s.last_error = err;
        }
        return rc;
    } catch (const std::bad_alloc &) {
        g_create_error = "host out of memory";
        return MT3D_OUT_OF_MEMORY;
    } catch (...) {
        g_create_error = "unexpected exception";
        return MT3D_CUDA_ERROR;
    }
}

int mt3d_fwdsolve_multi(int nh, mt3d_handle *hs, const int *nrhs, const double *const *omegas,
                        const int *const *trans, const double *const *bc, const double *const *src, double *const *e,
                        int *const *status, const int *zchunks)
{
    return fwdsolve_multi_entry(nh, hs, nrhs, omegas, trans, bc, src, e, status, zchunks, false);
}

int mt3d_fwdsolve_multi_device(int nh, mt3d_handle *hs, const int *nrhs, const double *const *omegas,
                               const int *const *trans, const double *const *bc_dev, const double *const *src_dev,
                               double *const *e_dev, int *const *status, const int *zchunks)
{
    return fwdsolve_multi_entry(nh, hs, nrhs, omegas, trans, bc_dev, src_dev, e_dev, status, zchunks, true);
}

int mt3d_set_fused(mt3d_handle h, int on)
{
    return wrap(h, [&] { return h->s.set_fused(on); });
}

int mt3d_set_poly(mt3d_handle h, double c)
{
    return wrap(h, [&] { return h->s.set_poly(c); });
}

int mt3d_set_wait_limit(mt3d_handle h, int polls)
{
    return wrap(h, [&] { return h->s.set_wait_limit(polls); });
}

int mt3d_apply_kernel(mt3d_handle h, int kernel, const double *x, double *y)
{
    return wrap(h, [&] { return h->s.apply_kernel(kernel, x, y); });
}

int mt3d_profile(mt3d_handle h, int enable)
{
    return wrap(h, [&] { return h->s.profile(enable); });
}

int mt3d_kernel_time(mt3d_handle h, int precision, int *launches, double *ms, int64_t *rhs_sweeps)
{
    return wrap(h, [&] { return h->s.kernel_time(precision, launches, ms, rhs_sweeps); });
}

int mt3d_get_diag(mt3d_handle h, int *nIterTotal, int *nDivCor, int *failed, double *EMrelErr, int len, double *divJ,
                  int lenDivJ, double *final_relres)
{
    if (!h) return MT3D_INVALID_ARGUMENT;
    const mt3d::Diag &d = h->s.diag;
    if (nIterTotal) *nIterTotal = d.nIterTotal;
    if (nDivCor) *nDivCor = d.nDivCor;
    if (failed) *failed = d.failed;
    if (EMrelErr && len > 0) {
        const int n = std::min<int>(len, (int)d.EMrelErr.size());
        std::memcpy(EMrelErr, d.EMrelErr.data(), n * sizeof(double));
        for (int i = n; i < len; i++) EMrelErr[i] = 0.0;
    }
    if (divJ && lenDivJ > 0) {
        const int n = std::min<int>(2 * lenDivJ, (int)d.divJ.size());
        std::memcpy(divJ, d.divJ.data(), n * sizeof(double));
        for (int i = n; i < 2 * lenDivJ; i++) divJ[i] = 0.0;
    }
    if (final_relres) *final_relres = d.final_relres;
    return MT3D_OK;
}

int mt3d_get_batch_diag(mt3d_handle h, int nrhs, int *niter, double *relres)
{
    if (!h || nrhs < 0) return MT3D_INVALID_ARGUMENT;
    const int n = std::min<int>(nrhs, (int)h->s.batch_niter.size());
    for (int r = 0; r < nrhs; r++) {
        if (niter) niter[r] = r < n ? h->s.batch_niter[r] : 0;
        if (relres) relres[r] = r < n ? h->s.batch_relres[r] : 0.0;
    }
    return MT3D_OK;
}

int mt3d_pmult_t(mt3d_handle h, int npol, const double *e0, const double *eadj, const double *m0_earth, double *dm)
{
    return wrap(h, [&] { return h->s.pmult_t(npol, e0, eadj, m0_earth, dm); });
}

int64_t mt3d_launch_counter(void) { return mt3d::g_launch_count.load(); }

int64_t mt3d_alloc_counter(void) { return mt3d::g_alloc_count.load(); }

int mt3d_write_soln(mt3d_handle h, const char *path, int nTx, int nPol, const double *omegas, const double *origin,
                    double rotdeg, const double *e, int device)
{
    return wrap(h, [&] { return h->s.write_soln(path, nTx, nPol, omegas, origin, rotdeg, e, device != 0); });
}

int mt3d_read_soln(mt3d_handle h, const char *path, int iTx, int iPol, double *omega, double *e, int device)
{
    return wrap(h, [&] { return h->s.read_soln(path, iTx, iPol, omega, e, device != 0); });
}

int mt3d_read_soln_header(const char *path, int *nTx, int *nPol, int *nx, int *ny, int *nz, int *nzAir, double *origin,
                          double *rotdeg, double *dx, double *dy, double *dz)
{
    try {
        return mt3d::read_soln_header(path, nTx, nPol, nx, ny, nz, nzAir, origin, rotdeg, dx, dy, dz, g_create_error);
    } catch (...) {
        g_create_error = "host out of memory";
        return MT3D_OUT_OF_MEMORY;
    }
}

int mt3d_last_error(mt3d_handle h, char *buf, int len)
{
    if (!buf || len < 1) return MT3D_INVALID_ARGUMENT;
    const std::string &m = h ? h->s.last_error : g_create_error;
    const int n = std::min<int>(len - 1, (int)m.size());
    std::memcpy(buf, m.data(), n);
    buf[n] = '\0';
    return MT3D_OK;
}

}  // extern "C"

// solver.h -- host-side solver object behind the C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "kernels.h"

namespace mt3d {

struct Control {
    int IterPerDivCor = 40;  // f90/3D_MT/FWD/EMsolve3D.f90:58-68 defaults
    int MaxDivCor = 20;
    int MaxIterDivCor = 100;
    double tolEMfwd = 1e-7;
    double tolEMadj = 1e-7;
    double tolDivCor = 1e-5;
    int solver = 1;     // 1: BiCGStab (reference BICG) + diagonal; 2: Bi-CG/COCG + z-line
    int precision = 0;  // 0 FP64, 1 mixed
    int formulation = 0;  // 0 curl-curl + divergence correction (MF), 1 curl-curl + grad-div (SP2)
    int restart = 120;    // grad-div formulation: BiCGStab restart length (cuBiCG's 120; 0 never)
    int fused = 1;        // mixed precision: FP32 iteration in preconditioned variables (hatkernels.cu)
    double poly = 0.0;    // fused iteration: polynomial preconditioner coefficient (0: diagonal alone)
};

struct Diag {
    int nIterTotal = 0, nDivCor = 0, failed = 0;
    std::vector<double> EMrelErr;
    std::vector<double> divJ;  // pairs
    double final_relres = 0.0;
};

class DevBuf {
  public:
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    int alloc(size_t bytes);
    void release();
    template <typename T> T *as() const { return reinterpret_cast<T *>(ptr_); }
    size_t bytes() const { return bytes_; }

  private:
    void *ptr_ = nullptr;
    size_t bytes_ = 0;
};

struct Workspace {
    int nrhs = 0;
    int precision = -1;
    int rlen = 0, dlen = 0;  // rerr row lengths the buffers were sized for
    int solver = 0;
    int formulation = 0;
    bool padded = false;  // FP32 vectors on the padded layout (TMA-staged kernels)
    // FP64 edge vectors [nrhs][nE]
    DevBuf b, X, x1, r, rt, p, v, ph, s, sh, t, bc, tmp;
    // FP32 edge vectors (mixed)
    DevBuf f_b, f_x0, f_x1, f_r, f_rt, f_p, f_v, f_ph, f_s, f_sh, f_t;
    // FP64 node vectors [nrhs][nN]
    DevBuf px, pr, pp, pq, phi0;
    DevBuf zm, zc, f_zm, f_zc;  // z-line pivots for BiCGStab + z-line
    DevBuf phi64, phi32;        // grad-div node potentials
    DevBuf jinv64, jinv32;      // inverse diagonal (diagonal preconditioner)
    DevBuf bst, pst, ost, qst, parts, cnt, rerr, dcrerr;
};

// state of one FWDsolve3D call over a batch between its phases (solve_begin,
// solve_pre, solve_fp32, solve_post, solve_end); a multi-grid batch drives
// several of these in lockstep
struct SolveRun {
    int nrhs = 0, prec = 0;
    bool device = false, refine = false, done = false;
    bool n32 = false, n64 = false;  // groups of the current mixed-precision cycle
    double *e = nullptr;
    int *status = nullptr;
    std::vector<OuterState> os, grp;
    std::vector<Diag> dg;
    std::vector<BicgState> bs;
    std::vector<double> rerr, prev_relres, inner_best;
    std::vector<char> hi;
    std::vector<int> stalls;
    bool any_active() const;
};

// fixed scratch of mt3d_mult_aii_device_noalloc (noalloc.cu): resolved and
// committed once per device at handle creation
int noalloc_prepare(int dev, std::string &err);

class Solver;
// FWDsolve3D over the right-hand sides of several handles, the FP32 cycles
// of all grids in shared launches (multi.cu); zch: node-plane chunks of each
// grid's stencil blocks (NULL or 0 entries: the occupancy-based choice)
int fwdsolve_multi(int nh, Solver *const *hs, const int *nrhs, const double *const *omegas, const int *const *trans,
                   const double *const *bc, const double *const *src, double *const *e, int *const *status,
                   const int *zch, bool device, std::string &err);

// header of a solution file (solnio.cu); any output may be NULL
int read_soln_header(const char *path, int *nTx, int *nMode, int *nx, int *ny, int *nz, int *nzAir, double *origin,
                     double *rotdeg, double *dx, double *dy, double *dz, std::string &err);

class Solver {
  public:
    ~Solver();
    int create(int dev, int nx, int ny, int nz, int nzAir, const double *dx, const double *dy, const double *dz);
    int update_cond(const double *m_earth, double airCond);
    int update_freq(double omega);
    int mult_aii(int adjt, const double *x, double *y);
    int mult_aii_noalloc(int adjt, const double *x, double *y);  // device vectors, fixed scratch
    int apply_kernel(int kernel, const double *x, double *y);   // one internal operator kernel
    int bicg(const double *b, double *x, int maxit, double tol, int *niter, double *rerr, int *failed);
    int solve(int nrhs, const double *omegas, const int *trans, const double *bc, const double *src, double *e,
              int *status, bool device = false);
    int solve_begin(SolveRun &run, int nrhs, const double *omegas, const int *trans, const double *bc,
                    const double *src, double *e, int *status, bool device);
    int solve_pre(SolveRun &run);
    int solve_fp32(SolveRun &run);
    int solve_post(SolveRun &run);
    int solve_end(SolveRun &run);
    bool fp32_fused(const SolveRun &run) const;
    // multi-grid batches (multi.cu): the arguments of this handle's fused
    // FP32 cycle, its cast and end kernels, and its stream and device
    KArgs<float> hat_args(int nrhs);
    int hat_cycle_begin(int nrhs, KArgs<float> &a);
    // n profiling events of the FP32 stencil launches (null unless mt3d_profile is on)
    cudaEvent_t *fp32_events(int n);
    // maxit fused FP32 iterations of a multi-grid batch on stream s: one
    // captured graph (kept on this handle) or, when profiling, timed launches
    int run_hat_multi(const KArgs<float> *args, const int *nrhs, const int *zch, int ng, int maxit, cudaStream_t s);
    int hat_cycle_end(int nrhs, const KArgs<float> &a);
    cudaStream_t stream() const { return stream_; }
    int device() const { return dev_; }
    int set_stream(void *s);
    int set_wait_limit(int polls);
    int set_fused(int on);
    int set_poly(double c);
    int profile(int enable);
    int kernel_time(int precision, int *launches, double *ms, int64_t *sweeps);
    int get_cond(double *sigma_e, double *divcorr, double *node_w);
    int compute_bc(int imode, double omega, double *e0, bool device);
    int write_soln(const char *path, int nTx, int nPol, const double *omegas, const double *origin, double rotdeg,
                   const double *e, bool device);
    int read_soln(const char *path, int iTx, int iPol, double *omega, double *e, bool device);
    int pmult_t(int npol, const double *e0, const double *eadj, const double *m0, double *dm);
    int impedance(double omega, int nsite, const double *xyz, const double *origin, const double *e1, const double *e2,
                  double *Z, bool device);
    int lmult_t(double omega, int nsite, const double *xyz, const double *origin, const double *e1, const double *e2,
                const double *d, double *s1, double *s2, bool device);
    int jmult_t(double omega, int nsite, const double *xyz, const double *origin, const double *e0, const double *d,
                const double *m0, double *dm, double *eadj, bool device);
    int data_functional(double omega, int nsite, const double *xyz, const double *origin, const double *e1,
                        const double *e2, const double *d, double *Z, double *s1, double *s2, bool device);

    int fail(int code, const std::string &msg);
    std::string last_error;
    Control ctl;
    Diag diag;
    std::vector<int> batch_niter;
    std::vector<double> batch_relres;
    int nx = 0, ny = 0, nz = 0, nzAir = 0;
    int64_t nE = 0, nEi = 0, nN = 0;
    std::vector<int32_t> edgei;  // 0-based interior edge list
    double omega = 0.0;
    bool cond_set = false;

  private:
    int ensure_workspace(int nrhs, int precision);
    int ensure_fp64_krylov(int nrhs);
    int run_bicg(int nrhs, int precision, int maxit);
    int run_divcorr(int nrhs);
    int run_hat(int nrhs, int maxit);
    void push_state(SolveRun &run);
    int pull_state(SolveRun &run);
    template <typename T> KArgs<T> kargs(int nrhs, int precision_ws);
    template <typename T> ColArgs<T> cargs();
    DArgs dargs(int nrhs);
    int check(cudaError_t e, const char *what);
    int sync(const char *what);

    int dev_ = 0;
    cudaStream_t stream_ = nullptr;      // active stream (own or caller's)
    cudaStream_t own_stream_ = nullptr;  // created with the handle
    // kernel timing: pairs of events around the stencil launches
    bool prof_ = false;
    std::vector<cudaEvent_t> ev_;
    size_t ev_used_ = 0;
    int prof_launches_[2] = {0, 0}, prof_cur_ = 0;  // per precision (0 FP64, 1 FP32)
    double prof_ms_[2] = {0.0, 0.0};
    std::vector<int> ev_prec_;  // precision of each recorded event
    DevBuf prof_cnt_;           // device sweep counters [FP64, FP32]
    HatGraph hat_graph_, hat_graph_multi_;  // captured FP32 cycles (single grid, multi-grid batch)
    cudaEvent_t *next_events(int n);
    void collect_events();
    Geo<double> g64_{};
    Geo<float> g32_{};
    DevBuf tab64_, tab32_, sig64_, sig32_, coef_, edgei_d_;
    DevBuf sigs64_, sigs32_, gdw64_, gdw32_, gde_, gdn64_, gdn32_;  // grad-div (SP2) data
    DevBuf setup_;  // model parameter, V_C, V_C sigma_C and sigma_C of the operator set-up
    DevBuf bcs_, bce_;  // 2-D boundary-condition scratch and host-bound output
    // padded FP32 layout of the TMA-staged kernels: sigma of both
    // formulations, signed node weights, the tensor maps and a device flag
    // that bounded waits set
    PadLayout pl_{};
    DevBuf sigP32_, sigsP32_, gdnP32_, errf_;
    TmaMaps *tma_ = nullptr;
    int wait_limit_ = 1 << 22;  // polls of a bounded device-side wait
    bool tma_stale_ = true;
    int tma_ready();
    int check_device_error(const char *what);
    Workspace ws_;
    std::vector<double> dx_, dy_, dz_, delX_, delY_, delZ_;
};

}  // namespace mt3d

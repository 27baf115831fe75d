// kernels.h -- kernel argument blocks and launchers (host-visible).
#pragma once
#include <vector>

#include "common.cuh"

namespace mt3d {

// Padded layout of the FP32 Krylov vectors for the TMA-staged kernels: each
// component is a Px x Py x Pz block (Px = nx + 1 rounded up to 4, Py = ny + 1,
// Pz = nz + 1), entry (c, i, j, k) at ((c Pz + k) Py + j) Px + i; entries
// outside the component's range are zero.  Rows are 16-byte multiples, which
// the TMA tensor maps need and the reference's own order (rows of nx and
// nx + 1) does not give.
struct PadLayout {
    int Px, Py, Pz;
    __host__ __device__ int idx(int c, int i, int j, int k) const { return ((c * Pz + k) * Py + j) * Px + i; }
    __host__ __device__ long long len() const { return 3LL * Px * Py * Pz; }
};

// tiles of kColX x kColY (i, j) columns for the column-marching kernels
struct ColMap {
    int tiles_x, tiles;
};
using ColMapHost = ColMap;
ColMapHost col_map(int nx, int ny);

// arguments of the edge-vector Krylov kernels (one precision T)
template <typename T> struct KArgs {
    Geo<T> g;
    const T *sigma;   // edge conductivity of the forward operator (air zeroed)
    OuterState *ost;  // per right-hand side: omega, activity, tolerances
    BicgState *st;
    C2<T> *r, *rt, *p, *v, *ph, *s, *sh, *t, *x0, *x1;
    const C2<T> *b;
    double *parts;
    unsigned *cnt;
    double *rerr;  // [nrhs][rerr_stride]
    int rerr_stride;
    size_t stride;  // elements between right-hand sides
    int chunk, nblk;
    int maxit;
    int inner;    // 1: tolerance from OuterState::tol_inner (mixed inner solve)
    int pc_ext;   // 1: ph / sh come from an external preconditioner kernel
    int restart;  // restart BiCGStab every `restart` iterations (0: never)
    // grad-div term (SP2 formulation): gd != 0 adds DFA G phi, phi computed by
    // launch_gd_phi from the stencil input; gdw / gde node weights and flags
    int gd;
    const T *gdw;
    const unsigned char *gde;
    const T *gdn;  // node weight with the earth flag as its sign (staged kernels)
    C2<T> *phi;
    // stencil kernels: 0 flat, 1 column-marching, 2 shared-memory staged
    // (grad-div potentials formed inside), 3 TMA-staged on the padded layout;
    // the precomputed inverse diagonal
    int colstencil;
    ColMap cmap;
    C2<T> *jinv;
    double dsgn;  // ISIGN (-1) for A, +1 for the conjugate transpose
    // entries per right-hand side swept by the elementwise kernels (nE, or
    // the padded length) and the padded layout of the vectors (padded != 0)
    int len;
    int padded;
    PadLayout pl;
    int *err;        // set by a bounded device-side wait that gave up
    int wait_limit;  // polls of one bounded wait before it gives up
    const struct TmaMaps *tma;  // host pointer: tensor maps of the padded vectors (colstencil == 3)
    // profiling: the staged stencil kernels count one sweep per active
    // right-hand side and launch here (nullptr when not profiling)
    unsigned long long *sweeps;
    // QMR: scalar state and the vectors of the reference's routine that
    // BiCGStab has no place for
    QmrState *qst;
    C2<T> *q, *w, *d;
    // fused FP32 iteration: coefficient c of the polynomial preconditioner
    // c D^-1 (2 I - c A D^-1) (0: the diagonal preconditioner alone)
    float pc;
};

// arguments of the divergence-correction kernels (FP64)
struct DArgs {
    Geo<double> g;
    const double *sigma;  // edge conductivity (air zeroed), as DivC uses it
    const double *coef;   // 7 node arrays (SoA): db1x db2x db1y db2y db1z db2z c
    OuterState *ost;
    PcgState *pst;
    double2 *E;            // fields being corrected [nrhs][estride]
    const double2 *phi0;   // scaled source divergence or null [nrhs][stride]
    double2 *px, *pr, *pp, *pq;
    double *parts;
    unsigned *cnt;
    double *rerr;
    int rerr_stride;
    size_t stride;   // node vector stride
    size_t estride;  // edge vector stride
    int chunk, nblk;    // node chunking
    int echunk, enblk;  // edge chunking
    int maxit;
    double tol;
};


template <typename T> struct ColArgs {
    Geo<T> g;
    const T *sigma;
    OuterState *ost;
    BicgState *st;
    ColMap map;
    C2<T> *r, *z, *p, *q, *x0, *x1;
    C2<T> *zm, *zc;  // z-line pivots m_k and c'_k (per right-hand side)
    double *parts;
    unsigned *cnt;
    double *rerr;
    int rerr_stride;
    size_t stride;
    double dsgn;
};
template <typename T> void launch_col_apply(const ColArgs<T> &a, const C2<T> *x, C2<T> *y, int neg, int nrhs,
                                            cudaStream_t s);
template <typename T> void launch_zl_setup(const ColArgs<T> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_cocg_start(const ColArgs<T> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_col_prec(const ColArgs<T> &a, const C2<T> *in, C2<T> *out, int nrhs, cudaStream_t s);
template <typename T> void launch_colb_init(const KArgs<T> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_colb_vt(const KArgs<T> &a, int which, int nrhs, cudaStream_t s);
void launch_colb_res64(const KArgs<double> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_colb_jacobi(const KArgs<T> &a, int nrhs, cudaStream_t s);
// shared-memory staged stencil kernels (colstencil == 2; grad-div potentials fused)
template <typename T> void launch_stage_init(const KArgs<T> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_stage_vt(const KArgs<T> &a, int which, int nrhs, cudaStream_t s);
void launch_stage_res64(const KArgs<double> &a, int nrhs, cudaStream_t s);
// TMA-staged FP32 stencil kernels on the padded layout (colstencil == 3):
// tensor maps of the input vectors, of sigma and of the signed node weights
struct TmaMaps;
int tma_maps_build(TmaMaps *m, const float2 *x0, const float2 *ph, const float2 *sh, const float2 *pw,
                   const float2 *sw, const float *sig, const float *gdn, PadLayout pl, int nrhs);
TmaMaps *tma_maps_new();
void tma_maps_free(TmaMaps *m);
void launch_tma_init(const KArgs<float> &a, const TmaMaps *m, int nrhs, cudaStream_t s);
void launch_tma_vt(const KArgs<float> &a, const TmaMaps *m, int which, int nrhs, cudaStream_t s);
// the fused FP32 BiCGStab iteration in preconditioned variables (hatkernels.cu)
void launch_hat_cast(const KArgs<float> &a, const double2 *r64, size_t stride64, int nrhs, cudaStream_t s);
void launch_hat_iter(const KArgs<float> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev = nullptr);
void launch_hat_apply(const KArgs<float> &a, int nrhs, cudaStream_t s);
// with the polynomial preconditioner: the cycle's iterate x = M^-1 yhat in x0
// (after launch_bicg_finish); nothing otherwise
void launch_hat_conv(const KArgs<float> &a, int nrhs, cudaStream_t s);
// One FP32 cycle of the fused iteration (maxit iterations of launch_hat_iter,
// or of launch_hat_iter_multi over ng grids) captured as a CUDA graph and
// replayed while the launch arguments stay the same; the graph is captured
// on a private stream and launched on the caller's.
struct HatGraph {
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap = nullptr;
    std::vector<unsigned char> key;
    long long launches = 0;  // kernel launches in one replay
    void reset();
    ~HatGraph();
};
// ng = 0: one grid (args[0], nrhs[0]); returns a CUDA error code
cudaError_t hat_graph_run(HatGraph &hg, const KArgs<float> *args, const int *nrhs, const int *zch, int ng, int maxit,
                          cudaStream_t s);
int launch_hat_iter_multi(const KArgs<float> *args, const int *nrhs, const int *zch, int ng, cudaStream_t s,
                          cudaEvent_t *ev = nullptr);
void launch_cast_padded(const Geo<double> &g, const OuterState *ost, size_t stride64, const double2 *r64,
                        PadLayout pl, float2 *b32, float2 *x32, int nrhs, cudaStream_t s);
void launch_update_padded(const Geo<double> &g, const OuterState *ost, size_t stride64, PadLayout pl,
                          const float2 *d32, double2 *X, int nrhs, cudaStream_t s);
void launch_to_padded(const Geo<double> &g, const double *src, PadLayout pl, float *dst, cudaStream_t s);
// conductivity-dependent operator set-up from the model parameter (setupkernels.cu);
// VC, CT, sigC: [nx*ny*nz] (cell volume, volume x conductivity, conductivity); coef: [7][nN]
void launch_setup_cond(const Geo<double> &g, const double *m_earth, double airCond, double *VC, double *CT,
                       double *sigC, double *sig, double *sigs, double *gdw, unsigned char *gde, double *gdn,
                       double *coef, float *sig32, float *sigs32, float *gdw32, float *gdn32, cudaStream_t s);

// 2-D TE boundary conditions (bc2d.cu)
struct BcArgs {
    int imode;         // 2: x-slices, field on the x-edges; 1: y-slices, field on the y-edges
    int nh, nz, nza;   // horizontal cells of a slice, vertical cells (air first), air cells
    int nslice, slice0;
    int nx, ny, nXe;   // 3-D grid; nXe = offset of the y-edges
    double omue;       // omega mu0
    const double *dh, *dz, *sigC;
    double2 *side;     // [nslice][2][nz+1] side columns
    double2 *cpr;      // [nslice][2][nz] elimination scratch of the side columns
    double2 *bottom;   // [nslice][nh+1] bottom node of each interior column
    double2 *U, *y;    // [chunk][n][nz], [chunk][n]: U rows and reduced right-hand side
    double2 *cd, *cb;  // [chunk][n] operator diagonal and right-hand side
    double *czc, *cyc; // [chunk][n] couplings A(r, r+1) and A(r, r+nz-1)
    double2 *W;        // [chunk][nz][nz] elimination window when it is not in shared memory
    double2 *e0;       // full edge vector (zeroed by the caller)
};
size_t bc_smem_bytes(int nz, bool window_in_smem);
void launch_bc1d(const BcArgs &a, cudaStream_t s);
void launch_bc_coef(const BcArgs &a, int nslices, cudaStream_t s);
void launch_bc_back(const BcArgs &a, int nslices, cudaStream_t s);
int launch_bc2d(const BcArgs &a, int nblocks, bool window_in_smem, cudaStream_t s);
void launch_nodes_to_padded(const Geo<double> &g, const double *src, PadLayout pl, float *dst, cudaStream_t s);
int stage_chunks(int nz, int tiles, int resident);
template <typename T> void launch_cocg_iter(const ColArgs<T> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev = nullptr);

template <typename T>
void launch_apply(const KArgs<T> &a, const C2<T> *x, C2<T> *y, int neg, int nrhs, cudaStream_t s, int use_gd = 0);
template <typename T> void launch_bicg_init(const KArgs<T> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_bicg_iter(const KArgs<T> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev = nullptr,
                                            const ColArgs<T> *pc = nullptr);
template <typename T> void launch_bicg_finish(const KArgs<T> &a, int nrhs, cudaStream_t s);
// QMR (FP64, diagonal preconditioner M1 = D, M2 = I) in the BiCGStab call's
// place: start, one iteration (six launches), end (statuses into BicgState)
void launch_qmr_init(const KArgs<double> &a, int nrhs, cudaStream_t s);
void launch_qmr_iter(const KArgs<double> &a, int nrhs, cudaStream_t s);
void launch_qmr_finish(const KArgs<double> &a, int nrhs, cudaStream_t s);
template <typename T> void launch_gd_phi(const KArgs<T> &a, const C2<T> *x, C2<T> *phi, int mode, int nrhs, cudaStream_t s);
template <typename T> void launch_gd_add(const KArgs<T> &a, C2<T> *b, const C2<T> *phi, int nrhs, cudaStream_t s);
void launch_norm_b(const KArgs<double> &a, int nrhs, cudaStream_t s);
void launch_res64(const KArgs<double> &a, int nrhs, cudaStream_t s);
void launch_cast(const OuterState *ost, int nE, size_t stride, const double2 *r64, float2 *b32, float2 *x32, int nrhs,
                 cudaStream_t s);
void launch_update(const OuterState *ost, int nE, size_t stride, const float2 *d32, double2 *X, int nrhs, cudaStream_t s);
void launch_divcorr_start(const DArgs &a, int nrhs, cudaStream_t s);
void launch_divcorr_iter(const DArgs &a, int nrhs, cudaStream_t s);
void launch_divcorr_finish(const DArgs &a, int nrhs, cudaStream_t s);
void launch_keep_boundary(const Geo<double> &g, double2 *v, size_t stride, int nrhs, cudaStream_t s);
void launch_keep_interior(const Geo<double> &g, double2 *v, size_t stride, int nrhs, cudaStream_t s);
void launch_add_src(const Geo<double> &g, double2 *b, const double2 *src, size_t stride, const OuterState *ost, int nrhs,
                    cudaStream_t s);
void launch_phi0(const Geo<double> &g, const double2 *src, size_t estride, double2 *phi0, size_t nstride,
                 const OuterState *ost, int nrhs, cudaStream_t s);
void launch_post(const Geo<double> &g, double2 *E, const double2 *bc, size_t stride, const OuterState *ost, int nrhs,
                 cudaStream_t s);
void launch_pmult_t(const Geo<double> &g, int npol, const double2 *e0, const double2 *ea, double omega, const double *m0,
                    double *dm, cudaStream_t s);
void launch_nonzero(const double2 *v, size_t stride, int n, int *flags, int nrhs, cudaStream_t s);
void launch_scatter_interior(int nEi, const int *edgei, const double2 *vi, double2 *vf, cudaStream_t s);
// load the modules of the FP64 operator-apply kernels (cudaFuncGetAttributes)
cudaError_t preload_apply_kernels();
void launch_gather_interior(int nEi, const int *edgei, const double2 *vf, double2 *vi, cudaStream_t s);

}  // namespace mt3d

/*
 * mt3d.h -- C ABI of the B200-native 3D magnetotelluric forward/adjoint
 * solver (libmt3d.so).
 *
 * The library replaces the solver calls of ModEM's 3D-MT forward problem:
 * the model-operator set-up (modelOperator3D), the Krylov call BICG/cuBiCG
 * and the driver FWDsolve3D with its divergence correction SdivCorr.  The
 * Fortran host keeps its types; a thin ISO_C_BINDING shim flattens them
 * with getCVector and calls the functions below.
 *
 * Conventions
 *  - Complex arrays are interleaved (re, im) doubles, i.e. the memory layout
 *    of Fortran complex(kind=8) and C double _Complex.
 *  - A "full edge vector" has nE = nx(ny+1)(nz+1) + (nx+1)ny(nz+1) +
 *    (nx+1)(ny+1)nz complex entries in ModEM's getCVector order
 *    (f90/3D_MT/SP_Topology/vecTranslate.f90:41-79): all x-edges, then all
 *    y-edges, then all z-edges, each block column-major (x fastest).
 *  - An "interior vector" has nEi entries: the interior edges in ascending
 *    full-edge order, i.e. the EDGEi list of boundaryIndex
 *    (vecTranslate.f90:436-526).
 *  - Model parameters are ln(sigma) (paramType LOGE) of the nx*ny*nzEarth
 *    earth cells, x fastest; the air cells take exp(airCond).
 *  - Every function returns an mt3d_status; nothing aborts the host process.
 *    mt3d_last_error() returns the message of the last failure on a handle.
 *  - A handle owns one CUDA stream and its device memory; it is not thread
 *    safe.  Host buffers are only borrowed for the duration of a call.
 */
#ifndef MT3D_H
#define MT3D_H

#include <stdint.h>

#if defined(__GNUC__)
#define MT3D_API __attribute__((visibility("default")))
#else
#define MT3D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mt3d_solver *mt3d_handle;

typedef enum {
    MT3D_OK = 0,               /* converged */
    MT3D_NOT_CONVERGED = 1,    /* iteration limits reached; best iterate returned */
    MT3D_BREAKDOWN = 2,        /* Krylov breakdown (rho, alpha, omega or beta zero) */
    MT3D_NAN_INPUT = 3,        /* NaN/Inf in the right-hand side or model */
    MT3D_CUDA_ERROR = 4,       /* a CUDA runtime call failed */
    MT3D_INVALID_ARGUMENT = 5, /* bad sizes, null pointers, unknown options */
    MT3D_DEVICE_TIMEOUT = 6,   /* a bounded device-side wait gave up */
    MT3D_NO_DEVICE = 7,        /* no usable CUDA device / library built without one */
    MT3D_OUT_OF_MEMORY = 8
} mt3d_status;

/* Krylov solver and precision choices */
/* MT3D_SOLVER_BICG: BiCGStab as in the reference's BICG with the diagonal
 * preconditioner.  MT3D_SOLVER_COCG: Bi-CG specialised to the complex-
 * symmetric operator (conjugate-orthogonal CG, one operator application per
 * iteration) with the vertical-line (z-line) tridiagonal preconditioner.
 * MT3D_SOLVER_BICG_ZLINE: BiCGStab with the z-line preconditioner.
 * MT3D_SOLVER_QMR: QMR without look-ahead, the reference's default solver
 * (QMR, f90/3D_MT/FWD/solver.f90:122-343; solver_name "QMR",
 * f90/3D_MT/FWD/EMsolve3D.f90:70), with the diagonal preconditioner as M1
 * and M2 = I; FP64 only. */
enum { MT3D_SOLVER_BICG = 1, MT3D_SOLVER_COCG = 2, MT3D_SOLVER_BICG_ZLINE = 3, MT3D_SOLVER_QMR = 4 };
enum { MT3D_PREC_FP64 = 0, MT3D_PREC_MIXED = 1 };

/* Library version string. */
MT3D_API const char *mt3d_version(void);

/* Number of CUDA devices visible (0 when none); replaces kernelc_getDevNum
 * (f90/3D_MT/FWD_SP2/kernel_c.cu:463-500). */
MT3D_API int mt3d_device_count(void);

/* Create a solver for one grid on device `device_id`.  Replaces
 * ModelDataInit + ModelOperatorSetUp (f90/3D_MT/FWD/modelOperator3D.f90:139-175,
 * f90/3D_MT/FWD/EMsolve3D.f90:497-512): metric elements and the curl-curl
 * coefficients are set up here.  dz lists the nzAir air layers first. */
MT3D_API int mt3d_create(int device_id, int nx, int ny, int nz, int nzAir, const double *dx, const double *dy,
                const double *dz, mt3d_handle *out);

/* Release all device memory of the handle (ModelDataCleanUp,
 * f90/3D_MT/FWD/modelOperator3D.f90:177-194). */
MT3D_API int mt3d_destroy(mt3d_handle h);

/* Solver control (setEMsolveControl / readEMsolveControl,
 * f90/3D_MT/FWD/EMsolve3D.f90:690-844): iterations per divergence correction,
 * maximum number of divergence corrections, maximum PCG iterations per
 * correction, forward / adjoint / div-correction tolerances, Krylov solver
 * (MT3D_SOLVER_BICG) and precision (MT3D_PREC_FP64 or MT3D_PREC_MIXED: complex
 * FP32 inner iterations wrapped in FP64 iterative refinement). */
MT3D_API int mt3d_set_control(mt3d_handle h, int IterPerDivCor, int MaxDivCor, int MaxIterDivCor, double tolEMfwd,
                     double tolEMadj, double tolDivCor, int solver, int precision);

/* Discretised system.  MT3D_FORM_CCDC: the curl-curl operator of the
 * matrix-free solver (f90/3D_MT/FWD/modelOperator3D.f90) with the divergence
 * correction SdivCorr every IterPerDivCor iterations (FWDsolve3D of
 * f90/3D_MT/FWD/EMsolve3D.f90).  MT3D_FORM_CCGD: curl-curl plus the grad-div
 * term of GradDivSetup2 (f90/3D_MT/FWD_SP2/modelOperator3D.f90:916-1008), no
 * divergence correction, BiCGStab restarted every 120 iterations and checked
 * against the true residual (FWDsolve3D + cuBiCG of f90/3D_MT/FWD_SP2); there
 * IterPerDivCor x MaxDivCor bounds the total iterations.  Both have the same
 * discrete solution. */
enum { MT3D_FORM_CCDC = 0, MT3D_FORM_CCGD = 1 };
MT3D_API int mt3d_set_formulation(mt3d_handle h, int formulation);

/* Restart length of BiCGStab in the grad-div formulation: cuBiCG restarts
 * every 120 iterations (f90/3D_MT/FWD_SP2/solver.f90:1545-1573), the default
 * here; 0 restarts only at the start of each IterPerDivCor-iteration cycle,
 * whose true-residual check restarts the iteration anyway.  On the
 * 200 x 200 x 100 random-field benchmark 0 takes 14 % fewer iterations. */
MT3D_API int mt3d_set_restart(mt3d_handle h, int restart);

/* The FP32 iteration of the mixed-precision BiCGStab (MT3D_PREC_MIXED with
 * MT3D_SOLVER_BICG).  on != 0 (default): the iteration runs in
 * preconditioned variables (u = D^-1 p, D^-1 r, D^-1 v, ...) with the
 * diagonal preconditioner fused into the operator kernels, 163 bytes of
 * memory traffic per edge and iteration; 0: the kernels that keep the
 * reference's variables (the preconditioned vectors formed in separate
 * passes), 211 bytes.  Both are BiCGStab with the diagonal preconditioner of
 * BICG (f90/3D_MT/FWD/solver.f90:346-555) and the shadow rt = r0; they
 * differ in rounding.  No counterpart in the reference. */
MT3D_API int mt3d_set_fused(mt3d_handle h, int on);

/* Polynomial preconditioner of the fused FP32 iteration: c > 0 replaces the
 * diagonal preconditioner D^-1 by the first-degree Neumann polynomial
 * M^-1 = c D^-1 (2 I - c A D^-1), two operator applications per
 * preconditioned product (4 stencil launches an iteration instead of 2).
 * c = 0 (default) keeps D^-1 alone.  c must lie in [0, 1.5]; an eigenvalue
 * z of A D^-1 becomes 1 - (1 - c z)^2, so c below 2 / max|z| keeps the
 * spectrum off zero, and c = 1 is the truncated Neumann series.  Applies
 * to MT3D_PREC_MIXED with
 * the fused iteration (mt3d_set_fused on); the FP64 refinement and the FP64
 * fall-back keep D^-1.  No counterpart in the reference. */
MT3D_API int mt3d_set_poly(mt3d_handle h, double c);

/* Set the conductivity model (UpdateCond, f90/3D_MT/FWD/modelOperator3D.f90:
 * 211-232): ModelParamToEdge (LOGE, ModelMap.inc:88-188) and DivCorrSetUp. */
MT3D_API int mt3d_update_cond(mt3d_handle h, const double *m_earth, double airCond);

/* Read back the conductivity-dependent operator data that mt3d_update_cond
 * built on the device -- the public module variables of the reference's
 * operator, for checking and for callers that need them:
 *   sigma_e [nE]   Sigma_E as the curl-curl operator uses it, the air edges
 *                  zero (f90/3D_MT/FWD/modelOperator3D.f90:1598-1605);
 *   divcorr [7*nN] DivCorrSetUp's db1%x, db2%x, db1%y, db2%y, db1%z, db2%z
 *                  and c (:1538-1650) per node, in that order; entry k of the
 *                  block of db1%x is the coefficient of node k (0 off the
 *                  interior nodes);
 *   node_w [nN]    the grad-div node weight of the SP2 operator with the air
 *                  nodes' sign (GradDivSetup2, f90/3D_MT/FWD_SP2/
 *                  modelOperator3D.f90:916-1008): -w at an earth node, +w in
 *                  the air.
 * Any of the three may be NULL. */
MT3D_API int mt3d_get_cond(mt3d_handle h, double *sigma_e, double *divcorr, double *node_w);

/* Boundary conditions and first guess of the forward problem for one
 * polarisation: ComputeBC -> BC_x0_WS (f90/3D_MT/FWD/modelOperator3D.f90:
 * 268-293, f90/3D_MT/FWD/boundary_ws.f90:21-168), 2-D TE solutions on the
 * slices of the model with 1-D TE solutions on their edges, computed on the
 * device from the conductivity of mt3d_update_cond.  imode = 2 fills the
 * x-edges (x-slices), imode = 1 the y-edges (y-slices).  e0 (full edge vector,
 * nE complex) receives E0 with the tangential field of the bottom face zero:
 * pass it to mt3d_fwdsolve as both bc (its boundary entries are the BC) and
 * e (its interior entries are the reference's first guess).
 * mt3d_compute_bc uses the handle's frequency and host memory;
 * mt3d_compute_bc_device takes omega and a device pointer. */
MT3D_API int mt3d_compute_bc(mt3d_handle h, int imode, double *e0);
MT3D_API int mt3d_compute_bc_device(mt3d_handle h, int imode, double omega, void *e0);

/* Set the angular frequency (UpdateFreq, f90/3D_MT/FWD/modelOperator3D.f90:
 * 196-204). */
MT3D_API int mt3d_update_freq(mt3d_handle h, double omega);

/* Sizes: number of edges, interior edges and nodes. */
MT3D_API int mt3d_sizes(mt3d_handle h, int64_t *nE, int64_t *nEi, int64_t *nN);

/* Interior edge list EDGEi, 1-based like the Fortran (boundaryIndex,
 * f90/3D_MT/SP_Topology/vecTranslate.f90:436-526); `edgei` holds nEi entries. */
MT3D_API int mt3d_interior_index(mt3d_handle h, int32_t *edgei);

/* y = A x on interior vectors, A = V_E (curl curl + ISIGN i omega mu0 sigma)
 * (Mult_Aii, f90/3D_MT/FWD_SP2/modelOperator3D.f90:415-436; the same
 * operator as MultA_N, f90/3D_MT/FWD/modelOperator3D.f90:879-918), plus the
 * grad-div term in MT3D_FORM_CCGD.  With adjt != 0 the conjugate-transposed
 * operator is applied: AAii^T x - i ISIGN VomegaMuSig x as Mult_Aii(adjt)
 * forms it, including the transpose of the (unsymmetric) grad-div term. */
MT3D_API int mt3d_mult_aii(mt3d_handle h, int adjt, const double *x, double *y);

/* The product of mt3d_mult_aii on DEVICE vectors, allocating no device
 * memory.  This entry has no counterpart in the reference.  It is meant for
 * callers that drive the operator from their own iterative loop on vectors
 * they already hold on the GPU and that cannot allocate per call: a memory
 * pool or caching allocator that owns all free device memory, or a loop in
 * which the device-wide synchronisation of cudaMalloc/cudaFree is unwanted.
 *
 * x and y are interior vectors (nEi complex doubles, 16-byte aligned) in
 * device memory of the handle's device.  The work is only enqueued on the
 * handle's stream (mt3d_set_stream); y is ready when that stream reaches
 * this point.  The scratch (two full edge vectors, the grad-div node
 * potentials and a state record) is one fixed 16 MiB device array per
 * device: grids whose 256 + 16 * (2 nE + nN) bytes exceed it (about 52^3
 * cells) are rejected with MT3D_INVALID_ARGUMENT.  The first mt3d_create on
 * a device looks up the scratch address (cudaGetSymbolAddress), which is
 * what commits the array's 16 MiB, and loads the kernels of this entry, so
 * this entry takes no device memory on any call; create the handle before a
 * memory pool takes the device's free memory.  The scratch is shared by all
 * handles on a device, so calls whose GPU work overlaps in time (different
 * streams, handles or host threads) race; calls on one stream are safe.
 * With adjt != 0 the product is the conjugate transpose, as mt3d_mult_aii's. */
MT3D_API int mt3d_mult_aii_device_noalloc(mt3d_handle h, int adjt, const double *x, double *y);

/* One Krylov call on the interior system A x = b: BICG(b, x, KSSiter,
 * device_id) -> cuBiCG (f90/3D_MT/FWD_SP2/EMsolve3D.f90:369-387,
 * f90/3D_MT/FWD_SP2/solver.f90:931-2009; algorithm of BICG,
 * f90/3D_MT/FWD/solver.f90:346-555) with the diagonal preconditioner.
 * b and x are interior vectors; x holds the initial guess on entry and the
 * solution (or the best iterate) on return.  rerr (maxit entries, may be
 * NULL) receives the relative residual of every iteration; *niter and
 * *failed mirror KSSiter%niter and KSSiter%failed. */
MT3D_API int mt3d_bicg(mt3d_handle h, const double *b, double *x, int maxit, double tol, int *niter, double *rerr,
              int *failed);

/* The forward or transposed solve FWDsolve3D (f90/3D_MT/FWD/EMsolve3D.f90:
 * 116-391, entry point of f90/3D_MT/FWD_SP2/EMsolve3D.f90:129-501).
 *   trans = 0: forward problem; bc (full edge vector, boundary entries used)
 *              holds the tangential boundary field, src (full edge vector,
 *              interior entries used, may be NULL) an interior source already
 *              multiplied by -ISIGN i omega mu0.
 *   trans = 1: transposed problem; src is the adjoint source, bc optional
 *              boundary data.  Without a source (src NULL or zero) the
 *              interior solution is zero and no Krylov call runs (0
 *              iterations), as in f90/3D_MT/FWD_SP2/EMsolve3D.f90:233-245.
 *   A right-hand side that is zero otherwise (no boundary data, no source)
 *   gives a zero solution reported as one iteration with relative residual
 *   0, as BICG reports b = 0 (f90/3D_MT/FWD_SP2/solver.f90:780-786).
 *   e: full edge vector; interior entries are the initial guess on entry, the
 *      solution on return (boundary entries as in the reference's post-
 *      processing).  A transposed solve returns its interior entries
 *      multiplied by the edge volumes V_E, as FWDsolve3D does
 *      (EMsolve3D.f90:356-359), so its output is no first guess for
 *      another transposed solve.
 * Returns MT3D_OK when converged. */
MT3D_API int mt3d_fwdsolve(mt3d_handle h, int trans, const double *bc, const double *src, double *e);

/* Batched FWDsolve3D: nrhs independent right-hand sides on the handle's grid
 * and model, each with its own angular frequency omegas[r] and transposition
 * flag trans[r], solved together.  bc and src hold nrhs full edge vectors each
 * (either may be NULL; an individual vector may be all zero); e holds nrhs full
 * edge vectors (initial guess in, solution out); status[r] receives each
 * right-hand side's mt3d_status.  The handle's frequency (mt3d_update_freq) is
 * left unchanged.  1 <= nrhs <= 65535 (MT3D_INVALID_ARGUMENT otherwise, before
 * any buffer is read). */
MT3D_API int mt3d_fwdsolve_batch(mt3d_handle h, int nrhs, const double *omegas, const int *trans, const double *bc,
                        const double *src, double *e, int *status);

/* As mt3d_fwdsolve_batch, with bc, src and e in device memory of the
 * handle's device (no host copies; for callers that keep the fields resident
 * in HBM).  bc / src may be NULL. */
MT3D_API int mt3d_fwdsolve_batch_device(mt3d_handle h, int nrhs, const double *omegas, const int *trans,
                                        const double *bc_dev, const double *src_dev, double *e_dev, int *status);

/* FWDsolve3D over several grids at once: handle hs[i] (its own grid, model
 * and control) solves nrhs[i] right-hand sides with omegas[i], trans[i],
 * bc[i], src[i] and e[i] as mt3d_fwdsolve_batch takes them (bc, src, trans
 * or any entry may be NULL), status[i] receives their statuses.  Replaces the
 * reference's farm of (transmitter, polarisation) solves over MPI ranks
 * (f90/MPI/Main_MPI.f90:1444-1649) for models of uneven size on one GPU:
 * the handles' FWDsolve3D phases run in lockstep on the first handle's
 * stream and the FP32 iterations of all grids share their launches (five per
 * iteration for the whole batch, seven with the polynomial preconditioner).
 * Every handle must be on one device, in mixed precision with
 * MT3D_SOLVER_BICG and the fused FP32 iteration (mt3d_set_fused), with the
 * same IterPerDivCor and mt3d_set_poly coefficient; 1 to 8 handles.  zchunks
 * (nh entries, may be NULL; 0 = the occupancy-based default) sets how many
 * chunks of node planes each grid's stencil blocks split the column into --
 * the knob mt3d/tune.py tunes.  Errors are reported by mt3d_last_error(NULL)
 * and on hs[0].  No counterpart in the reference. */
MT3D_API int mt3d_fwdsolve_multi(int nh, mt3d_handle *hs, const int *nrhs, const double *const *omegas,
                                 const int *const *trans, const double *const *bc, const double *const *src,
                                 double *const *e, int *const *status, const int *zchunks);
/* As mt3d_fwdsolve_multi with bc, src and e in device memory. */
MT3D_API int mt3d_fwdsolve_multi_device(int nh, mt3d_handle *hs, const int *nrhs, const double *const *omegas,
                                        const int *const *trans, const double *const *bc_dev,
                                        const double *const *src_dev, double *const *e_dev, int *const *status,
                                        const int *zchunks);

/* Run the handle's work on a caller-owned CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the handle's own stream.  The handle's own stream
 * is a blocking stream: it is ordered with the legacy default stream (whose
 * handle is also NULL, e.g. torch's default stream), so device buffers a
 * caller writes there are complete before the handle's next call reads them,
 * and its results are complete before later default-stream work uses them.
 * Work on other non-blocking streams must be ordered by the caller. */
MT3D_API int mt3d_set_stream(mt3d_handle h, void *stream);

/* Polls of one bounded device-side wait (the mbarrier waits of the FP32
 * stencil kernels) before it gives up and the call returns
 * MT3D_DEVICE_TIMEOUT; default 4194304.  0 makes every such wait give up at
 * once (the copies in flight are still waited for, under the default
 * limit, before a block exits).  No counterpart in the reference: a small
 * limit lets a caller check its handling of that status without any device
 * fault. */
MT3D_API int mt3d_set_wait_limit(mt3d_handle h, int polls);

/* y = A x on FULL edge vectors in host memory through one of the library's
 * internal operator kernels, for checking the kernels against each other and
 * against an independent operator (no counterpart in the reference; the
 * operator is the one of mt3d_mult_aii at the handle's formulation and
 * frequency, boundary entries of y zero):
 *   kernel 0  the FP64 edge-parallel apply behind mt3d_mult_aii;
 *   kernel 1  the shared-memory staged FP64 stencil of the FP64 BiCGStab;
 *   kernel 2  the TMA-staged FP32 stencil of the mixed-precision BiCGStab
 *             on its padded layout (x is rounded to complex FP32 first);
 *   kernel 3  the operator kernel of the fused FP32 iteration
 *             (mt3d_set_fused): y = D^-1 A x, D = diag(A), x rounded to FP32. */
MT3D_API int mt3d_apply_kernel(mt3d_handle h, int kernel, const double *x, double *y);

/* Kernel timing: with enable != 0 every launch of the BiCGStab stencil
 * kernels (v = A ph with the fused dot product) is bracketed by CUDA events
 * on the solver stream.  mt3d_kernel_time returns, for the launches of one
 * precision (0 FP64, 1 FP32) since the last enable, their number, their
 * summed device time in milliseconds and rhs_sweeps: the number of
 * (launch, right-hand side) pairs in which the staged stencil kernels swept a
 * still-running right-hand side, i.e. the stencil work in units of nE edges.
 * In a multi-grid batch (mt3d_fwdsolve_multi) the shared stencil launches
 * are timed on the first grid's handle and every handle counts its own
 * grid's sweeps.  Any output may be NULL. */
MT3D_API int mt3d_profile(mt3d_handle h, int enable);
MT3D_API int mt3d_kernel_time(mt3d_handle h, int precision, int *launches, double *ms, int64_t *rhs_sweeps);

/* Solver diagnostics of the last mt3d_fwdsolve (getEMsolveDiag,
 * f90/3D_MT/FWD/EMsolve3D.f90:866-876): total Krylov iterations, number of
 * divergence corrections, failure flag, the relative residual history
 * EMrelErr (up to len entries), divJ before/after each correction (pairs, up
 * to lenDivJ pairs) and the relative residual of the returned field. */
MT3D_API int mt3d_get_diag(mt3d_handle h, int *nIterTotal, int *nDivCor, int *failed, double *EMrelErr, int len,
                  double *divJ, int lenDivJ, double *final_relres);

/* Per right-hand-side diagnostics of the last solve (batched or not): the
 * total Krylov iterations and the true relative residual ||b - A e|| / ||b||
 * of each returned interior field; arrays of at least nrhs entries. */
MT3D_API int mt3d_get_batch_diag(mt3d_handle h, int nrhs, int *niter, double *relres);

/* Gradient with respect to ln(sigma) of the earth cells from background
 * fields e0 and adjoint fields eadj of npol polarisations (npol full edge
 * vectors each) at the handle's frequency: PmultT (f90/3D_MT/SolverSens.f90:
 * 63-116) followed by dEdgeToModelParam (f90/3D_MT/modelParam/ModelMap.inc:
 * 302-374).  m0_earth is the background model; dm receives nx*ny*nzEarth
 * values. */
MT3D_API int mt3d_pmult_t(mt3d_handle h, int npol, const double *e0, const double *eadj, const double *m0_earth,
                 double *dm);

/* Full impedance tensor at nsite sites from the fields of the two
 * polarisations at angular frequency omega: dataResp for Full_Impedance
 * (f90/3D_MT/DataFunc.f90:143-189) with the interpolation functionals
 * EinterpSetUp and BfromESetUp (f90/3D_MT/EMfieldInterp.f90:141-324,
 * 470-647), site azimuths zero.  xyz holds x, y, z per site (z positive down,
 * 0 at the Earth's surface) in the frame of the grid origin `origin` (ox, oy,
 * oz of the reference's grid: the first x and y nodes and the surface depth);
 * e1, e2 are full edge vectors (polarisations 1 and 2).  Z receives
 * Zxx, Zxy, Zyx, Zyy (complex, interleaved) per site: E / B in SI units. */
MT3D_API int mt3d_impedance(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                            const double *e1, const double *e2, double *Z);
/* As mt3d_impedance with e1 and e2 in device memory of the handle's device
 * (the fields stay in HBM; only the sites and Z cross the bus). */
MT3D_API int mt3d_impedance_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                                   const double *e1_dev, const double *e2_dev, double *Z);

/* Adjoint sources of the Full_Impedance functional: Lrows + LmultT
 * (f90/3D_MT/DataFunc.f90:465-869, f90/SENS/DataSens.f90:130-225) for the
 * same sites and background fields e1, e2 as mt3d_impedance.  d holds the
 * data weights per site (Zxx, Zxy, Zyx, Zyy, complex); s1, s2 (full edge
 * vectors, overwritten) receive sum_ij conj(d_ij) L_ij,k, the source of the
 * transposed solve of polarisation k, where L_ij,k = B^-1(k, j) (Le_i -
 * Z_i1 Lbx - Z_i2 Lby) is the derivative of Z_ij with respect to the field of
 * polarisation k. */
MT3D_API int mt3d_lmult_t(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                          const double *e1, const double *e2, const double *d, double *s1, double *s2);
/* As mt3d_lmult_t with e1, e2, s1, s2 in device memory (d and xyz on the host). */
MT3D_API int mt3d_lmult_t_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                                 const double *e1_dev, const double *e2_dev, const double *d, double *s1_dev,
                                 double *s2_dev);

/* E-field solution files in the reference's binary layout (write_solnVectorMTX
 * / read_solnVectorMTX, f90/3D_MT/ioMod/ioAscii.f90:493-597, with
 * FileWriteInit :188-215, FileReadInit f90/3D_MT/ioMod/ioBinary.f90:61-93,
 * EfileWrite / EfileRead :314-368): Fortran unformatted sequential records
 * (int32 length before and after each), a header with the grid, then per
 * transmitter j and polarisation k a record (omega, j, k, name) and the Ex,
 * Ey, Ez blocks of the full edge vector.  Files written by the reference on a
 * little-endian host read here and the other way round.
 *   mt3d_write_soln: e holds nTx * nPol full edge vectors (transmitter major)
 *     in host memory, or device memory when device != 0; omegas[nTx];
 *     origin[3] (grid%ox, oy, oz; may be NULL for zeros) and rotdeg go to the
 *     header; the polarisations of a two-polarisation file are named Ex, Ey.
 *   mt3d_read_soln: one full edge vector (transmitter iTx, polarisation iPol,
 *     1-based) into e (host, or device when device != 0) and its omega; the
 *     file's grid sizes must match the handle's.
 *   mt3d_read_soln_header: the header without a handle; any output may be
 *     NULL (dx, dy, dz take nx, ny, nz entries; nz includes the air).
 * Field components longer than 2^31 - 1 bytes (gfortran sub-records) are
 * refused. */
MT3D_API int mt3d_write_soln(mt3d_handle h, const char *path, int nTx, int nPol, const double *omegas,
                             const double *origin, double rotdeg, const double *e, int device);
MT3D_API int mt3d_read_soln(mt3d_handle h, const char *path, int iTx, int iPol, double *omega, double *e, int device);
MT3D_API int mt3d_read_soln_header(const char *path, int *nTx, int *nPol, int *nx, int *ny, int *nz, int *nzAir,
                                   double *origin, double *rotdeg, double *dx, double *dy, double *dz);

/* J^T d for one transmitter (one frequency, both polarisations) and the
 * Full_Impedance functional: JmultT_TX (f90/SENS/SensComp.f90:408-488) from
 * saved background fields, i.e. LmultT (as mt3d_lmult_t) of the data weights
 * d at the sites, the transposed solves of both polarisations (sensSolve with
 * TRN; as mt3d_fwdsolve_batch with trans = 1, zero first guess, under the
 * handle's control) and PmultT (as mt3d_pmult_t) at the background model
 * m0_earth.  The impedance functional does not depend on the conductivity, so
 * JmultT_TX's QmultT term is zero.  e0 holds the background fields of
 * polarisations 1 and 2 (two full edge vectors) at angular frequency omega;
 * xyz, origin and d are as for mt3d_lmult_t.  dm receives nx*ny*nzEarth
 * values (the real part, as JmultT_TX keeps); eadj (two full edge vectors,
 * may be NULL) the adjoint fields.  Returns MT3D_NOT_CONVERGED (with dm
 * formed from the best iterates) when a transposed solve reached its limits.
 * The misfit gradient of an inversion (gradient, f90/INV/INVcore.f90:141-206)
 * is -2/Ndata times the sum over transmitters of J^T applied to the
 * error-weighted residuals (d - dHat)/err^2. */
MT3D_API int mt3d_jmult_t(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                          const double *e0, const double *d, const double *m0_earth, double *dm, double *eadj);
/* As mt3d_jmult_t with e0, dm and eadj in device memory of the handle's
 * device (xyz, origin, d and m0_earth on the host). */
MT3D_API int mt3d_jmult_t_device(mt3d_handle h, double omega, int nsite, const double *xyz, const double *origin,
                                 const double *e0_dev, const double *d, const double *m0_earth, double *dm_dev,
                                 double *eadj_dev);

/* Number of kernel launches the library has issued in this process, over all
 * handles (no counterpart in the reference; for launch accounting). */
MT3D_API int64_t mt3d_launch_counter(void);

/* Number of device allocations (cudaMalloc) the library has made in this
 * process, over all handles (no counterpart in the reference; for checking
 * which calls allocate). */
MT3D_API int64_t mt3d_alloc_counter(void);

/* Message of the last error on the handle (NUL-terminated, truncated to len).
 * With h = NULL: the last error of this thread's calls that take no handle
 * (mt3d_create, mt3d_read_soln_header). */
MT3D_API int mt3d_last_error(mt3d_handle h, char *buf, int len);

#ifdef __cplusplus
}
#endif

#endif /* MT3D_H */

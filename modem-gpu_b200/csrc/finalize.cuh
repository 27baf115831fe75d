// finalize.cuh -- scalar updates of the Krylov state, done by the last block
// of a right-hand side after the block partials are reduced (shared by the
// flat and the column-marching kernels).
#pragma once
#include "common.cuh"

namespace mt3d {

// start of a BiCGStab call (BICG, f90/3D_MT/FWD/solver.f90:346-400): norms of
// b and r = b - A x, tolerance, zero right-hand side and good-enough-guess exits
__device__ inline void fin_init(BicgState &st, const double *tot, double *rerr, int maxit, double tol)
{
    const double bnorm = sqrt(tot[0]), rnorm = sqrt(tot[1]);
    st.iter = 0;
    st.maxit = maxit;
    st.xcur = 0;
    st.xbest = 0;
    st.imin = 0;
    st.first = 1;
    st.pad = 0;
    st.bnorm = bnorm;
    st.rnorm = rnorm;
    st.rnormin = rnorm;
    st.btol = tol * bnorm;
    st.rho1 = {1.0, 0.0};
    st.omega = {1.0, 0.0};
    st.alpha = {0.0, 0.0};
    st.rho = {tot[1], 0.0};
    if (!isfinite(bnorm)) {
        st.status = KS_NAN;
    } else if (bnorm == 0.0) {
        st.status = KS_CONVERGED;  // zero right-hand side: zero solution
        st.xbest = -1;
        st.iter = 1;
        rerr[0] = 0.0;
    } else if (rnorm <= st.btol) {
        st.status = KS_CONVERGED;  // the first guess is already good enough
        st.iter = 1;
        rerr[0] = rnorm / bnorm;
    } else {
        st.status = KS_RUNNING;
        rerr[0] = rnorm / bnorm;
        if (tot[1] == 0.0) st.status = KS_BREAKDOWN;
    }
}

// alpha = rho / (rt . v)
__device__ inline void fin_v(BicgState &st, const double *tot)
{
    cd rtv = {tot[0], tot[1]};
    if (!cd_finite(rtv)) { st.status = KS_NAN; return; }
    if (cd_zero(rtv)) { st.status = KS_BREAKDOWN; return; }
    st.alpha = cd_div(st.rho, rtv);
    if (cd_zero(st.alpha)) st.status = KS_BREAKDOWN;
}

// omega = (t . s) / (t . t)
__device__ inline void fin_t(BicgState &st, const double *tot)
{
    if (!isfinite(tot[0]) || !isfinite(tot[1]) || !isfinite(tot[2])) { st.status = KS_NAN; return; }
    if (tot[2] == 0.0) { st.status = KS_BREAKDOWN; return; }
    cd ts = {tot[0], tot[1]};
    st.omega = {ts.re / tot[2], ts.im / tot[2]};
    if (cd_zero(st.omega)) st.status = KS_BREAKDOWN;
}

// relative true residual and the scale of the next FP32 right-hand side
__device__ inline void fin_res64(OuterState &os, const double *tot)
{
    const double rn = sqrt(tot[0]);
    // a zero right-hand side with its zero solution has residual 0, as BICG
    // reports for b = 0 (not 0 / 0)
    os.relres = (os.bnorm64 == 0.0 && rn == 0.0) ? 0.0 : rn / os.bnorm64;
    os.scale = rn > 0.0 ? 1.0 / rn : 0.0;
}

}  // namespace mt3d

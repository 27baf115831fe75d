// multi.cu -- FWDsolve3D over several grids (models of uneven size) at once.
//
// The reference farms (transmitter, polarisation) solves over MPI ranks,
// each with its own per-call set-up (f90/MPI/Main_MPI.f90:1444-1649,
// f90/3D_MT/FWD_SP2/solver.f90:1148-1300).  Here the right-hand sides of
// several handles -- each its own grid, model and frequencies -- are solved
// in lockstep on one stream: the phases of every handle's FWDsolve3D run one
// after the other (set-up, the FP64 residual of each refinement cycle, the
// FP64 fallback cycles, post-processing), and the FP32 iterations of all
// grids run together, five launches per iteration over the right-hand sides
// of every grid (launch_hat_iter_multi), so the small grids and the
// right-hand sides that are still running share the GPU instead of each
// leaving most of it idle.
//
// Conditions: all handles on one device, mixed precision with the fused FP32
// iteration, BiCGStab + diagonal, the same IterPerDivCor and polynomial
// preconditioner coefficient (the FP32 cycles run in step); at most
// kMaxMultiGrids handles.
#include <algorithm>
#include <string>
#include <vector>

#include "solver.h"
#include "tma.cuh"

namespace mt3d {

int fwdsolve_multi(int nh, Solver *const *hs, const int *nrhs, const double *const *omegas, const int *const *trans,
                   const double *const *bc, const double *const *src, double *const *e, int *const *status,
                   const int *zch, bool device, std::string &err)
{
    if (nh < 1 || nh > kMaxMultiGrids || !hs || !nrhs || !omegas || !e) {
        err = "mt3d_fwdsolve_multi: invalid arguments (1 to 8 handles)";
        return 5;
    }
    Solver *h0 = hs[0];
    for (int i = 0; i < nh; i++) {
        Solver *h = hs[i];
        if (!h || nrhs[i] < 1 || !omegas[i] || !e[i]) {
            err = "mt3d_fwdsolve_multi: invalid arguments for handle " + std::to_string(i);
            return 5;
        }
        for (int j = 0; j < i; j++)
            if (hs[j] == h) {
                err = "mt3d_fwdsolve_multi: a handle appears twice";
                return 5;
            }
        if (h->device() != h0->device()) {
            err = "mt3d_fwdsolve_multi: all handles must be on one device";
            return 5;
        }
        if (h->ctl.precision != 1 || h->ctl.solver != 1 || !h->ctl.fused ||
            h->ctl.IterPerDivCor != h0->ctl.IterPerDivCor || h->ctl.poly != h0->ctl.poly) {
            err = "mt3d_fwdsolve_multi: every handle needs mixed precision, BiCGStab + diagonal, the fused FP32 "
                  "iteration, the same IterPerDivCor and the same polynomial coefficient";
            return 5;
        }
    }
    // one stream for all: the first handle's
    cudaStream_t s = h0->stream();
    std::vector<cudaStream_t> keep(nh);
    for (int i = 0; i < nh; i++) {
        keep[i] = hs[i]->stream();
        if (i) hs[i]->set_stream(s);
    }
    auto restore = [&]() {
        for (int i = 1; i < nh; i++) hs[i]->set_stream(keep[i]);
    };
    std::vector<SolveRun> runs(nh);
    int rc = 0;
    auto failed = [&](int i) {
        err = "handle " + std::to_string(i) + ": " + hs[i]->last_error;
        restore();
        return rc;
    };
    for (int i = 0; i < nh; i++)
        if ((rc = hs[i]->solve_begin(runs[i], nrhs[i], omegas[i], trans ? trans[i] : nullptr, bc ? bc[i] : nullptr,
                                     src ? src[i] : nullptr, e[i], status ? status[i] : nullptr, device)))
            return failed(i);
    const int maxit = h0->ctl.IterPerDivCor;
    for (;;) {
        bool any = false;
        std::vector<char> live(nh, 0);
        for (int i = 0; i < nh; i++) {
            if (runs[i].done) continue;
            if ((rc = hs[i]->solve_pre(runs[i]))) return failed(i);
            live[i] = !runs[i].done;
            any = any || live[i];
        }
        if (!any) break;
        // FP32 cycles: the fused groups together, any other alone
        std::vector<int> ids;
        std::vector<KArgs<float>> args;
        std::vector<int> nr, zc;
        for (int i = 0; i < nh; i++) {
            if (!live[i]) continue;
            if (hs[i]->fp32_fused(runs[i])) {
                KArgs<float> a{};
                if ((rc = hs[i]->hat_cycle_begin(runs[i].nrhs, a))) return failed(i);
                ids.push_back(i);
                args.push_back(a);
                nr.push_back(runs[i].nrhs);
                zc.push_back(zch ? zch[i] : 0);
            } else if ((rc = hs[i]->solve_fp32(runs[i]))) {
                return failed(i);
            }
        }
        if (!ids.empty()) {
            // the cycle of the whole batch as one CUDA graph kept on the
            // first grid's handle; with mt3d_profile on, timed launches
            // instead (each handle counts its own grid's sweeps)
            const int mrc = hs[ids[0]]->run_hat_multi(args.data(), nr.data(), zc.data(), (int)ids.size(), maxit, s);
            if (mrc == 5) {
                err = "mt3d_fwdsolve_multi: too many grids";
                restore();
                return 5;
            }
            const cudaError_t ce = cudaGetLastError();
            if (mrc == 4 || ce != cudaSuccess) {
                err = std::string("mt3d_fwdsolve_multi: launch failed: ") +
                      cudaGetErrorString(ce != cudaSuccess ? ce : cudaErrorUnknown);
                restore();
                return 4;
            }
            for (size_t q = 0; q < ids.size(); q++)
                if ((rc = hs[ids[q]]->hat_cycle_end(nr[q], args[q]))) return failed(ids[q]);
        }
        for (int i = 0; i < nh; i++)
            if (live[i] && (rc = hs[i]->solve_post(runs[i]))) return failed(i);
    }
    int worst = 0, wi = 0;
    for (int i = 0; i < nh; i++) {
        const int r = hs[i]->solve_end(runs[i]);
        if (r > worst) {
            worst = r;
            wi = i;
        }
    }
    if (worst) err = "handle " + std::to_string(wi) + ": " + hs[wi]->last_error;
    restore();
    return worst;
}

}  // namespace mt3d

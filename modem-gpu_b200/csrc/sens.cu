// sens.cu -- the transpose of the sensitivity for one transmitter and the
// Full_Impedance functional, on the device: JmultT_TX
// (f90/SENS/SensComp.f90:408-488) from saved background fields.
//
//   LmultT   adjoint sources of the data weights d (datafunc.cu),
//   sensSolve(TRN)  the transposed solves of both polarisations (the batched
//            FWDsolve3D of solver.cu, under the handle's control),
//   PmultT   Re(-ISIGN i omega mu0 sum_pol e0 * eadj) mapped to the model
//            parameter by dEdgeToModelParam (k_pmult_t).
// The impedance functional does not depend on the conductivity, so the
// QmultT term of JmultT_TX is zero.  Everything between the inputs and dm
// stays in device memory.
#include <cmath>
#include <string>

#include "solver.h"

namespace mt3d {

int Solver::jmult_t(double om, int nsite, const double *xyz, const double *origin, const double *e0, const double *d,
                    const double *m0, double *dm, double *eadj, bool device)
{
    const char *who = device ? "mt3d_jmult_t_device" : "mt3d_jmult_t";
    if (!cond_set) return fail(5, std::string(who) + ": conductivity not set (call mt3d_update_cond)");
    if (nsite < 1 || !xyz || !origin || !e0 || !d || !m0 || !dm || !(om > 0) || !std::isfinite(om))
        return fail(5, std::string(who) + ": invalid arguments");
    const int64_t nEarth = (int64_t)nx * ny * (nz - nzAir);
    const size_t eb = (size_t)nE * sizeof(double2);
    DevBuf E0, S, EA, M0, DM;
    int bad = S.alloc(2 * eb) || M0.alloc(nEarth * sizeof(double));
    if (!device) bad = bad || E0.alloc(2 * eb) || DM.alloc(nEarth * sizeof(double));
    if (!(device && eadj)) bad = bad || EA.alloc(2 * eb);  // adjoint fields on the device
    if (bad) return fail(8, std::string(who) + ": out of device memory");
    const double2 *e0d = reinterpret_cast<const double2 *>(e0);
    if (!device) {
        cudaMemcpyAsync(E0.as<void>(), e0, 2 * eb, cudaMemcpyHostToDevice, stream_);
        e0d = E0.as<double2>();
    }
    double2 *ead = (device && eadj) ? reinterpret_cast<double2 *>(eadj) : EA.as<double2>();
    double *dmd = device ? dm : DM.as<double>();
    int rc;
    // adjoint sources of both polarisations (LmultT)
    if ((rc = lmult_t(om, nsite, xyz, origin, reinterpret_cast<const double *>(e0d),
                      reinterpret_cast<const double *>(e0d + nE), d, S.as<double>(), S.as<double>() + 2 * nE, true)))
        return rc;
    // transposed solves from a zero first guess (sensSolve with TRN)
    if ((rc = check(cudaMemsetAsync(ead, 0, 2 * eb, stream_), who))) return rc;
    const double oms[2] = {om, om};
    const int tr[2] = {1, 1};
    int st[2] = {0, 0};
    const int src = solve(2, oms, tr, nullptr, S.as<double>(), reinterpret_cast<double *>(ead), st, true);
    if (src > 1) return src;
    // PmultT at the background model, both polarisations summed
    cudaMemcpyAsync(M0.as<void>(), m0, nEarth * sizeof(double), cudaMemcpyHostToDevice, stream_);
    launch_pmult_t(g64_, 2, e0d, ead, om, M0.as<double>(), dmd, stream_);
    if (!device) {
        cudaMemcpyAsync(dm, dmd, nEarth * sizeof(double), cudaMemcpyDeviceToHost, stream_);
        if (eadj) cudaMemcpyAsync(eadj, ead, 2 * eb, cudaMemcpyDeviceToHost, stream_);
    }
    if ((rc = sync(who))) return rc;
    return src;  // MT3D_OK, or MT3D_NOT_CONVERGED when a transposed solve stopped at its limits
}

}  // namespace mt3d

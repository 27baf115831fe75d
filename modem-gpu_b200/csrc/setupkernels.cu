// setupkernels.cu -- the conductivity-dependent operator set-up on the GPU.
//
// From the model parameter (log conductivity of the earth cells, the air
// cells at exp(airCond): ModelParamToCell, LOGE) the kernels build:
//   - the edge conductivity: ModelParamToEdge, Cell2Edge of V_C sigma over
//     Cell2Edge of V_C with the adjacent cells summed in the order
//     (a-1, b-1), (a, b-1), (a-1, b), (a, b) (f90/3D_MT/modelParam/
//     ModelMap.inc:88-188, f90/3D_MT/GridCalc.f90:430-598);
//   - the SP2 edge conductivity (boundary edges zero), the node weights and
//     earth flags of GradDivSetup2 with airNIndex (f90/3D_MT/FWD_SP2/
//     modelOperator3D.f90:176-230, 916-1008, 1086-1130);
//   - the divergence-correction coefficients of DivCorrSetUp with the air
//     edges at SIGMA_AIR, then the air edges zeroed (f90/3D_MT/FWD/
//     modelOperator3D.f90:1538-1650);
//   - the FP32 copies.
// Every expression keeps the operation order of the reference and this file
// is compiled without fused multiply-adds, so from the same cell
// conductivities the results are bitwise those of the same loops on the host;
// the cell conductivities themselves come from the device exp().
#include <atomic>

#include "kernels.h"

namespace mt3d {

extern std::atomic<long long> g_launch_count;

namespace {
constexpr int kT = 256;
inline int blocks(long long n) { return (int)std::min<long long>((n + kT - 1) / kT, 148LL * 32); }
}  // namespace

// cell volume V_C, V_C sigma_C and sigma_C
__global__ void ks_cells(Geo<double> g, const double *m_earth, double airCond, double *VC, double *CT, double *sigC)
{
    const long long nC = (long long)g.nx * g.ny * g.nz, nAir = (long long)g.nx * g.ny * g.nzAir;
    for (long long c = blockIdx.x * (long long)kT + threadIdx.x; c < nC; c += (long long)gridDim.x * kT) {
        const int i = (int)(c % g.nx), t = (int)(c / g.nx), j = t % g.ny;
        const int k = t / g.ny;
        const double v = g.dx[i] * g.dy[j] * g.dz[k];
        const double s = c < nAir ? exp(airCond) : exp(m_earth[c - nAir]);
        VC[c] = v;
        CT[c] = v * s;
        sigC[c] = s;
    }
}

// the edges of the air cells (1-based iz <= nzAir, ix <= nx, iy <= ny in the
// loops of DivCorrSetUp)
__device__ __forceinline__ bool air_edge(const Geo<double> &g, const EdgeIdx &q)
{
    return q.k < g.nzAir && (q.c == 0 ? q.j < g.ny : q.c == 1 ? q.i < g.nx : (q.i < g.nx && q.j < g.ny));
}

// edge conductivity (volume-weighted mean of the 2 or 4 adjacent cells) and
// its SP2 copy with the non-interior edges zero
__global__ void ks_edge_sigma(Geo<double> g, const double *VC, const double *CT, double *sig, double *sigs)
{
    for (long long e = blockIdx.x * (long long)kT + threadIdx.x; e < g.nE; e += (long long)gridDim.x * kT) {
        const EdgeIdx q = edge_decode(g, (int)e);
        double num = 0.0, den = 0.0;
        int n = 0;
        for (int s = 0; s < 4; s++) {
            const int da = (s & 1) ? 0 : -1, db = (s & 2) ? 0 : -1;
            int ci = q.i, cj = q.j, ck = q.k;
            if (q.c == 0) { cj = q.j + da; ck = q.k + db; }
            if (q.c == 1) { ci = q.i + da; ck = q.k + db; }
            if (q.c == 2) { cj = q.j + da; ci = q.i + db; }
            if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny || ck < 0 || ck >= g.nz) continue;
            const long long c = ci + (long long)g.nx * (cj + (long long)g.ny * ck);
            num += CT[c];
            den += VC[c];
            n++;
        }
        const double v = (num / n) / (den / n);
        sig[e] = v;
        sigs[e] = edge_interior(g, q) ? v : 0.0;
    }
}

// per node: grad-div weight, earth flag and signed weight (GradDivSetup2) and
// the DivCorrSetUp coefficients [db1x db2x db1y db2y db1z db2z c][nN], read
// from the edge conductivity with the air edges at SIGMA_AIR
__global__ void ks_nodes(Geo<double> g, const double *VC, const double *CT, const double *sig, const double *sigs,
                         double *gdw, unsigned char *gde, double *gdn, float *gdw32, float *gdn32, double *coef)
{
    const long long nN = g.nN;
    for (long long n = blockIdx.x * (long long)kT + threadIdx.x; n < nN; n += (long long)gridDim.x * kT) {
        const int i = (int)(n % (g.nx + 1)), t = (int)(n / (g.nx + 1)), j = t % (g.ny + 1), k = t / (g.ny + 1);
        double w = 0.0, c[7] = {0, 0, 0, 0, 0, 0, 0};
        unsigned char earth = 0;
        if (i >= 1 && i < g.nx && j >= 1 && j < g.ny && k >= 1 && k < g.nz) {
            const int ex0 = iX(g, i - 1, j, k), ex1 = iX(g, i, j, k), ey0 = iY(g, i, j - 1, k), ey1 = iY(g, i, j, k),
                      ez0 = iZ(g, i, j, k - 1), ez1 = iZ(g, i, j, k);
            const double thr = 1.1 * kSigmaAir;
            earth = (sigs[ex0] >= thr || sigs[ex1] >= thr || sigs[ey0] >= thr || sigs[ey1] >= thr || sigs[ez0] >= thr ||
                     sigs[ez1] >= thr)
                        ? 1
                        : 0;
            double num = 0.0, den = 0.0;
            for (int q = 0; q < 8; q++) {
                const int ci = i - 1 + (q & 1), cj = j - 1 + ((q >> 1) & 1), ck = k - 1 + ((q >> 2) & 1);
                const long long cl = ci + (long long)g.nx * (cj + (long long)g.ny * ck);
                num += CT[cl];
                den += VC[cl];
            }
            const double vn = g.delX[i] * g.delY[j] * g.delZ[k];
            w = earth ? 1.0 / ((num / den) * vn) : 1.0 / vn;
            // air cells at SIGMA_AIR: an x-edge (i, j, k) is air for k < nzAir, j < ny;
            // a y-edge for k < nzAir, i < nx; a z-edge for k < nzAir, i < nx, j < ny
            const bool ak0 = k < g.nzAir, ak1 = k - 1 < g.nzAir;
            const double sx0 = (ak0 && j < g.ny) ? kSigmaAir : sig[ex0];
            const double sx1 = (ak0 && j < g.ny) ? kSigmaAir : sig[ex1];
            const double sy0 = (ak0 && i < g.nx) ? kSigmaAir : sig[ey0];
            const double sy1 = (ak0 && i < g.nx) ? kSigmaAir : sig[ey1];
            const double sz0 = (ak1 && i < g.nx && j < g.ny) ? kSigmaAir : sig[ez0];
            const double sz1 = (ak0 && i < g.nx && j < g.ny) ? kSigmaAir : sig[ez1];
            c[0] = sx0 / (g.dx[i - 1] * g.delX[i]);
            c[1] = sx1 / (g.dx[i] * g.delX[i]);
            c[2] = sy0 / (g.dy[j - 1] * g.delY[j]);
            c[3] = sy1 / (g.dy[j] * g.delY[j]);
            c[4] = sz0 / (g.dz[k - 1] * g.delZ[k]);
            c[5] = sz1 / (g.dz[k] * g.delZ[k]);
            c[6] = -(c[0] + c[1] + c[2] + c[3] + c[4] + c[5]);
            for (int q = 0; q < 7; q++) c[q] = c[q] * vn;
            // coefficients that multiply boundary nodes are zero
            if (i == 1) c[0] = 0.0;
            if (i == g.nx - 1) c[1] = 0.0;
            if (j == 1) c[2] = 0.0;
            if (j == g.ny - 1) c[3] = 0.0;
            if (k == 1) c[4] = 0.0;
            if (k == g.nz - 1) c[5] = 0.0;
        }
        const double wn = earth ? -w : w;
        gdw[n] = w;
        gde[n] = earth;
        gdn[n] = wn;
        gdw32[n] = (float)w;
        gdn32[n] = (float)wn;
        for (int q = 0; q < 7; q++) coef[q * nN + n] = c[q];
    }
}

// the air edges zeroed in the forward operator's conductivity; FP32 copies
__global__ void ks_edge_final(Geo<double> g, double *sig, const double *sigs, float *sig32, float *sigs32)
{
    for (long long e = blockIdx.x * (long long)kT + threadIdx.x; e < g.nE; e += (long long)gridDim.x * kT) {
        const EdgeIdx q = edge_decode(g, (int)e);
        double v = sig[e];
        if (air_edge(g, q)) {
            v = 0.0;
            sig[e] = 0.0;
        }
        sig32[e] = (float)v;
        sigs32[e] = (float)sigs[e];
    }
}

void launch_setup_cond(const Geo<double> &g, const double *m_earth, double airCond, double *VC, double *CT,
                       double *sigC, double *sig, double *sigs, double *gdw, unsigned char *gde, double *gdn, double *coef,
                       float *sig32, float *sigs32, float *gdw32, float *gdn32, cudaStream_t s)
{
    const long long nC = (long long)g.nx * g.ny * g.nz;
    g_launch_count.fetch_add(4, std::memory_order_relaxed);
    ks_cells<<<blocks(nC), kT, 0, s>>>(g, m_earth, airCond, VC, CT, sigC);
    ks_edge_sigma<<<blocks(g.nE), kT, 0, s>>>(g, VC, CT, sig, sigs);
    ks_nodes<<<blocks(g.nN), kT, 0, s>>>(g, VC, CT, sig, sigs, gdw, gde, gdn, gdw32, gdn32, coef);
    ks_edge_final<<<blocks(g.nE), kT, 0, s>>>(g, sig, sigs, sig32, sigs32);
}

}  // namespace mt3d

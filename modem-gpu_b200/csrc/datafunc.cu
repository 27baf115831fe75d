// datafunc.cu -- the Full_Impedance data functional on the GPU.
//
// dataResp for Full_Impedance (f90/3D_MT/DataFunc.f90:143-189): at each site
// the horizontal electric fields (EinterpSetUp, f90/3D_MT/EMfieldInterp.f90:
// 141-324) and magnetic fields (BfromESetUp, :470-647, on BinterpSetUp,
// :329-465) of the two polarisations are sparse linear functionals of the
// edge field; Z = E B^-1 (Kramer's rule), Z(2(i-1)+j) = sum_m E(i,m) B^-1(m,j).
// The functionals are set up on the host (a few dozen terms per site, as the
// reference does per site), the dot products with the fields and the 2 x 2
// inversions run on the device, so the fields never leave HBM.  Site
// azimuths are zero (the reference's rotate_Model2Data with zero angles).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include <atomic>

#include "solver.h"

namespace mt3d {

extern std::atomic<long long> g_launch_count;
__host__ __device__ inline cd cd_add(cd a, cd b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ inline cd cd_sub(cd a, cd b) { return {a.re - b.re, a.im - b.im}; }

namespace {

// grid coordinates as setup_grid builds them (f90/3D_MT/GridDef.f90:301-394),
// 1-based like the Fortran (index 0 unused)
struct Coords {
    std::vector<double> xE, yE, zE, xC, yC, zC, dx, dy, dz, dX, dY, dZ;
};

Coords make_coords(const std::vector<double> &dx, const std::vector<double> &dy, const std::vector<double> &dz,
                   const std::vector<double> &delX, const std::vector<double> &delY, const std::vector<double> &delZ,
                   int nzAir, const double *origin)
{
    const int nx = (int)dx.size(), ny = (int)dy.size(), nz = (int)dz.size();
    Coords c;
    auto one = [](const std::vector<double> &v) {
        std::vector<double> r(v.size() + 1, 0.0);
        for (size_t i = 0; i < v.size(); i++) r[i + 1] = v[i];
        return r;
    };
    c.dx = one(dx); c.dy = one(dy); c.dz = one(dz);
    c.dX = one(delX); c.dY = one(delY); c.dZ = one(delZ);
    c.xE.assign(nx + 2, 0.0); c.yE.assign(ny + 2, 0.0); c.zE.assign(nz + 2, 0.0);
    c.xC.assign(nx + 1, 0.0); c.yC.assign(ny + 1, 0.0); c.zC.assign(nz + 1, 0.0);
    c.xE[1] = origin[0];
    c.yE[1] = origin[1];
    double cum = 0.0;
    for (int i = 1; i <= nx; i++) { cum += c.dx[i]; c.xE[i + 1] = cum + origin[0]; }
    cum = 0.0;
    for (int i = 1; i <= ny; i++) { cum += c.dy[i]; c.yE[i + 1] = cum + origin[1]; }
    cum = 0.0;
    c.zE[1] = 0.0;
    for (int i = 1; i <= nz; i++) { cum += c.dz[i]; c.zE[i + 1] = cum; }
    const double air = c.zE[nzAir + 1];
    cum = 0.0;
    for (int i = 1; i <= nx; i++) { cum += c.dX[i]; c.xC[i] = cum + origin[0]; }
    cum = 0.0;
    for (int i = 1; i <= ny; i++) { cum += c.dY[i]; c.yC[i] = cum + origin[1]; }
    cum = 0.0;
    for (int i = 1; i <= nz; i++) { cum += c.dZ[i]; c.zC[i] = cum; }
    for (int i = 1; i <= nz; i++) {
        c.zC[i] = c.zC[i] - air + origin[2];
        c.zE[i] = c.zE[i] - air + origin[2];
    }
    c.zE[nz + 1] = c.zE[nz + 1] - air + origin[2];
    return c;
}

// clean and minNode (f90/UTILS/utilities.f90:100-114, 196-225); nodes 1..n
double clean(double x) { return std::round(x * 1.0e13) / 1.0e13; }
int min_node(double x, const std::vector<double> &node, int n)
{
    for (int i = 1; i <= n; i++)
        if (clean(node[i]) > clean(x)) return i - 1;
    return n;
}

struct Term {
    int c, i, j, k;  // component 1..3 and 1-based indices of an edge or face
    double re, im;
};

// EinterpSetUp without conductivity weighting (f90/3D_MT/EMfieldInterp.f90:141-324)
std::vector<Term> e_interp(const Coords &g, int nx, int ny, int nz, const double *x, int xyz)
{
    int nxMax = nx + 1, nyMax = ny + 1, nzMax = nz + 1;
    int i0 = min_node(x[0], g.xE, nx + 1), j0 = min_node(x[1], g.yE, ny + 1), k0 = min_node(x[2], g.zE, nz + 1);
    if (xyz == 1) { i0 = min_node(x[0], g.xC, nx); nxMax -= 1; }
    if (xyz == 2) { j0 = min_node(x[1], g.yC, ny); nyMax -= 1; }
    if (xyz == 3) { k0 = min_node(x[2], g.zC, nz); nzMax -= 1; }
    double w[3][2];
    auto weight = [&](int a, int n0, int nMax, bool centred, const std::vector<double> &C,
                      const std::vector<double> &D, const std::vector<double> &E, const std::vector<double> &d) {
        if (n0 > 0 && n0 < nMax)
            w[a][1] = centred ? (x[a] - C[n0]) / D[n0 + 1] : (x[a] - E[n0]) / d[n0];
        else
            w[a][1] = n0 <= 0 ? 1.0 : 0.0;
    };
    weight(0, i0, nxMax, xyz == 1, g.xC, g.dX, g.xE, g.dx);
    weight(1, j0, nyMax, xyz == 2, g.yC, g.dY, g.yE, g.dy);
    weight(2, k0, nzMax, xyz == 3, g.zC, g.dZ, g.zE, g.dz);
    for (int a = 0; a < 3; a++) w[a][0] = 1.0 - w[a][1];
    std::vector<Term> t;
    for (int n = 0; n < 2; n++)
        for (int m = 0; m < 2; m++)
            for (int p = 0; p < 2; p++) {
                const double wadd = w[0][n] * w[1][m] * w[2][p];
                if (wadd > 0) t.push_back({xyz, i0 + n, j0 + m, k0 + p, wadd, 0.0});
            }
    return t;
}

// BinterpSetUp (f90/3D_MT/EMfieldInterp.f90:329-465): faces
std::vector<Term> b_interp(const Coords &g, int nx, int ny, int nz, const double *x, int xyz)
{
    int nxMax = nx, nyMax = ny, nzMax = nz, i0, j0, k0;
    if (xyz == 1) {
        i0 = min_node(x[0], g.xE, nx + 1); j0 = min_node(x[1], g.yC, ny); k0 = min_node(x[2], g.zC, nz);
        nxMax += 1;
    } else if (xyz == 2) {
        i0 = min_node(x[0], g.xC, nx); j0 = min_node(x[1], g.yE, ny + 1); k0 = min_node(x[2], g.zC, nz);
        nyMax += 1;
    } else {
        i0 = min_node(x[0], g.xC, nx); j0 = min_node(x[1], g.yC, ny); k0 = min_node(x[2], g.zE, nz + 1);
        nzMax += 1;
    }
    double w[3][2];
    auto weight = [&](int a, int n0, int nMax, bool edge, const std::vector<double> &C, const std::vector<double> &D,
                      const std::vector<double> &E, const std::vector<double> &d) {
        if (n0 > 0 && n0 < nMax)
            w[a][1] = edge ? (x[a] - E[n0]) / d[n0] : (x[a] - C[n0]) / D[n0 + 1];
        else
            w[a][1] = n0 <= 0 ? 1.0 : 0.0;
    };
    weight(0, i0, nxMax, xyz == 1, g.xC, g.dX, g.xE, g.dx);
    weight(1, j0, nyMax, xyz == 2, g.yC, g.dY, g.yE, g.dy);
    weight(2, k0, nzMax, xyz == 3, g.zC, g.dZ, g.zE, g.dz);
    for (int a = 0; a < 3; a++) w[a][0] = 1.0 - w[a][1];
    std::vector<Term> t;
    for (int n = 0; n < 2; n++)
        for (int m = 0; m < 2; m++)
            for (int p = 0; p < 2; p++) {
                const double wadd = w[0][n] * w[1][m] * w[2][p];
                if (wadd > 0) t.push_back({xyz, i0 + n, j0 + m, k0 + p, wadd, 0.0});
            }
    return t;
}

// BfromESetUp (f90/3D_MT/EMfieldInterp.f90:470-647): B_xyz = (i ISIGN / omega)
// sum_faces w_f (circulation of E around face f) / area_f
std::vector<Term> b_from_e(const Coords &g, int nx, int ny, int nz, double omega, const double *x, int xyz)
{
    const double ioi = -1.0 / omega;  // i * ISIGN / omega, ISIGN = -1: (0, -1/omega)
    std::vector<Term> out;
    for (const Term &f : b_interp(g, nx, ny, nz, x, xyz)) {
        const int I = f.i, J = f.j, K = f.k;
        Term e[4];
        if (f.c == 1) {
            const double S = g.dy[J] * g.dz[K];
            e[0] = {2, I, J, K, g.dy[J] / S, 0};
            e[1] = {2, I, J, K + 1, -g.dy[J] / S, 0};
            e[2] = {3, I, J, K, -g.dz[K] / S, 0};
            e[3] = {3, I, J + 1, K, g.dz[K] / S, 0};
        } else if (f.c == 2) {
            const double S = g.dx[I] * g.dz[K];
            e[0] = {3, I, J, K, g.dz[K] / S, 0};
            e[1] = {3, I + 1, J, K, -g.dz[K] / S, 0};
            e[2] = {1, I, J, K, -g.dx[I] / S, 0};
            e[3] = {1, I, J, K + 1, g.dx[I] / S, 0};
        } else {
            const double S = g.dx[I] * g.dy[J];
            e[0] = {1, I, J, K, g.dx[I] / S, 0};
            e[1] = {1, I, J + 1, K, -g.dx[I] / S, 0};
            e[2] = {2, I, J, K, -g.dy[J] / S, 0};
            e[3] = {2, I + 1, J, K, g.dy[J] / S, 0};
        }
        for (Term &t : e) {
            const double c = t.re * f.re;  // real: C * w
            t.re = 0.0;
            t.im = c * ioi;
            out.push_back(t);
        }
    }
    return out;
}

}  // namespace

// flat 0-based edge index of a 1-based (component, i, j, k); -1 outside the grid
static long long edge_flat(int nx, int ny, int nz, const Term &t)
{
    const long long nXe = (long long)nx * (ny + 1) * (nz + 1), nYe = (long long)(nx + 1) * ny * (nz + 1);
    const int i = t.i - 1, j = t.j - 1, k = t.k - 1;
    if (i < 0 || j < 0 || k < 0) return -1;
    if (t.c == 1) return (i < nx && j <= ny && k <= nz) ? i + (long long)nx * (j + (long long)(ny + 1) * k) : -1;
    if (t.c == 2) return (i <= nx && j < ny && k <= nz) ? nXe + i + (long long)(nx + 1) * (j + (long long)ny * k) : -1;
    return (i <= nx && j <= ny && k < nz) ? nXe + nYe + i + (long long)(nx + 1) * (j + (long long)(ny + 1) * k) : -1;
}

// the four functionals (Ex, Ey, Bx, By) of every site as CSR rows 4 s + f
static int build_functionals(const Coords &c, int nx, int ny, int nz, double om, int nsite, const double *xyz,
                             std::vector<int> &off, std::vector<int> &idx, std::vector<double2> &coef, std::string &err)
{
    off.assign(4 * (size_t)nsite + 1, 0);
    idx.clear();
    coef.clear();
    for (int s = 0; s < nsite; s++) {
        const double *x = xyz + 3 * (size_t)s;
        if (!std::isfinite(x[0]) || !std::isfinite(x[1]) || !std::isfinite(x[2])) {
            err = "site coordinates must be finite";
            return 5;
        }
        const std::vector<Term> L[4] = {e_interp(c, nx, ny, nz, x, 1), e_interp(c, nx, ny, nz, x, 2),
                                        b_from_e(c, nx, ny, nz, om, x, 1), b_from_e(c, nx, ny, nz, om, x, 2)};
        for (int f = 0; f < 4; f++) {
            for (const Term &t : L[f]) {
                const long long e = edge_flat(nx, ny, nz, t);
                if (e < 0) {
                    err = "site " + std::to_string(s) + " needs an edge outside the grid";
                    return 5;
                }
                idx.push_back((int)e);
                coef.push_back(make_double2(t.re, t.im));
            }
            off[4 * (size_t)s + f + 1] = (int)idx.size();
        }
    }
    return 0;
}

// per site: the functionals on both polarisations, Z and B^-1 (dataResp);
// with d non-null also the weights of the four functionals in the adjoint
// source of each polarisation k (Lrows + LmultT for Full_Impedance,
// f90/3D_MT/DataFunc.f90:465-869, f90/SENS/DataSens.f90:130-225):
//   s_k = sum_ij conj(d_ij) B^-1(k, j) (Le_i - Z_i1 Lbx - Z_i2 Lby)
__global__ void k_site(int nsite, const int *off, const int *idx, const double2 *coef, const double2 *e1,
                       const double2 *e2, double2 *Z, const double2 *d, double2 *W)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsite) return;
    cd v[4][2];
    for (int f = 0; f < 4; f++) {
        cd a = {0.0, 0.0}, b = {0.0, 0.0};
        for (int q = off[4 * s + f]; q < off[4 * s + f + 1]; q++) {
            const cd c = {coef[q].x, coef[q].y};
            const double2 x1 = e1[idx[q]], x2 = e2[idx[q]];
            a = cd_add(a, cd_mul(c, cd{x1.x, x1.y}));
            b = cd_add(b, cd_mul(c, cd{x2.x, x2.y}));
        }
        v[f][0] = a;
        v[f][1] = b;
    }
    // EE(i, m) = v[i][m], BB(i, m) = v[2 + i][m]; BB^-1 by Kramer's rule
    const cd det = cd_sub(cd_mul(v[2][0], v[3][1]), cd_mul(v[2][1], v[3][0]));
    cd bi[2][2], z[2][2];
    bi[0][0] = cd_div(v[3][1], det);
    bi[1][1] = cd_div(v[2][0], det);
    bi[0][1] = cd_div(cd{-v[2][1].re, -v[2][1].im}, det);
    bi[1][0] = cd_div(cd{-v[3][0].re, -v[3][0].im}, det);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            z[i][j] = cd_add(cd_mul(v[i][0], bi[0][j]), cd_mul(v[i][1], bi[1][j]));
            if (Z) Z[4 * (size_t)s + 2 * i + j] = make_double2(z[i][j].re, z[i][j].im);
        }
    if (!d) return;
    for (int k = 0; k < 2; k++) {
        cd w[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                const double2 dd = d[4 * (size_t)s + 2 * i + j];
                const cd c = cd_mul(cd{dd.x, -dd.y}, bi[k][j]);  // conj(d_ij) B^-1(k, j)
                w[i] = cd_add(w[i], c);                          // Lex (i = 0) or Ley (i = 1)
                w[2] = cd_sub(w[2], cd_mul(c, z[i][0]));         // Lbx
                w[3] = cd_sub(w[3], cd_mul(c, z[i][1]));         // Lby
            }
        for (int f = 0; f < 4; f++) W[(4 * (size_t)s + f) * 2 + k] = make_double2(w[f].re, w[f].im);
    }
}

// adjoint sources: each distinct edge sums its (site, functional, coefficient)
// entries in a fixed order (deterministic; no atomics)
__global__ void k_scatter(int nu, const int *uoff, const int *uedge, const int *urow, const double2 *ucoef,
                          const double2 *W, double2 *s1, double2 *s2)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= nu) return;
    cd a = {0, 0}, b = {0, 0};
    for (int q = uoff[u]; q < uoff[u + 1]; q++) {
        const cd c = {ucoef[q].x, ucoef[q].y};
        const double2 w0 = W[(size_t)urow[q] * 2], w1 = W[(size_t)urow[q] * 2 + 1];
        a = cd_add(a, cd_mul(c, cd{w0.x, w0.y}));
        b = cd_add(b, cd_mul(c, cd{w1.x, w1.y}));
    }
    s1[uedge[u]] = make_double2(a.re, a.im);
    s2[uedge[u]] = make_double2(b.re, b.im);
}

int Solver::impedance(double om, int nsite, const double *xyz, const double *origin, const double *e1,
                      const double *e2, double *Zout, bool device)
{
    return data_functional(om, nsite, xyz, origin, e1, e2, nullptr, Zout, nullptr, nullptr, device);
}

int Solver::lmult_t(double om, int nsite, const double *xyz, const double *origin, const double *e1, const double *e2,
                    const double *d, double *s1, double *s2, bool device)
{
    if (!d || !s1 || !s2) return fail(5, "mt3d_lmult_t: invalid arguments");
    return data_functional(om, nsite, xyz, origin, e1, e2, d, nullptr, s1, s2, device);
}

int Solver::data_functional(double om, int nsite, const double *xyz, const double *origin, const double *e1,
                            const double *e2, const double *d, double *Zout, double *s1, double *s2, bool device)
{
    const char *who = d ? "mt3d_lmult_t" : "mt3d_impedance";
    if (nsite < 1 || !xyz || !origin || !e1 || !e2 || !(om > 0) || !std::isfinite(om) || (!d && !Zout))
        return fail(5, std::string(who) + ": invalid arguments");
    const Coords c = make_coords(dx_, dy_, dz_, delX_, delY_, delZ_, nzAir, origin);
    std::vector<int> off, idx;
    std::vector<double2> coef;
    std::string err;
    if (int rc = build_functionals(c, nx, ny, nz, om, nsite, xyz, off, idx, coef, err))
        return fail(rc, std::string(who) + ": " + err);
    // transposed rows for the adjoint sources: entries grouped by edge in
    // (site, functional, term) order
    std::vector<int> uoff, uedge, urow;
    std::vector<double2> ucoef;
    if (d) {
        std::vector<int> order(idx.size());
        for (size_t q = 0; q < idx.size(); q++) order[q] = (int)q;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return idx[a] < idx[b]; });
        std::vector<int> row(idx.size());
        for (size_t r = 0; r + 1 < off.size(); r++)
            for (int q = off[r]; q < off[r + 1]; q++) row[q] = (int)r;
        for (size_t n = 0; n < order.size(); n++) {
            const int q = order[n];
            if (uedge.empty() || uedge.back() != idx[q]) {
                uedge.push_back(idx[q]);
                uoff.push_back((int)n);
            }
            urow.push_back(row[q]);
            ucoef.push_back(coef[q]);
        }
        uoff.push_back((int)order.size());
    }
    const size_t eb = (size_t)nE * sizeof(double2);
    DevBuf doff, didx, dcoef, dz, de1, de2, dd, dw, duoff, duedge, durow, ducoef, ds1, ds2;
    int bad = doff.alloc(off.size() * sizeof(int)) || didx.alloc(idx.size() * sizeof(int)) ||
              dcoef.alloc(coef.size() * sizeof(double2)) || (!device && (de1.alloc(eb) || de2.alloc(eb)));
    if (Zout) bad = bad || dz.alloc(4 * (size_t)nsite * sizeof(double2));
    if (d)
        bad = bad || dd.alloc(4 * (size_t)nsite * sizeof(double2)) || dw.alloc(8 * (size_t)nsite * sizeof(double2)) ||
              duoff.alloc(uoff.size() * sizeof(int)) || duedge.alloc(uedge.size() * sizeof(int)) ||
              durow.alloc(urow.size() * sizeof(int)) || ducoef.alloc(ucoef.size() * sizeof(double2)) ||
              (!device && (ds1.alloc(eb) || ds2.alloc(eb)));
    if (bad) return fail(8, std::string(who) + ": out of device memory");
    cudaMemcpyAsync(doff.as<void>(), off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(didx.as<void>(), idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, stream_);
    cudaMemcpyAsync(dcoef.as<void>(), coef.data(), coef.size() * sizeof(double2), cudaMemcpyHostToDevice, stream_);
    const double2 *p1 = reinterpret_cast<const double2 *>(e1), *p2 = reinterpret_cast<const double2 *>(e2);
    if (!device) {
        cudaMemcpyAsync(de1.as<void>(), e1, eb, cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(de2.as<void>(), e2, eb, cudaMemcpyHostToDevice, stream_);
        p1 = de1.as<double2>();
        p2 = de2.as<double2>();
    }
    double2 *q1 = nullptr, *q2 = nullptr;
    if (d) {
        cudaMemcpyAsync(dd.as<void>(), d, 4 * (size_t)nsite * sizeof(double2), cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(duoff.as<void>(), uoff.data(), uoff.size() * sizeof(int), cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(duedge.as<void>(), uedge.data(), uedge.size() * sizeof(int), cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(durow.as<void>(), urow.data(), urow.size() * sizeof(int), cudaMemcpyHostToDevice, stream_);
        cudaMemcpyAsync(ducoef.as<void>(), ucoef.data(), ucoef.size() * sizeof(double2), cudaMemcpyHostToDevice,
                        stream_);
        q1 = device ? reinterpret_cast<double2 *>(s1) : ds1.as<double2>();
        q2 = device ? reinterpret_cast<double2 *>(s2) : ds2.as<double2>();
        cudaMemsetAsync(q1, 0, eb, stream_);
        cudaMemsetAsync(q2, 0, eb, stream_);
    }
    g_launch_count.fetch_add(d ? 2 : 1, std::memory_order_relaxed);
    k_site<<<(nsite + 127) / 128, 128, 0, stream_>>>(nsite, doff.as<int>(), didx.as<int>(), dcoef.as<double2>(), p1,
                                                      p2, Zout ? dz.as<double2>() : nullptr,
                                                      d ? dd.as<double2>() : nullptr, d ? dw.as<double2>() : nullptr);
    if (d) {
        const int nu = (int)uedge.size();
        k_scatter<<<(nu + 127) / 128, 128, 0, stream_>>>(nu, duoff.as<int>(), duedge.as<int>(), durow.as<int>(),
                                                          ducoef.as<double2>(), dw.as<double2>(), q1, q2);
        if (!device) {
            cudaMemcpyAsync(s1, q1, eb, cudaMemcpyDeviceToHost, stream_);
            cudaMemcpyAsync(s2, q2, eb, cudaMemcpyDeviceToHost, stream_);
        }
    }
    if (Zout)
        cudaMemcpyAsync(Zout, dz.as<void>(), 4 * (size_t)nsite * sizeof(double2), cudaMemcpyDeviceToHost, stream_);
    return sync(who);
}

}  // namespace mt3d

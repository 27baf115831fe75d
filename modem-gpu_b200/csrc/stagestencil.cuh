// stagestencil.cuh -- shared-memory staged form of the edge stencil with the
// grad-div term fused in.
//
// A block owns a tile of kStX x kStY node columns (i, j) and marches the node
// planes k of its chunk [k0, k1).  The planes of Ex, Ey, Ez and of the edge
// conductivity, each with a one-column halo in i and j, are copied into a
// four-slot ring in shared memory with cp.async (8-byte copies: the edge
// layout's row lengths nx and nx + 1 rule out 16-byte aligned bulk copies),
// one plane ahead of the plane being computed, so every global read is a
// coalesced row and the copies of plane k + 2 overlap the arithmetic of plane
// k.  Out-of-range entries are zero-filled by the copies themselves.
//
// The grad-div node potentials phi = W G^T (C DFA x) of the SP2 operator
// (GradDivSetup2, f90/3D_MT/FWD_SP2/modelOperator3D.f90:916-1008) are formed
// from the staged planes for the tile's nodes plus one node row/column of
// halo, so the operator apply needs no separate potential pass.
//
// The stencil arithmetic is that of col_march (colstencil.cuh): the Maxwell
// operator of f90/3D_MT/FWD/modelOperator3D.f90:692-800 times V_E.
#pragma once
#include <climits>

#include "colstencil.cuh"

namespace mt3d {

constexpr int kStX = 32, kStY = 8;              // node columns per tile (kThreads threads)
constexpr int kHX = kStX + 2, kHY = kStY + 2;   // staged plane with a halo column / row on each side
constexpr int kHP = kHX * kHY;
constexpr int kNX = kStX + 1, kNY = kStY + 1;   // nodes whose potential the tile needs
constexpr int kNP = kNX * kNY;
constexpr int kRing = 4;                        // staged planes k-1 .. k+2
static_assert(kStX * kStY == kThreads, "one thread per node column");

template <typename T> struct StageSmem {
    C2<T> f[kRing][3][kHP];  // Ex, Ey, Ez planes
    T s[kRing][3][kHP];      // edge conductivity planes
    C2<T> phi[2][kNP];       // node potentials of planes k and k + 1
    T nw[2][kNP];            // signed node weights (grad-div) of planes p, p + 1
};

template <int B> __device__ __forceinline__ void cp_async_zfill(void *dst, const void *src, bool ok)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = ok ? B : 0;
    if constexpr (B == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(B), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Which staged entries a thread copies, fixed for the whole march: entries
// t = threadIdx.x + kThreads m of a plane (t = comp kHP + lj kHX + li, all
// three components), with their offset at plane 0 (-1 outside the grid in
// (i, j)), and the node-weight entries of the tile's nodes.
struct StageMap {
    int goff[4];   // edge offset of entry m at plane 0; -1: outside the grid; INT_MIN: no entry
    int cm;        // component of entry m in bits 2m, 2m+1
    int goffn[2];  // node offset of node entry m at plane 0; -1 outside; INT_MIN: no entry
};

template <typename T> __device__ __forceinline__ StageMap stage_map(const Geo<T> &g, int i0, int j0)
{
    StageMap m;
    m.cm = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int t = threadIdx.x + kThreads * q;
        m.goff[q] = INT_MIN;
        if (t < 3 * kHP) {
            const int comp = t / kHP, rem = t - comp * kHP, lj = rem / kHX, li = rem - lj * kHX;
            const int i = i0 - 1 + li, j = j0 - 1 + lj;
            bool ok;
            int e;
            if (comp == 0) {
                ok = i >= 0 && i < g.nx && j >= 0 && j <= g.ny;
                e = i + g.nx * j;
            } else if (comp == 1) {
                ok = i >= 0 && i <= g.nx && j >= 0 && j < g.ny;
                e = g.nXe + i + (g.nx + 1) * j;
            } else {
                ok = i >= 0 && i <= g.nx && j >= 0 && j <= g.ny;
                e = g.nXe + g.nYe + i + (g.nx + 1) * j;
            }
            m.goff[q] = ok ? e : -1;
            m.cm |= comp << (2 * q);
        }
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int t = threadIdx.x + kThreads * q;
        m.goffn[q] = INT_MIN;
        if (t < kNP) {
            const int nj = t / kNX, ni = t - nj * kNX;
            const int i = i0 + ni, j = j0 + nj;
            m.goffn[q] = (i <= g.nx && j <= g.ny) ? i + (g.nx + 1) * j : -1;
        }
    }
    return m;
}

// copy plane p (Ex, Ey, Ez and sigma over the tile and its halo, and with
// gdn the node weights of the tile's nodes) into ring slot p mod kRing;
// entries outside the grid are zero-filled
template <typename T>
__device__ __forceinline__ void stage_plane(StageSmem<T> &sm, const Geo<T> &g, const StageMap &m,
                                            const C2<T> *__restrict__ x, const T *__restrict__ sig,
                                            const T *__restrict__ gdn, int p)
{
    const int slot = p & (kRing - 1);
    const int psx = g.nx * (g.ny + 1) * p, psy = (g.nx + 1) * g.ny * p, psz = (g.nx + 1) * (g.ny + 1) * p;
    const bool pin = p >= 0 && p <= g.nz, pinz = p >= 0 && p < g.nz;
    C2<T> *fs = &sm.f[slot][0][0];
    T *ss = &sm.s[slot][0][0];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        if (m.goff[q] == INT_MIN) continue;
        const int comp = (m.cm >> (2 * q)) & 3;
        const bool ok = m.goff[q] >= 0 && (comp == 2 ? pinz : pin);
        const int e = ok ? m.goff[q] + (comp == 0 ? psx : comp == 1 ? psy : psz) : 0;
        const int t = threadIdx.x + kThreads * q;
        cp_async_zfill<sizeof(C2<T>)>(fs + t, x + e, ok);
        cp_async_zfill<sizeof(T)>(ss + t, sig + e, ok);
    }
    if (gdn) {
        const int pn = (g.nx + 1) * (g.ny + 1) * p;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            if (m.goffn[q] == INT_MIN) continue;
            const bool ok = m.goffn[q] >= 0 && pin;
            cp_async_zfill<sizeof(T)>(&sm.nw[p & 1][threadIdx.x + kThreads * q], gdn + (ok ? m.goffn[q] + pn : 0), ok);
        }
    }
    cp_async_commit();
}

// grad-div potential of node (i, j, p) (local node ni, nj of the tile) from
// the staged Ex, Ey of plane p and Ez of planes p-1, p: the sums of
// k_gd_phi (mode 0) in the same order.  The staged node weight carries the
// earth flag in its sign: w < 0 marks an earth node of weight |w|.  dX, dY
// are delX[i], delY[j]; dZ is delZ[p].
template <typename T>
__device__ __forceinline__ C2<T> stage_phi_node(const StageSmem<T> &sm, const Geo<T> &g, int i, int j, int p, int ni,
                                                int nj, T dX, T dY, T dZ)
{
    if (!(i >= 1 && i <= g.nx - 1 && j >= 1 && j <= g.ny - 1 && p >= 1 && p <= g.nz - 1)) return mk<T>(0, 0);
    const int sp = p & (kRing - 1), sz = (p - 1) & (kRing - 1);
    const T wn = sm.nw[p & 1][nj * kNX + ni];
    const int h = (nj + 1) * kHX + ni + 1;
    const T dfa0 = dY * dZ, dfa1 = dX * dZ, dfa2 = dX * dY;
    const C2<T> *fp = sm.f[sp][0], *fz = sm.f[sz][2];
    C2<T> acc;
    if (wn < T(0)) {  // earth node: C = sigma_E
        const T *sp0 = sm.s[sp][0], *szz = sm.s[sz][2];
        acc = cscale(fp[h - 1], dfa0 * sp0[h - 1]);                          // Ex(i-1, j, p): ends at the node
        acc = csub(acc, cscale(fp[h], dfa0 * sp0[h]));                        // Ex(i, j, p): starts at the node
        acc = cadd(acc, cscale(fp[kHP + h - kHX], dfa1 * sp0[kHP + h - kHX]));  // Ey(i, j-1, p)
        acc = csub(acc, cscale(fp[kHP + h], dfa1 * sp0[kHP + h]));            // Ey(i, j, p)
        acc = cadd(acc, cscale(fz[h], dfa2 * szz[h]));                        // Ez(i, j, p-1)
        acc = csub(acc, cscale(fp[2 * kHP + h], dfa2 * sp0[2 * kHP + h]));    // Ez(i, j, p)
        return cscale(acc, -wn);
    }
    acc = cscale(fp[h - 1], dfa0);
    acc = csub(acc, cscale(fp[h], dfa0));
    acc = cadd(acc, cscale(fp[kHP + h - kHX], dfa1));
    acc = csub(acc, cscale(fp[kHP + h], dfa1));
    acc = cadd(acc, cscale(fz[h], dfa2));
    acc = csub(acc, cscale(fp[2 * kHP + h], dfa2));
    return cscale(acc, wn);
}

// March planes [k0, k1) of the tile (i0, j0) for the input field x (one
// right-hand side).  For every existing edge of the thread's node column
// calls f(comp, e, interior, Ax, x_e, aux_e) with Ax = (A x)_e on interior
// edges (zero otherwise) and aux_e the entry of the auxiliary vector aux
// (read one plane ahead; zero when aux is null).  With gdn non-null (signed
// node weights) the grad-div term DFA_e (phi_end - phi_start) is added.
// Every thread of the block must call this (barriers inside).
template <typename T, typename F>
__device__ __forceinline__ void stage_march(StageSmem<T> &sm, const Geo<T> &g, const C2<T> *__restrict__ x,
                                            const T *__restrict__ sig, const T *__restrict__ gdn,
                                            const C2<T> *__restrict__ aux, T wmu, int i0, int j0, int k0, int k1,
                                            F &&f)
{
    using C = C2<T>;
    const int tx = threadIdx.x % kStX, ty = threadIdx.x / kStX;
    const int i = i0 + tx, j = j0 + ty;
    const bool live = i <= g.nx && j <= g.ny;
    const ColGeo<T> cg = col_geo(g, min(i, g.nx), min(j, g.ny));
    const int h = (ty + 1) * kHX + tx + 1;  // own entry in a staged plane
    const int hn = ty * kNX + tx;           // own node in a potential plane
    const int sxj = g.nx, syj = g.nx + 1, szj = g.nx + 1;
    const int bx = i + sxj * j, by = g.nXe + i + syj * j, bz = g.nXe + g.nYe + i + szj * j;
    const int sxk = g.nx * (g.ny + 1), syk = (g.nx + 1) * g.ny, szk = (g.nx + 1) * (g.ny + 1);
    const C zero = mk<T>(0, 0);
    const bool gd = gdn != nullptr;
    const StageMap map = stage_map(g, i0, j0);
    // halo node of this thread (threads 0..kStX-1: row j0 + kStY; the next
    // kStY + 1: column i0 + kStX), potentials of the tile's +i / +j halo
    const bool hasH = threadIdx.x < kStX + kNY;
    const int hni = threadIdx.x < kStX ? threadIdx.x : kStX;
    const int hnj = threadIdx.x < kStX ? kStY : threadIdx.x - kStX;
    const int hi = i0 + hni, hj = j0 + hnj;
    const T hdX = (hasH && hi <= g.nx) ? g.delX[hi] : T(0), hdY = (hasH && hj <= g.ny) ? g.delY[hj] : T(0);
    auto phi_plane = [&](int p) {
        const T dZ = (p >= 0 && p <= g.nz) ? g.delZ[p] : T(0);
        sm.phi[p & 1][hn] = stage_phi_node(sm, g, i, j, p, tx, ty, cg.delXi, cg.delYj, dZ);
        if (hasH) sm.phi[p & 1][hnj * kNX + hni] = stage_phi_node(sm, g, hi, hj, p, hni, hnj, hdX, hdY, dZ);
    };
    // aux entries of the own edges of plane k (ax, ay, az)
    C ax = zero, ay = zero, az = zero;
    auto load_aux = [&](int k) {
        if (!aux || !live || k > g.nz) return;
        if (cg.hasX) ax = aux[bx + sxk * k];
        if (cg.hasY) ay = aux[by + syk * k];
        if (k < g.nz) az = aux[bz + szk * k];
    };
    load_aux(k0);
    stage_plane(sm, g, map, x, sig, (const T *)nullptr, k0 - 1);  // node weights of k0 - 1 are not needed
    stage_plane(sm, g, map, x, sig, gdn, k0);
    stage_plane(sm, g, map, x, sig, gdn, k0 + 1);
    cp_async_wait_all();
    __syncthreads();
    if (gd) phi_plane(k0);
    for (int k = k0; k < k1; k++) {
        stage_plane(sm, g, map, x, sig, gdn, k + 2);
        if (gd) phi_plane(k + 1);
        __syncthreads();
        if (live) {
            const int sm1 = (k - 1) & (kRing - 1), s0 = k & (kRing - 1), s1 = (k + 1) & (kRing - 1);
            const C *Xm = sm.f[sm1][0], *X0 = sm.f[s0][0], *Xp = sm.f[s1][0];
            const C *Ym = sm.f[sm1][1], *Y0 = sm.f[s0][1], *Yp = sm.f[s1][1];
            const C *Zm = sm.f[sm1][2], *Z0 = sm.f[s0][2];
            const C *P0 = sm.phi[k & 1], *P1 = sm.phi[(k + 1) & 1];
            const PlaneGeo<T> pg = plane_geo(g, k);
            const bool kin = k >= 1 && k <= g.nz - 1;
            // ---- Ex(i, j, k)
            if (cg.hasX) {
                const int e = bx + sxk * k;
                const C X1 = X0[h];
                const T dt = wmu * sm.s[s0][0][h] * (cg.dxi * (cg.delYj * pg.delZk));
                C out = zero;
                const bool in = cg.intX && kin;
                if (in) {
                    const C yy = csub(cadd(csub(Y0[h + 1], Y0[h]), Y0[h - kHX]), Y0[h + 1 - kHX]);
                    const C zz = csub(cadd(csub(Z0[h + 1], Z0[h]), Zm[h]), Zm[h + 1]);
                    const C fyp = cscale(csub(X0[h + kHX], X1), cg.rdyj);
                    const C fym = cscale(csub(X1, X0[h - kHX]), cg.rdyjm1);
                    const C fzp = cscale(csub(Xp[h], X1), pg.rdzk);
                    const C fzm = cscale(csub(X1, Xm[h]), pg.rdzkm1);
                    out = cadd(cscale(yy, pg.delZk), cscale(zz, cg.delYj));
                    out = csub(out, cscale(csub(fyp, fym), cg.dxi * pg.delZk));
                    out = csub(out, cscale(csub(fzp, fzm), cg.dxi * cg.delYj));
                    out.x -= dt * X1.y;
                    out.y += dt * X1.x;
                    if (gd) out = cadd(out, cscale(csub(P0[hn + 1], P0[hn]), cg.delYj * pg.delZk));
                }
                f(0, e, in, out, X1, ax);
            }
            // ---- Ey(i, j, k)
            if (cg.hasY) {
                const int e = by + syk * k;
                const C Y1 = Y0[h];
                const T dt = wmu * sm.s[s0][1][h] * (cg.dyj * (cg.delXi * pg.delZk));
                C out = zero;
                const bool in = cg.intY && kin;
                if (in) {
                    const C zz = csub(cadd(csub(Z0[h + kHX], Z0[h]), Zm[h]), Zm[h + kHX]);
                    const C xx = csub(cadd(csub(X0[h + kHX], X0[h]), X0[h - 1]), X0[h - 1 + kHX]);
                    const C fzp = cscale(csub(Yp[h], Y1), pg.rdzk);
                    const C fzm = cscale(csub(Y1, Ym[h]), pg.rdzkm1);
                    const C fxp = cscale(csub(Y0[h + 1], Y1), cg.rdxi);
                    const C fxm = cscale(csub(Y1, Y0[h - 1]), cg.rdxim1);
                    out = cadd(cscale(zz, cg.delXi), cscale(xx, pg.delZk));
                    out = csub(out, cscale(csub(fzp, fzm), cg.dyj * cg.delXi));
                    out = csub(out, cscale(csub(fxp, fxm), cg.dyj * pg.delZk));
                    out.x -= dt * Y1.y;
                    out.y += dt * Y1.x;
                    if (gd) out = cadd(out, cscale(csub(P0[hn + kNX], P0[hn]), cg.delXi * pg.delZk));
                }
                f(1, e, in, out, Y1, ay);
            }
            // ---- Ez(i, j, k)
            if (k < g.nz) {
                const int e = bz + szk * k;
                const C Z1 = Z0[h];
                const T dt = wmu * sm.s[s0][2][h] * (pg.dzk * (cg.delXi * cg.delYj));
                C out = zero;
                const bool in = cg.intZ;
                if (in) {
                    const C xx = csub(cadd(csub(Xp[h], X0[h]), X0[h - 1]), Xp[h - 1]);
                    const C yy = csub(cadd(csub(Yp[h], Y0[h]), Y0[h - kHX]), Yp[h - kHX]);
                    const C fxp = cscale(csub(Z0[h + 1], Z1), cg.rdxi);
                    const C fxm = cscale(csub(Z1, Z0[h - 1]), cg.rdxim1);
                    const C fyp = cscale(csub(Z0[h + kHX], Z1), cg.rdyj);
                    const C fym = cscale(csub(Z1, Z0[h - kHX]), cg.rdyjm1);
                    out = cadd(cscale(xx, cg.delYj), cscale(yy, cg.delXi));
                    out = csub(out, cscale(csub(fxp, fxm), pg.dzk * cg.delYj));
                    out = csub(out, cscale(csub(fyp, fym), pg.dzk * cg.delXi));
                    out.x -= dt * Z1.y;
                    out.y += dt * Z1.x;
                    if (gd) out = cadd(out, cscale(csub(P1[hn], P0[hn]), cg.delXi * cg.delYj));
                }
                f(2, e, in, out, Z1, az);
            }
            if (k + 1 < k1) load_aux(k + 1);
        }
        cp_async_wait_all();
        __syncthreads();
    }
}

}  // namespace mt3d

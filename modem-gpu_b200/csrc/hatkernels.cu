// hatkernels.cu -- the FP32 BiCGStab iteration of the mixed-precision solve
// with the diagonal preconditioner fused into the operator kernels.
//
// BiCGStab right-preconditioned with D = diag(A) (BICG, f90/3D_MT/FWD/
// solver.f90:346-555, as the unfused kernels run it) is carried in
// preconditioned variables: u = D^-1 p, vh = D^-1 v, rh = D^-1 r,
// sh = D^-1 s, th = D^-1 t.  Then every vector update is a plain axpy, the
// preconditioner is one division at the output edge of the operator kernels
// (vh = D^-1 A u, th = D^-1 A sh), and no vector of D^-1 exists:
//
//   kh_u         u  = rh + beta (u - omega vh)   (u = rh on the first iteration)
//   kh_vt st. 0  vh = D^-1 A u,       (rt, v)                  -> alpha
//   kh_s         sh = rh - alpha vh
//   kh_vt st. 1  th = D^-1 A sh,      (t, s), (t, t), (s, s)   -> omega, ||r||
//   kh_xr        x += alpha u + omega sh,  rh = sh - omega th,  (rt, r) -> beta
//
// 163 bytes per edge and iteration instead of the 211 of the unfused
// kernels (kb_p, kct_vt, kb_s, kct_vt, kb_xr).  With the polynomial
// preconditioner M^-1 = c D^-1 (2 I - c A D^-1) each operator launch becomes
// two (stages 2, 3 and 4, 5 of hat_vt); kh_xr accumulates yhat = sum (alpha
// u + omega sh) as in the diagonal case, and the end of the cycle turns the
// best yhat into x = M^-1 D yhat = c (2 yhat - c D^-1 A yhat) (stage 6 and
// kh_conv).  The inner products of the
// method in the original variables follow from the hat ones:
//   - the shadow residual is the reference's rt = r0 = b; with y =
//     conj(D) b stored once per cycle (written by kh_cast), (rt, r) =
//     sum conj(y) rh and (rt, v) = sum conj(y) vh;
//   - with W = |D|^2 per edge, computed in the operator kernel where D is,
//     (t, s) = sum W conj(th) sh, (t, t) = sum W |th|^2, and the true
//     residual norm of the new iterate follows without another pass:
//     ||s - omega t||^2 = ||s||^2 - 2 Re(conj(omega) (t, s)) + |omega|^2 ||t||^2.
// The iterates, step lengths and residual norms are those of the unfused
// kernels up to rounding.  (A shadow generated from the edge index instead
// of a stored one, rt = D^-H z with z = +-1 +- i, saves 16 bytes an
// iteration, but its entries scale as 1/|D|, which on the benchmark model
// cost 40 % more iterations and on the reference's cylinder model stalled
// the solve.)
//
// The operator kernels stage u or sh with the tensor copies of tma.cuh.  D =
// V_E xXO-diagonal of the curl-curl term (col_ccdiag) + the grad-div diagonal
// DFA^2 (w_s c_s + w_e c_e) + i omega mu0 sigma V_E, from the staged sigma
// and signed node weights (the weights of each node column's three nodes at
// plane k are kept in registers from the previous plane, so the node ring
// keeps two slots).  kh_cast computes the same D from the global tables.
#include <atomic>
#include <cstring>

#include "finalize.cuh"
#include "tma.cuh"

namespace mt3d {

extern std::atomic<long long> g_launch_count;
static inline void counted(int n) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

// diagonal of A at an interior edge: dr + i di
__device__ __forceinline__ void hat_diag(int comp, const ColGeo<float> &cg, const PlaneGeo<float> &pg, float wmu,
                                         float sig, bool gd, float wns, float wne, float &dr, float &di)
{
    float ve, dfa;
    if (comp == 0) {
        ve = cg.dxi * (cg.delYj * pg.delZk);
        dfa = cg.delYj * pg.delZk;
    } else if (comp == 1) {
        ve = cg.dyj * (cg.delXi * pg.delZk);
        dfa = cg.delXi * pg.delZk;
    } else {
        ve = pg.dzk * (cg.delXi * cg.delYj);
        dfa = cg.delXi * cg.delYj;
    }
    dr = col_ccdiag(comp, cg, pg);
    if (gd) {
        const float cs = wns < 0.f ? sig : 1.f, ce = wne < 0.f ? sig : 1.f;
        dr += dfa * dfa * (fabsf(wns) * cs + fabsf(wne) * ce);
    }
    di = wmu * sig * ve;
}

// y / D and |D|^2 (the fast reciprocal intrinsic: D^-1 only has to be the
// same in every kernel that applies it, which one function guarantees)
__device__ __forceinline__ float2 hat_div(float2 y, float dr, float di, float &W)
{
    W = dr * dr + di * di;
    const float inv = __fdividef(1.f, W);
    return make_float2((y.x * dr + y.y * di) * inv, (y.y * dr - y.x * di) * inv);
}

// ---------------------------------------------------------------------------
// start of an FP32 cycle: rh = D^-1 b with b = r64 scale on the padded
// layout, the shadow y = conj(D) b (rt = b), x = 0; ||b||^2 = rho = (rt, r).
// The first guess is zero, so r = b and no operator pass is needed.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) kh_cast(KArgs<float> a, const double2 *r64, size_t stride64)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    const Geo<float> &g = a.g;
    const size_t off = (size_t)r * stride64, offp = (size_t)r * a.stride;
    const double sc = a.ost[r].scale;
    const float wmu = (float)(a.dsgn * a.ost[r].omega * kMu0);
    double u[1] = {0.0};
    for (int e = blockIdx.x * kThreads + threadIdx.x; e < g.nE; e += gridDim.x * kThreads) {
        const EdgeIdx q = edge_decode(g, e);
        const int pe = a.pl.idx(q.c, q.i, q.j, q.k);
        const double2 v = r64[off + e];
        const float2 b = make_float2((float)(v.x * sc), (float)(v.y * sc));
        float2 rh = make_float2(0.f, 0.f), y = rh;
        if (edge_interior(g, q)) {
            const ColGeo<float> cg = col_geo(g, q.i, q.j);
            const PlaneGeo<float> pg = plane_geo(g, q.k);
            float wns = 0.f, wne = 0.f;
            if (a.gd) {
                const int ns = iN(g, q.i, q.j, q.k);
                wns = a.gdn[ns];
                wne = a.gdn[q.c == 0 ? ns + 1 : q.c == 1 ? ns + g.nx + 1 : ns + (g.nx + 1) * (g.ny + 1)];
            }
            float dr, di, W;
            hat_diag(q.c, cg, pg, wmu, a.sigma[e], a.gd != 0, wns, wne, dr, di);
            rh = hat_div(b, dr, di, W);
            y = make_float2(dr * b.x + di * b.y, dr * b.y - di * b.x);  // conj(D) b
            u[0] += (double)b.x * b.x + (double)b.y * b.y;
        }
        a.r[offp + pe] = rh;
        a.rt[offp + pe] = y;
        a.x0[offp + pe] = make_float2(0.f, 0.f);
    }
    double tot[1];
    if (block_reduce_last<1>(u, a.parts, a.cnt, r, blockIdx.x, gridDim.x, tot) && threadIdx.x == 0) {
        const double t2[2] = {tot[0], tot[0]};
        fin_init(a.st[r], t2, a.rerr + (size_t)r * a.rerr_stride, a.maxit, a.ost[r].tol_inner);
    }
}

// ---------------------------------------------------------------------------
// elementwise kernels (two complex entries per thread and step)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 c2mul2(float2 c, float4 v)
{
    return make_float4(c.x * v.x - c.y * v.y, c.x * v.y + c.y * v.x, c.x * v.z - c.y * v.w, c.x * v.w + c.y * v.z);
}
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 sub4(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

// pairs of entries of block bx of a right-hand side (a.chunk entries per block)
#define HAT_PAIRS(a, bx)                                                             \
    const int hp_n2 = (a).len / 2, hp_c2 = (a).chunk / 2;                            \
    const int q1 = min(((bx) + 1) * hp_c2, hp_n2);                                    \
    for (int q = (bx) * hp_c2 + threadIdx.x; q < q1; q += kThreads)

// u = rh + beta (u - omega vh); u = rh on the first iteration of a cycle or
// after a restart (block bx of right-hand side r)
__device__ __forceinline__ void hat_u(const KArgs<float> &a, int r, int bx)
{
    const BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride / 2;
    const float4 *RH = reinterpret_cast<const float4 *>(a.r) + off;
    const float4 *VH = reinterpret_cast<const float4 *>(a.v) + off;
    float4 *U = reinterpret_cast<float4 *>(a.ph) + off;
    if (st.first) {
        HAT_PAIRS(a, bx) U[q] = RH[q];
        return;
    }
    const float2 be = make_float2((float)st.beta.re, (float)st.beta.im);
    const float2 om = make_float2((float)st.omega.re, (float)st.omega.im);
    HAT_PAIRS(a, bx) U[q] = add4(RH[q], c2mul2(be, sub4(U[q], c2mul2(om, VH[q]))));
}

// sh = rh - alpha vh
__device__ __forceinline__ void hat_s(const KArgs<float> &a, int r, int bx)
{
    const BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride / 2;
    const float4 *RH = reinterpret_cast<const float4 *>(a.r) + off;
    const float4 *VH = reinterpret_cast<const float4 *>(a.v) + off;
    float4 *SH = reinterpret_cast<float4 *>(a.sh) + off;
    const float2 al = make_float2((float)st.alpha.re, (float)st.alpha.im);
    HAT_PAIRS(a, bx) SH[q] = sub4(RH[q], c2mul2(al, VH[q]));
}

// x += alpha u + omega sh (into the buffer that does not hold the best
// iterate); rh = sh - omega th; rho = (z, rh).  The true residual norm of the
// new iterate comes from the inner products of kh_vt stage 1 or 5
// (BicgState::rn2).
__device__ __forceinline__ void hat_xr(const KArgs<float> &a, int r, int bx)
{
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride / 2;
    const float2 al = make_float2((float)st.alpha.re, (float)st.alpha.im);
    const float2 om = make_float2((float)st.omega.re, (float)st.omega.im);
    const int cur = st.xcur, dst = (st.xcur == st.xbest) ? 1 - st.xcur : st.xcur;
    const float4 *XS = reinterpret_cast<const float4 *>(cur == 0 ? a.x0 : a.x1) + off;
    float4 *XD = reinterpret_cast<float4 *>(dst == 0 ? a.x0 : a.x1) + off;
    const float4 *U = reinterpret_cast<const float4 *>(a.ph) + off;
    const float4 *SH = reinterpret_cast<const float4 *>(a.sh) + off;
    const float4 *TH = reinterpret_cast<const float4 *>(a.t) + off;
    float4 *RH = reinterpret_cast<float4 *>(a.r) + off;
    const float4 *Y = reinterpret_cast<const float4 *>(a.rt) + off;
    // with the polynomial preconditioner the iterate is x = M^-1 yhat, and
    // yhat = sum (alpha u + omega sh) accumulates here like the diagonal
    // case's x (u = D^-1 p, sh = D^-1 s); launch_hat_conv turns the cycle's
    // best yhat into x = c (2 yhat - c D^-1 A yhat) at its end
    double u[2] = {0.0, 0.0};
    HAT_PAIRS(a, bx)
    {
        const float4 sh = SH[q];
        XD[q] = add4(add4(XS[q], c2mul2(al, U[q])), c2mul2(om, sh));
        const float4 rn = sub4(sh, c2mul2(om, TH[q]));
        RH[q] = rn;
        const float4 y = Y[q];  // conj(y) rh
        u[0] += (double)y.x * rn.x + (double)y.y * rn.y + (double)y.z * rn.z + (double)y.w * rn.w;
        u[1] += (double)y.x * rn.y - (double)y.y * rn.x + (double)y.z * rn.w - (double)y.w * rn.z;
    }
    double tot[2];
    if (block_reduce_last<2>(u, a.parts, a.cnt, r, bx, a.nblk, tot) && threadIdx.x == 0) {
        double *rerr = a.rerr + (size_t)r * a.rerr_stride;
        const double rnorm = sqrt(st.rn2);
        st.iter += 1;
        st.xcur = dst;
        st.first = 0;
        st.rnorm = rnorm;
        rerr[st.iter - 1] = rnorm / st.bnorm;
        if (!isfinite(rnorm) || !isfinite(tot[0]) || !isfinite(tot[1])) { st.status = KS_NAN; return; }
        if (rnorm < st.btol) {
            st.status = KS_CONVERGED;
            st.xbest = dst;
            return;
        }
        if (rnorm < st.rnormin) {
            st.rnormin = rnorm;
            st.xbest = dst;
            st.imin = st.iter;
        }
        if (st.iter >= st.maxit) {
            st.status = KS_MAXIT;
            return;
        }
        const cd rho_new = {tot[0], tot[1]};
        if (a.restart > 0 && st.iter % a.restart == 0) {
            // restart towards steepest descent (cuBiCG, f90/3D_MT/FWD_SP2/
            // solver.f90:1545-1573): rt = r, rho = (rt, r) = ||r||^2, p = r,
            // omega = 1; the next kh_vt stage 0 or 2 writes the new shadow y = W rh
            st.first = 1;
            st.pad = 1;
            st.rho = {st.rn2, 0.0};
            st.omega = {1.0, 0.0};
            if (cd_zero(st.rho)) st.status = KS_BREAKDOWN;
            return;
        }
        st.rho1 = st.rho;
        st.rho = rho_new;
        if (cd_zero(st.rho)) { st.status = KS_BREAKDOWN; return; }
        st.beta = cd_mul(cd_div(st.rho, st.rho1), cd_div(st.alpha, st.omega));
        if (cd_zero(st.beta)) st.status = KS_BREAKDOWN;
    }
}

// ---------------------------------------------------------------------------
// the operator kernels: the staged stencil of tmakernels.cu with the output
// divided by D at the edge
// ---------------------------------------------------------------------------

// March planes [k0, k1) of tile (i0, j0), right-hand side r, calling
// f(e, yhat, x_e, W, aux_e) for the three edge slots (Ex, Ey, Ez) of every
// node of the thread's two columns, padding slots included: yhat =
// D^-1 (A x)_e and W = |D_e|^2 at interior edges (zero otherwise), e the
// padded index, aux_e the entry of the vector aux (read one plane ahead,
// zero when aux is null).  A block of kHatThreads threads covers the 32 x 8
// node tile: thread (tx, ty) takes the node columns (i0 + tx, j0 + ty) and
// (i0 + tx, j0 + ty + 4), so the per-plane work of a thread (waits,
// barriers, plane geometry, loop control) is shared by six edges and the
// register budget of four blocks per SM is 128 per thread.  Returns false
// (all threads of the block alike) when a wait gave up.
template <bool gd, typename F>
__device__ __forceinline__ bool hat_march(TmaSmem &sm, const TmaParams &tp, const Geo<float> &g, PadLayout pl, int r,
                                          const float2 *__restrict__ aux, float wmu, int i0, int j0, int k0, int k1,
                                          int *err, int limit, F &&f)
{
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    const int i = i0 + tx, jA = j0 + ty, jB = jA + kHatRows;
    const bool liveA = i <= g.nx && jA <= g.ny, liveB = i <= g.nx && jB <= g.ny;
    const ColGeo<float> cgA = col_geo(g, min(i, g.nx), min(jA, g.ny));
    const ColGeo<float> cgB = col_geo(g, min(i, g.nx), min(jB, g.ny));
    const int hfA = (ty + 1) * kFW + tx + 2;  // own column in a field plane of the tile
    const int hsA = (ty + 1) * kSW + tx + 4;  // own column in a sigma plane
    const int hnA = ty * kPhX + tx;           // own node in a potential plane
    const int hwA = ty * kNW + tx;            // own node in a node-weight plane
    constexpr int dF = kHatRows * kFW, dS = kHatRows * kSW, dN = kHatRows * kPhX, dW = kHatRows * kNW;
    const int cf = kFR * kFW, cs = kFR * kSW;
    const int pxy = pl.Px * pl.Py, pc = pl.Pz * pxy;
    const int colA = min(i, pl.Px - 1) + pl.Px * min(jA, pl.Py - 1);
    const int colB = min(i, pl.Px - 1) + pl.Px * min(jB, pl.Py - 1);
    const bool issuer = threadIdx.x == 0;
    const unsigned tx_bytes = kFBytes + kSBytes;
    // halo nodes of the potentials: (i0 + 32, j0 .. j0 + 8) and (i0 .. i0 + 31, j0 + 8)
    const bool hasH = threadIdx.x < kTX + kTY + 1;
    const int hni = threadIdx.x < kTX ? threadIdx.x : kTX;
    const int hnj = threadIdx.x < kTX ? kTY : threadIdx.x - kTX;
    const int hi = i0 + hni, hj = j0 + hnj;
    const float hdX = (hasH && hi <= g.nx) ? g.delX[hi] : 0.f, hdY = (hasH && hj <= g.ny) ? g.delY[hj] : 0.f;

    // a chunk past the last node plane (the last chunks when the chunk count
    // does not divide the planes) has no work; it must return before it
    // issues a copy, since it would never wait for its third plane
    if (k0 >= k1) return true;
    if ((smem_addr(sm.fld[0]) | smem_addr(sm.sig[0]) | smem_addr(sm.nod[0])) & 127u) {
        if (issuer) atomicExch(err, 2);
        return false;
    }
    if (issuer) {
        for (int q = 0; q < 4; q++) mbar_init(smem_addr(&sm.mbar[q]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    unsigned phase = 0;
    // node weights are staged for planes k0 .. k1 (the diagonal and the
    // potentials need them), in slot p & 1
    auto issue = [&](int p) {
        if (!issuer) return;
        const int s = p & 3;
        const bool node = gd && p >= k0;
        const unsigned mb = smem_addr(&sm.mbar[s]);
        mbar_expect(mb, tx_bytes + (node ? kNBytes : 0u));
        tma_load4(smem_addr(sm.fld[s]), &tp.in, 2 * (i0 - 2), j0 - 1, p, 3 * r, mb);
        tma_load4(smem_addr(sm.sig[mod3(p)]), &tp.sig, i0 - 4, j0 - 1, p, 0, mb);
        if (node) tma_load3(smem_addr(sm.nod[p & 1]), &tp.node, i0, j0, p, mb);
    };
    auto wait = [&](int p) -> bool {
        const int s = p & 3;
        if (mbar_wait(smem_addr(&sm.mbar[s]), (phase >> s) & 1u, limit)) {
            phase ^= 1u << s;
            return true;
        }
        return false;
    };
    auto give_up = [&](int first, int last) {
        if (!issuer) return;
        atomicExch(err, 1);
        for (int q = first; q <= last; q++)
            if (mbar_wait(smem_addr(&sm.mbar[q & 3]), (phase >> (q & 3)) & 1u, kWaitLimit)) phase ^= 1u << (q & 3);
    };
    auto phi_plane = [&](int p) {
        const float dZ = (p >= 0 && p <= g.nz) ? g.delZ[p] : 0.f;
        float2 *P = sm.phi[p & 1];
        P[hnA] = tma_phi_node(sm, g, i, jA, p, tx, ty, cgA.delXi, cgA.delYj, dZ);
        P[hnA + dN] = tma_phi_node(sm, g, i, jB, p, tx, ty + kHatRows, cgB.delXi, cgB.delYj, dZ);
        if (hasH) P[hnj * kPhX + hni] = tma_phi_node(sm, g, hi, hj, p, hni, hnj, hdX, hdY, dZ);
    };
    const float2 zero = make_float2(0.f, 0.f);
    // signed node weights of each column's nodes (i, j), (i+1, j), (i, j+1)
    // at the plane being computed
    float wSA = 0.f, wXA = 0.f, wYA = 0.f, wSB = 0.f, wXB = 0.f, wYB = 0.f;
    auto node_w = [&](int p, float &sa, float &xa, float &ya, float &sb, float &xb, float &yb) {
        const float *N = reinterpret_cast<const float *>(sm.nod[p & 1]);
        sa = N[hwA];
        xa = N[hwA + 1];
        ya = N[hwA + kNW];
        sb = N[hwA + dW];
        xb = N[hwA + dW + 1];
        yb = N[hwA + dW + kNW];
    };
    // (padding entries of aux, where Ex, Ey or Ez does not exist, are zero)
    float2 axA = zero, ayA = zero, azA = zero, axB = zero, ayB = zero, azB = zero;
    auto load_aux = [&](int k) {
        if (!aux || k > g.nz) return;
        if (liveA) {
            const int b = colA + pxy * k;
            axA = aux[b];
            ayA = aux[pc + b];
            azA = aux[2 * pc + b];
        }
        if (liveB) {
            const int b = colB + pxy * k;
            axB = aux[b];
            ayB = aux[pc + b];
            azB = aux[2 * pc + b];
        }
    };

    // the three edges of one node column at plane k.  Every edge slot is
    // formed without branches: an edge that is not interior (or does not
    // exist: Ex at i = nx, Ey at j = ny, Ez at k = nz, all padding entries
    // of the layout) gets yhat = 0 and W = 0, so it adds nothing to the
    // inner products and keeps its zero.  The shared-memory reads stay
    // inside the tile whatever the edge.
    auto node_edges = [&](const ColGeo<float> &cg, const PlaneGeo<float> &pg, int k, bool kin, int h, int hs, int hn,
                          float wS, float wX, float wY, float nS, int eb, float2 ax, float2 ay, float2 az) {
        const float2 *Fm = reinterpret_cast<const float2 *>(sm.fld[(k - 1) & 3]);
        const float2 *F0 = reinterpret_cast<const float2 *>(sm.fld[k & 3]);
        const float2 *Fp = reinterpret_cast<const float2 *>(sm.fld[(k + 1) & 3]);
        const float *S0 = reinterpret_cast<const float *>(sm.sig[k % 3]);
        const float2 *Xm = Fm, *X0 = F0, *Xp = Fp;
        const float2 *Ym = Fm + cf, *Y0 = F0 + cf, *Yp = Fp + cf;
        const float2 *Zm = Fm + 2 * cf, *Z0 = F0 + 2 * cf;
        const float2 *P0 = sm.phi[k & 1], *P1 = sm.phi[(k + 1) & 1];
        // ---- Ex(i, j, k)
        {
            const float2 X1 = X0[h];
            const bool in = cg.intX && kin;
            float dr, di, W;
            hat_diag(0, cg, pg, wmu, S0[hs], gd, wS, wX, dr, di);
            const float2 yy = csub(cadd(csub(Y0[h + 1], Y0[h]), Y0[h - kFW]), Y0[h + 1 - kFW]);
            const float2 zz = csub(cadd(csub(Z0[h + 1], Z0[h]), Zm[h]), Zm[h + 1]);
            const float2 fyp = cscale(csub(X0[h + kFW], X1), cg.rdyj);
            const float2 fym = cscale(csub(X1, X0[h - kFW]), cg.rdyjm1);
            const float2 fzp = cscale(csub(Xp[h], X1), pg.rdzk);
            const float2 fzm = cscale(csub(X1, Xm[h]), pg.rdzkm1);
            float2 out = cadd(cscale(yy, pg.delZk), cscale(zz, cg.delYj));
            out = csub(out, cscale(csub(fyp, fym), cg.dxi * pg.delZk));
            out = csub(out, cscale(csub(fzp, fzm), cg.dxi * cg.delYj));
            out.x -= di * X1.y;
            out.y += di * X1.x;
            if (gd) out = cadd(out, cscale(csub(P0[hn + 1], P0[hn]), cg.delYj * pg.delZk));
            out = hat_div(out, dr, di, W);
            f(eb, in ? out : zero, X1, in ? W : 0.f, ax);
        }
        // ---- Ey(i, j, k)
        {
            const float2 Y1 = Y0[h];
            const bool in = cg.intY && kin;
            float dr, di, W;
            hat_diag(1, cg, pg, wmu, S0[cs + hs], gd, wS, wY, dr, di);
            const float2 zz = csub(cadd(csub(Z0[h + kFW], Z0[h]), Zm[h]), Zm[h + kFW]);
            const float2 xx = csub(cadd(csub(X0[h + kFW], X0[h]), X0[h - 1]), X0[h - 1 + kFW]);
            const float2 fzp = cscale(csub(Yp[h], Y1), pg.rdzk);
            const float2 fzm = cscale(csub(Y1, Ym[h]), pg.rdzkm1);
            const float2 fxp = cscale(csub(Y0[h + 1], Y1), cg.rdxi);
            const float2 fxm = cscale(csub(Y1, Y0[h - 1]), cg.rdxim1);
            float2 out = cadd(cscale(zz, cg.delXi), cscale(xx, pg.delZk));
            out = csub(out, cscale(csub(fzp, fzm), cg.dyj * cg.delXi));
            out = csub(out, cscale(csub(fxp, fxm), cg.dyj * pg.delZk));
            out.x -= di * Y1.y;
            out.y += di * Y1.x;
            if (gd) out = cadd(out, cscale(csub(P0[hn + kPhX], P0[hn]), cg.delXi * pg.delZk));
            out = hat_div(out, dr, di, W);
            f(pc + eb, in ? out : zero, Y1, in ? W : 0.f, ay);
        }
        // ---- Ez(i, j, k)
        {
            const float2 Z1 = Z0[h];
            const bool in = cg.intZ && k < g.nz;
            float dr, di, W;
            hat_diag(2, cg, pg, wmu, S0[2 * cs + hs], gd, wS, nS, dr, di);
            const float2 xx = csub(cadd(csub(Xp[h], X0[h]), X0[h - 1]), Xp[h - 1]);
            const float2 yy = csub(cadd(csub(Yp[h], Y0[h]), Y0[h - kFW]), Yp[h - kFW]);
            const float2 fxp = cscale(csub(Z0[h + 1], Z1), cg.rdxi);
            const float2 fxm = cscale(csub(Z1, Z0[h - 1]), cg.rdxim1);
            const float2 fyp = cscale(csub(Z0[h + kFW], Z1), cg.rdyj);
            const float2 fym = cscale(csub(Z1, Z0[h - kFW]), cg.rdyjm1);
            float2 out = cadd(cscale(xx, cg.delYj), cscale(yy, cg.delXi));
            out = csub(out, cscale(csub(fxp, fxm), pg.dzk * cg.delYj));
            out = csub(out, cscale(csub(fyp, fym), pg.dzk * cg.delXi));
            out.x -= di * Z1.y;
            out.y += di * Z1.x;
            if (gd) out = cadd(out, cscale(csub(P1[hn], P0[hn]), cg.delXi * cg.delYj));
            out = hat_div(out, dr, di, W);
            f(2 * pc + eb, in ? out : zero, Z1, in ? W : 0.f, az);
        }
    };

    load_aux(k0);
    issue(k0 - 1);
    issue(k0);
    issue(k0 + 1);
    {
        const bool w0 = wait(k0 - 1), w1 = w0 && wait(k0);
        if (w1 && gd) {
            phi_plane(k0);
            node_w(k0, wSA, wXA, wYA, wSB, wXB, wYB);
        }
        if (!__syncthreads_and(w1)) {
            give_up(w1 ? k0 + 1 : w0 ? k0 : k0 - 1, k0 + 1);
            return false;
        }
    }
    // One barrier per plane.  Plane k reads the potentials of plane k at the
    // thread's node and at its +x and +y neighbours, published by the
    // barrier that ended the previous plane, and those of plane k + 1 at its
    // own node only, which it has just formed; so it can be computed as soon
    // as the thread's own wait for plane k + 1 has completed.  The barrier at
    // the end publishes plane k + 1's potentials, frees the ring slots of
    // plane k - 1 for the copies the next plane issues, and makes a wait
    // that gave up end the block as a whole.
    for (int k = k0; k < k1; k++) {
        const int last = k + 2 <= k1 ? k + 2 : k + 1;
        if (k + 2 <= k1) issue(k + 2);
        const bool ok = wait(k + 1);
        float nSA = 0.f, nXA = 0.f, nYA = 0.f, nSB = 0.f, nXB = 0.f, nYB = 0.f;  // plane k + 1
        if (ok) {
            if (gd) {
                phi_plane(k + 1);
                node_w(k + 1, nSA, nXA, nYA, nSB, nXB, nYB);
            }
            const PlaneGeo<float> pg = plane_geo(g, k);
            const bool kin = k >= 1 && k <= g.nz - 1;
            if (liveA)
                node_edges(cgA, pg, k, kin, hfA, hsA, hnA, wSA, wXA, wYA, nSA, colA + pxy * k, axA, ayA, azA);
            if (liveB)
                node_edges(cgB, pg, k, kin, hfA + dF, hsA + dS, hnA + dN, wSB, wXB, wYB, nSB, colB + pxy * k, axB,
                           ayB, azB);
            if (k + 1 < k1) load_aux(k + 1);
        }
        wSA = nSA;
        wXA = nXA;
        wYA = nYA;
        wSB = nSB;
        wXB = nXB;
        wYB = nYB;
        if (!__syncthreads_and(ok)) {
            give_up(ok ? k + 2 : k + 1, last);
            return false;
        }
    }
    return true;
}

// The operator launches of one iteration, by stage:
//   diagonal preconditioner
//     0  vh = D^-1 A u,            (rt, v) = sum conj(y) vh  -> alpha
//     1  th = D^-1 A sh,           (t, s)_W, (t, t)_W, (s, s)_W -> omega, ||r||
//   polynomial preconditioner M^-1 = c D^-1 (2 I - c A D^-1)
//     2  w1 = D^-1 A u
//     3  vh = c (2 w1 - c D^-1 A w1),  (rt, v)              -> alpha
//     4  w2 = D^-1 A sh
//     5  th = c (2 w2 - c D^-1 A w2),  (t, s)_W ... with s = sh read from memory
//     6  p = D^-1 A yhat at the end of a cycle (yhat in x0; see kh_conv)
// (D^-1 A (M^-1 p) = c (2 D^-1 A u - c D^-1 A w1) since u = D^-1 p.)  Stages
// 0 and 2 stage u and, after a restart, write the new shadow y = W rh
// (u = rh on that iteration).  For column tile bx and plane chunk bz of gz of
// right-hand side r; the stage and the grad-div term are compile-time.
template <int stage, bool gd>
__device__ __forceinline__ void hat_vt(const TmaParams &tp, const KArgs<float> &a, int r, int bx, int bz, int gz)
{
    constexpr bool kv = stage == 0 || stage == 3;  // (rt, v) and alpha
    constexpr bool kt = stage == 1 || stage == 5;  // omega and ||r||
    constexpr bool poly = stage == 3 || stage == 5;
    constexpr bool dots = kv || kt;
    constexpr bool conv = stage == 6;  // after the cycle, whatever the status
    BicgState &st = a.st[r];
    if ((!conv && st.status != KS_RUNNING) || !a.ost[r].active) return;
    if (!conv && a.sweeps && threadIdx.x == 0 && bx == 0 && bz == 0) atomicAdd(a.sweeps, 1ULL);
    int i0, j0, k0, k1;
    tma_tile_at(a.cmap, bx, i0, j0);
    tma_range_at(a.g.nz, bz, gz, k0, k1);
    const size_t off = (size_t)r * a.stride;
    float2 *out = (stage == 0 || stage == 3 ? a.v : stage == 2 || stage == 6 ? a.p : stage == 4 ? a.s : a.t) + off;
    float2 *Yr = a.rt + off;
    // after a restart (first iteration, pad set) the shadow becomes the
    // current residual: y = W rh, rh being the staged u of this launch
    const bool reset = (stage == 0 || stage == 2) && st.first && st.pad;
    const float2 *aux = nullptr;
    if (kv && !reset) aux = Yr;
    if (stage == 5) aux = a.sh + off;
    const float c2 = 2.f * a.pc, cc = a.pc * a.pc;
    // inner products summed per edge in FP64 (per-plane FP32 partial sums
    // changed the Krylov rounding enough to send more right-hand sides to
    // the FP64 fallback)
    double u[4] = {0.0, 0.0, 0.0, 0.0};
    TmaSmem &sm = tma_smem();
    const bool ok = hat_march<gd>(
        sm, tp, a.g, a.pl, r, aux, (float)(a.dsgn * a.ost[r].omega * kMu0), i0, j0, k0, k1, a.err, a.wait_limit,
        // y and W are zero at edges that are not interior, and so are x
        // and xa there (u, sh, w1, w2 and the shadow vanish off the
        // interior): those edges add nothing and need no test
        [&](int e, float2 y, float2 x, float W, float2 xa) {
            if (reset) Yr[e] = make_float2(W * x.x, W * x.y);
            if (poly) y = make_float2(c2 * x.x - cc * y.x, c2 * x.y - cc * y.y);  // c (2 x - c D^-1 A x)
            if (kv) {
                const float2 z = reset ? make_float2(W * x.x, W * x.y) : xa;
                u[0] += (double)z.x * y.x + (double)z.y * y.y;  // conj(y) vh
                u[1] += (double)z.x * y.y - (double)z.y * y.x;
            } else if (kt) {
                const float2 sv = stage == 5 ? xa : x;
                const double w = W;
                u[0] += w * ((double)y.x * sv.x + (double)y.y * sv.y);  // conj(t) s
                u[1] += w * ((double)y.x * sv.y - (double)y.y * sv.x);
                u[2] += w * ((double)y.x * y.x + (double)y.y * y.y);
                u[3] += w * ((double)sv.x * sv.x + (double)sv.y * sv.y);
            }
            out[e] = y;
        });
    if (!ok || !dots) return;
    // the march has read its last staged plane: the field ring is free
    double tot[4];
    if (block_reduce_last_in<4, kHatThreads>(u, a.parts, a.cnt, r, bx + a.cmap.tiles * bz, a.cmap.tiles * gz, tot,
                                reinterpret_cast<double *>(sm.fld[0]), reinterpret_cast<int *>(sm.fld[1])) &&
        threadIdx.x == 0) {
        if (kv) {
            fin_v(st, tot);
            st.pad = 0;
        } else {
            fin_t(st, tot);
            if (st.status == KS_RUNNING) {
                const cd ts = {tot[0], tot[1]}, om = st.omega;
                const double rn2 = tot[3] - 2.0 * (om.re * ts.re + om.im * ts.im) + (om.re * om.re + om.im * om.im) * tot[2];
                st.rn2 = rn2 > 0.0 ? rn2 : 0.0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// kernels of one grid (blockIdx.y = right-hand side) and of a multi-grid
// batch (one flat block index over the right-hand sides of every grid)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) kh_u(KArgs<float> a) { hat_u(a, blockIdx.y, blockIdx.x); }
__global__ void __launch_bounds__(kThreads) kh_s(KArgs<float> a) { hat_s(a, blockIdx.y, blockIdx.x); }
__global__ void __launch_bounds__(kThreads) kh_xr(KArgs<float> a) { hat_xr(a, blockIdx.y, blockIdx.x); }
template <int stage, bool gd>
__global__ void __launch_bounds__(kHatThreads, 4) kh_vt(const __grid_constant__ TmaParams tp, KArgs<float> a)
{
    hat_vt<stage, gd>(tp, a, blockIdx.y, blockIdx.x, blockIdx.z, gridDim.z);
}

// the grids of a multi-grid batch, passed by value: each grid's arguments,
// its tensor maps (u and sh inputs) and where its blocks start in the flat
// launches
struct alignas(64) HatMulti {
    TmaParams tp[kMaxMultiGrids][4];  // inputs u, sh, w1, w2
    KArgs<float> a[kMaxMultiGrids];
    int ng;
    int nr[kMaxMultiGrids];            // right-hand sides of each grid
    int zch[kMaxMultiGrids];           // node-plane chunks of its stencil launches
    int eb0[kMaxMultiGrids + 1];       // first flat block of each grid: elementwise launches
    int sb0[kMaxMultiGrids + 1];       // first flat block of each grid: stencil launches
};
__device__ __forceinline__ int multi_grid_of(const int *b0, int ng, int b)
{
    int g = 0;
    while (g + 1 < ng && b >= b0[g + 1]) g++;
    return g;
}
template <int K> __global__ void __launch_bounds__(kThreads) kh_elem_multi(const __grid_constant__ HatMulti p)
{
    const int g = multi_grid_of(p.eb0, p.ng, blockIdx.x);
    const KArgs<float> &a = p.a[g];
    const int local = blockIdx.x - p.eb0[g];
    const int r = local / a.nblk, bx = local - r * a.nblk;
    if (K == 0) hat_u(a, r, bx);
    else if (K == 1) hat_s(a, r, bx);
    else hat_xr(a, r, bx);
}
// input map of each stage: u, sh, u, w1, sh, w2, x0
__host__ __device__ constexpr int stage_input(int stage)
{
    return stage == 0 || stage == 2 ? 0 : stage == 1 || stage == 4 ? 1 : stage == 3 ? 2 : stage == 6 ? 4 : 3;
}
template <int stage> __global__ void __launch_bounds__(kHatThreads, 4) kh_vt_multi(const __grid_constant__ HatMulti p)
{
    const int g = multi_grid_of(p.sb0, p.ng, blockIdx.x);
    const KArgs<float> &a = p.a[g];
    const int per = a.cmap.tiles * p.zch[g];
    const int local = blockIdx.x - p.sb0[g];
    const int r = local / per, rem = local - r * per;
    const int bz = rem / a.cmap.tiles, bx = rem - bz * a.cmap.tiles;
    const TmaParams &tp = p.tp[g][stage_input(stage)];
    if (a.gd) hat_vt<stage, true>(tp, a, r, bx, bz, p.zch[g]);
    else hat_vt<stage, false>(tp, a, r, bx, bz, p.zch[g]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int hat_grid(long n) { return (int)std::min<long>((n + kThreads - 1) / kThreads, 148L * 16); }

void launch_hat_cast(const KArgs<float> &a, const double2 *r64, size_t stride64, int nrhs, cudaStream_t s)
{
    counted(1);
    kh_cast<<<dim3(hat_grid(a.g.nE), nrhs), kThreads, 0, s>>>(a, r64, stride64);
}

template <int stage, bool gd> static void launch_hat_vt_t(const KArgs<float> &a, const TmaParams &tp, int nrhs,
                                                           cudaStream_t s)
{
    const size_t sm = sizeof(TmaSmem);
    const int res = tma_resident(kh_vt<stage, gd>, sm, 2 + 2 * stage + (gd ? 1 : 0), kHatThreads);
    kh_vt<stage, gd><<<dim3(a.cmap.tiles, nrhs, stage_chunks(a.g.nz, a.cmap.tiles, res)), kHatThreads, sm, s>>>(tp,
                                                                                                              a);
}
template <int stage> static void launch_hat_stage(const KArgs<float> &a, int nrhs, cudaStream_t s)
{
    counted(1);
    const TmaMaps *m = a.tma;
    TmaParams tp;
    constexpr int in = stage_input(stage);
    tp.in = in == 0 ? m->ph : in == 1 ? m->sh : in == 2 ? m->pw : in == 3 ? m->sw : m->x0;
    tp.sig = m->sig;
    tp.node = m->node;
    if (a.gd) launch_hat_vt_t<stage, true>(a, tp, nrhs, s);
    else launch_hat_vt_t<stage, false>(a, tp, nrhs, s);
}

// one iteration; the events bracket the operator launches (the two of the
// polynomial preconditioner's first and second half together)
void launch_hat_iter(const KArgs<float> &a, int nrhs, cudaStream_t s, cudaEvent_t *ev)
{
    counted(3);
    const dim3 grid(a.nblk, nrhs);
    const bool poly = a.pc > 0.f;
    kh_u<<<grid, kThreads, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[0], s);
    if (poly) {
        launch_hat_stage<2>(a, nrhs, s);
        launch_hat_stage<3>(a, nrhs, s);
    } else {
        launch_hat_stage<0>(a, nrhs, s);
    }
    if (ev) cudaEventRecord(ev[1], s);
    kh_s<<<grid, kThreads, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[2], s);
    if (poly) {
        launch_hat_stage<4>(a, nrhs, s);
        launch_hat_stage<5>(a, nrhs, s);
    } else {
        launch_hat_stage<1>(a, nrhs, s);
    }
    if (ev) cudaEventRecord(ev[3], s);
    kh_xr<<<grid, kThreads, 0, s>>>(a);
}

void launch_hat_apply(const KArgs<float> &a, int nrhs, cudaStream_t s) { launch_hat_stage<0>(a, nrhs, s); }

// x = c (2 yhat - c p) with p = D^-1 A yhat (stage 6): the cycle's iterate
// from its accumulation in the D^-1-scaled space, for every active right-hand
// side (x0 holds the best yhat after launch_bicg_finish)
__global__ void __launch_bounds__(kThreads) kh_conv(KArgs<float> a)
{
    const int r = blockIdx.y, bx = blockIdx.x;
    if (!a.ost[r].active) return;
    const size_t off = (size_t)r * a.stride / 2;
    float4 *X = reinterpret_cast<float4 *>(a.x0) + off;
    const float4 *P = reinterpret_cast<const float4 *>(a.p) + off;
    const float c2 = 2.f * a.pc, cc = a.pc * a.pc;
    HAT_PAIRS(a, bx)
    {
        const float4 x = X[q], w = P[q];
        X[q] = make_float4(c2 * x.x - cc * w.x, c2 * x.y - cc * w.y, c2 * x.z - cc * w.z, c2 * x.w - cc * w.w);
    }
}
void launch_hat_conv(const KArgs<float> &a, int nrhs, cudaStream_t s)
{
    if (!(a.pc > 0.f)) return;
    launch_hat_stage<6>(a, nrhs, s);
    counted(1);
    kh_conv<<<dim3(a.nblk, nrhs), kThreads, 0, s>>>(a);
}

// the shared-memory attribute and occupancy of every operator kernel, set
// before a capture (tma_resident calls the runtime only the first time)
template <int stage> static void hat_prime_stage()
{
    const size_t sm = sizeof(TmaSmem);
    tma_resident(kh_vt<stage, false>, sm, 2 + 2 * stage, kHatThreads);
    tma_resident(kh_vt<stage, true>, sm, 3 + 2 * stage, kHatThreads);
    if (stage < 6) tma_resident(kh_vt_multi<(stage < 6 ? stage : 0)>, sm, 16 + stage, kHatThreads);
}
static void hat_prime()
{
    hat_prime_stage<0>();
    hat_prime_stage<1>();
    hat_prime_stage<2>();
    hat_prime_stage<3>();
    hat_prime_stage<4>();
    hat_prime_stage<5>();
    hat_prime_stage<6>();
}

void HatGraph::reset()
{
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
}
HatGraph::~HatGraph()
{
    reset();
    if (cap) cudaStreamDestroy(cap);
}

cudaError_t hat_graph_run(HatGraph &hg, const KArgs<float> *args, const int *nrhs, const int *zch, int ng, int maxit,
                          cudaStream_t s)
{
    const int n = ng > 0 ? ng : 1;
    if (ng > kMaxMultiGrids) return cudaErrorInvalidValue;
    // the key: the launch arguments, the tensor maps they point to, the
    // right-hand-side and chunk counts and the cycle length
    std::vector<unsigned char> k;
    auto put = [&](const void *p, size_t b) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        k.insert(k.end(), c, c + b);
    };
    for (int g = 0; g < n; g++) {
        put(&args[g], sizeof(KArgs<float>));
        if (args[g].tma) put(args[g].tma, sizeof(TmaMaps));
        put(&nrhs[g], sizeof(int));
        const int z = zch ? zch[g] : 0;
        put(&z, sizeof z);
    }
    put(&ng, sizeof ng);
    put(&maxit, sizeof maxit);
    if (!hg.exec || k != hg.key) {
        hg.reset();
        if (!hg.cap) {
            cudaError_t e = cudaStreamCreateWithFlags(&hg.cap, cudaStreamNonBlocking);
            if (e != cudaSuccess) return e;
        }
        hat_prime();
        const long long c0 = g_launch_count.load();
        cudaError_t e = cudaStreamBeginCapture(hg.cap, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        for (int it = 0; it < maxit; it++) {
            if (ng > 0) launch_hat_iter_multi(args, nrhs, zch, ng, hg.cap);
            else launch_hat_iter(args[0], nrhs[0], hg.cap);
        }
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(hg.cap, &graph);
        hg.launches = g_launch_count.load() - c0;
        g_launch_count.fetch_sub(hg.launches);
        if (e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            return e;
        }
        e = cudaGraphInstantiate(&hg.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            hg.exec = nullptr;
            return e;
        }
        hg.key.swap(k);
    }
    g_launch_count.fetch_add(hg.launches);
    return cudaGraphLaunch(hg.exec, s);
}

// one iteration of the fused FP32 BiCGStab over the grids of a multi-grid
// batch: five launches in all, each over the right-hand sides of every grid
// (zch[g]: node-plane chunks of grid g's stencil blocks, 0 for the
// occupancy-based choice)
// as launch_hat_iter, for the grids of a multi-grid batch; ev (4 events, may
// be null) brackets the operator launches
int launch_hat_iter_multi(const KArgs<float> *args, const int *nrhs, const int *zch, int ng, cudaStream_t s,
                          cudaEvent_t *ev)
{
    if (ng < 1 || ng > kMaxMultiGrids) return 1;
    static_assert(sizeof(HatMulti) <= 32000, "multi-grid parameters exceed the kernel parameter space");
    HatMulti p;
    std::memset(&p, 0, sizeof p);
    p.ng = ng;
    const size_t smb = sizeof(TmaSmem);
    const int res = tma_resident(kh_vt_multi<0>, smb, 16, kHatThreads);
    tma_resident(kh_vt_multi<1>, smb, 17, kHatThreads);
    tma_resident(kh_vt_multi<2>, smb, 18, kHatThreads);
    tma_resident(kh_vt_multi<3>, smb, 19, kHatThreads);
    tma_resident(kh_vt_multi<4>, smb, 20, kHatThreads);
    tma_resident(kh_vt_multi<5>, smb, 21, kHatThreads);
    p.eb0[0] = p.sb0[0] = 0;
    for (int g = 0; g < ng; g++) {
        p.a[g] = args[g];
        p.nr[g] = nrhs[g];
        p.tp[g][0].in = args[g].tma->ph;
        p.tp[g][1].in = args[g].tma->sh;
        p.tp[g][2].in = args[g].tma->pw;
        p.tp[g][3].in = args[g].tma->sw;
        for (int w = 0; w < 4; w++) {
            p.tp[g][w].sig = args[g].tma->sig;
            p.tp[g][w].node = args[g].tma->node;
        }
        p.zch[g] = zch && zch[g] > 0 ? zch[g] : stage_chunks(args[g].g.nz, args[g].cmap.tiles, res);
        p.eb0[g + 1] = p.eb0[g] + nrhs[g] * args[g].nblk;
        p.sb0[g + 1] = p.sb0[g] + nrhs[g] * args[g].cmap.tiles * p.zch[g];
    }
    // the polynomial preconditioner is used when the first grid's handle
    // has it (every handle of a batch shares the control)
    const bool poly = args[0].pc > 0.f;
    counted(poly ? 7 : 5);
    const size_t sm = sizeof(TmaSmem);
    kh_elem_multi<0><<<p.eb0[ng], kThreads, 0, s>>>(p);
    if (ev) cudaEventRecord(ev[0], s);
    if (poly) {
        kh_vt_multi<2><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
        kh_vt_multi<3><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
    } else {
        kh_vt_multi<0><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
    }
    if (ev) cudaEventRecord(ev[1], s);
    kh_elem_multi<1><<<p.eb0[ng], kThreads, 0, s>>>(p);
    if (ev) cudaEventRecord(ev[2], s);
    if (poly) {
        kh_vt_multi<4><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
        kh_vt_multi<5><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
    } else {
        kh_vt_multi<1><<<p.sb0[ng], kHatThreads, sm, s>>>(p);
    }
    if (ev) cudaEventRecord(ev[3], s);
    kh_elem_multi<2><<<p.eb0[ng], kThreads, 0, s>>>(p);
    return 0;
}

}  // namespace mt3d

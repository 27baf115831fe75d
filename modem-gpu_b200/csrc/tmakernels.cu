// tmakernels.cu -- the FP32 BiCGStab stencil kernels with their planes staged
// by the Tensor Memory Accelerator, on the padded layout (PadLayout).
//
// A block owns 32 x 8 node columns of one right-hand side and marches a chunk
// of node planes, as the cp.async kernels of stagekernels.cu do.  Per plane
// one thread issues three tensor copies into a four-slot ring in shared
// memory (separate rings for fields, sigma and node weights), completed on an
// mbarrier per plane slot:
//   - Ex, Ey, Ez over i0-2 .. i0+33, j0-1 .. j0+8 (one copy for the three
//     components: box 72 floats x 10 rows x 3 components),
//   - sigma over i0-4 .. i0+35, j0-1 .. j0+8 (box 40 x 10 x 3),
//   - the signed node weights over i0 .. i0+35, j0 .. j0+8 (box 36 x 9).
// The x coordinates are the tile origin rounded down to a 16-byte boundary,
// as tensor copies require; the halo columns the stencil does not use are
// read and ignored.  Coordinates outside a tensor read zeros.  The copies of
// plane k + 2 are issued before plane k is computed, so the threads only
// wait for data and no longer spend instructions on moving it.
//
// Every wait on an mbarrier is bounded: a thread polls at most `limit` times
// (KArgs::wait_limit).  The block then decides together, in the barrier that
// follows every wait (__syncthreads_and), so either every thread goes on or
// every thread leaves: on a timeout the issuing thread sets *err and waits
// (bounded by kWaitLimit) for its copies still in flight, so none lands after
// the block has exited, and the host reports MT3D_DEVICE_TIMEOUT.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "finalize.cuh"
#include "tma.cuh"

namespace mt3d {

extern std::atomic<long long> g_launch_count;
static inline void counted(int n) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

// March planes [k0, k1) of tile (i0, j0), right-hand side r (tensor
// coordinate 3 r), calling f(comp, e, interior, Ax, x_e, aux_e) for every
// existing edge of the thread's node column; e indexes the padded layout.
// Returns false (all threads of the block alike) when a wait gave up.
template <typename F>
__device__ __forceinline__ bool tma_march(TmaSmem &sm, const TmaParams &tp, const Geo<float> &g, PadLayout pl,
                                          int r, const float2 *__restrict__ aux, bool gd, float wmu, int i0, int j0,
                                          int k0, int k1, int *err, int limit, F &&f)
{
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    const int i = i0 + tx, j = j0 + ty;
    const bool live = i <= g.nx && j <= g.ny;
    const ColGeo<float> cg = col_geo(g, min(i, g.nx), min(j, g.ny));
    const int hf = (ty + 1) * kFW + tx + 2;  // own column in a field plane of the tile
    const int hs = (ty + 1) * kSW + tx + 4;  // own column in a sigma plane
    const int hn = ty * kPhX + tx;           // own node in a potential plane
    const int cf = kFR * kFW, cs = kFR * kSW;
    const int pxy = pl.Px * pl.Py, pc = pl.Pz * pxy;
    const int col = min(i, pl.Px - 1) + pl.Px * min(j, pl.Py - 1);  // (i, j) in a plane of the padded layout
    const bool issuer = threadIdx.x == 0;
    const unsigned tx_bytes = kFBytes + kSBytes;
    // halo potentials: threads 0..31 the row j0 + 8, the next 9 the column i0 + 32
    const bool hasH = threadIdx.x < kTX + kTY + 1;
    const int hni = threadIdx.x < kTX ? threadIdx.x : kTX;
    const int hnj = threadIdx.x < kTX ? kTY : threadIdx.x - kTX;
    const int hi = i0 + hni, hj = j0 + hnj;
    const float hdX = (hasH && hi <= g.nx) ? g.delX[hi] : 0.f, hdY = (hasH && hj <= g.ny) ? g.delY[hj] : 0.f;

    // tensor-copy destinations must be 128-byte aligned: refuse otherwise
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
    // the copies of plane p complete on the mbarrier of its field slot; the
    // node weights of plane k0 - 1 are not needed (no potential is formed
    // there) and would share a slot with plane k0 + 1
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
    // this thread's bounded wait for the copies of plane p
    auto wait = [&](int p) -> bool {
        const int s = p & 3;
        if (mbar_wait(smem_addr(&sm.mbar[s]), (phase >> s) & 1u, limit)) {
            phase ^= 1u << s;
            return true;
        }
        return false;
    };
    // the block gave up: the issuer records it and waits (bounded) for its
    // copies of planes first .. last, which no thread has seen complete, so
    // that none lands in shared memory after the block has exited
    auto give_up = [&](int first, int last) {
        if (!issuer) return;
        atomicExch(err, 1);
        for (int q = first; q <= last; q++)
            if (mbar_wait(smem_addr(&sm.mbar[q & 3]), (phase >> (q & 3)) & 1u, kWaitLimit)) phase ^= 1u << (q & 3);
    };
    auto phi_plane = [&](int p) {
        const float dZ = (p >= 0 && p <= g.nz) ? g.delZ[p] : 0.f;
        sm.phi[p & 1][hn] = tma_phi_node(sm, g, i, j, p, tx, ty, cg.delXi, cg.delYj, dZ);
        if (hasH) sm.phi[p & 1][hnj * kPhX + hni] = tma_phi_node(sm, g, hi, hj, p, hni, hnj, hdX, hdY, dZ);
    };
    const float2 zero = make_float2(0.f, 0.f);
    float2 ax = zero, ay = zero, az = zero;
    auto load_aux = [&](int k) {
        if (!aux || !live || k > g.nz) return;
        const int b = col + pxy * k;
        if (cg.hasX) ax = aux[b];
        if (cg.hasY) ay = aux[pc + b];
        if (k < g.nz) az = aux[2 * pc + b];
    };

    load_aux(k0);
    issue(k0 - 1);
    issue(k0);
    issue(k0 + 1);
    {
        const bool w0 = wait(k0 - 1), w1 = w0 && wait(k0);
        if (w1 && gd) phi_plane(k0);
        // plane k0 + 2 goes into the sigma slot of plane k0 - 1 and the node
        // slot of plane k0, which the potentials of plane k0 have just read
        if (!__syncthreads_and(w1)) {
            give_up(w1 ? k0 + 1 : w0 ? k0 : k0 - 1, k0 + 1);
            return false;
        }
    }
    for (int k = k0; k < k1; k++) {
        const int last = k + 2 <= k1 ? k + 2 : k + 1;
        if (k + 2 <= k1) issue(k + 2);
        const bool ok = wait(k + 1);
        if (ok && gd) phi_plane(k + 1);
        if (!__syncthreads_and(ok)) {
            give_up(ok ? k + 2 : k + 1, last);
            return false;
        }
        if (live) {
            const float2 *Fm = reinterpret_cast<const float2 *>(sm.fld[(k - 1) & 3]);
            const float2 *F0 = reinterpret_cast<const float2 *>(sm.fld[k & 3]);
            const float2 *Fp = reinterpret_cast<const float2 *>(sm.fld[(k + 1) & 3]);
            const float *S0 = reinterpret_cast<const float *>(sm.sig[k % 3]);
            const float2 *Xm = Fm, *X0 = F0, *Xp = Fp;
            const float2 *Ym = Fm + cf, *Y0 = F0 + cf, *Yp = Fp + cf;
            const float2 *Zm = Fm + 2 * cf, *Z0 = F0 + 2 * cf;
            const float2 *P0 = sm.phi[k & 1], *P1 = sm.phi[(k + 1) & 1];
            const PlaneGeo<float> pg = plane_geo(g, k);
            const bool kin = k >= 1 && k <= g.nz - 1;
            const int h = hf;
            const int eb = col + pxy * k;
            // ---- Ex(i, j, k)
            if (cg.hasX) {
                const float2 X1 = X0[h];
                const float dt = wmu * S0[hs] * (cg.dxi * (cg.delYj * pg.delZk));
                float2 out = zero;
                const bool in = cg.intX && kin;
                if (in) {
                    const float2 yy = csub(cadd(csub(Y0[h + 1], Y0[h]), Y0[h - kFW]), Y0[h + 1 - kFW]);
                    const float2 zz = csub(cadd(csub(Z0[h + 1], Z0[h]), Zm[h]), Zm[h + 1]);
                    const float2 fyp = cscale(csub(X0[h + kFW], X1), cg.rdyj);
                    const float2 fym = cscale(csub(X1, X0[h - kFW]), cg.rdyjm1);
                    const float2 fzp = cscale(csub(Xp[h], X1), pg.rdzk);
                    const float2 fzm = cscale(csub(X1, Xm[h]), pg.rdzkm1);
                    out = cadd(cscale(yy, pg.delZk), cscale(zz, cg.delYj));
                    out = csub(out, cscale(csub(fyp, fym), cg.dxi * pg.delZk));
                    out = csub(out, cscale(csub(fzp, fzm), cg.dxi * cg.delYj));
                    out.x -= dt * X1.y;
                    out.y += dt * X1.x;
                    if (gd) out = cadd(out, cscale(csub(P0[hn + 1], P0[hn]), cg.delYj * pg.delZk));
                }
                f(0, eb, in, out, X1, ax);
            }
            // ---- Ey(i, j, k)
            if (cg.hasY) {
                const float2 Y1 = Y0[h];
                const float dt = wmu * S0[cs + hs] * (cg.dyj * (cg.delXi * pg.delZk));
                float2 out = zero;
                const bool in = cg.intY && kin;
                if (in) {
                    const float2 zz = csub(cadd(csub(Z0[h + kFW], Z0[h]), Zm[h]), Zm[h + kFW]);
                    const float2 xx = csub(cadd(csub(X0[h + kFW], X0[h]), X0[h - 1]), X0[h - 1 + kFW]);
                    const float2 fzp = cscale(csub(Yp[h], Y1), pg.rdzk);
                    const float2 fzm = cscale(csub(Y1, Ym[h]), pg.rdzkm1);
                    const float2 fxp = cscale(csub(Y0[h + 1], Y1), cg.rdxi);
                    const float2 fxm = cscale(csub(Y1, Y0[h - 1]), cg.rdxim1);
                    out = cadd(cscale(zz, cg.delXi), cscale(xx, pg.delZk));
                    out = csub(out, cscale(csub(fzp, fzm), cg.dyj * cg.delXi));
                    out = csub(out, cscale(csub(fxp, fxm), cg.dyj * pg.delZk));
                    out.x -= dt * Y1.y;
                    out.y += dt * Y1.x;
                    if (gd) out = cadd(out, cscale(csub(P0[hn + kPhX], P0[hn]), cg.delXi * pg.delZk));
                }
                f(1, pc + eb, in, out, Y1, ay);
            }
            // ---- Ez(i, j, k)
            if (k < g.nz) {
                const float2 Z1 = Z0[h];
                const float dt = wmu * S0[2 * cs + hs] * (pg.dzk * (cg.delXi * cg.delYj));
                float2 out = zero;
                const bool in = cg.intZ;
                if (in) {
                    const float2 xx = csub(cadd(csub(Xp[h], X0[h]), X0[h - 1]), Xp[h - 1]);
                    const float2 yy = csub(cadd(csub(Yp[h], Y0[h]), Y0[h - kFW]), Yp[h - kFW]);
                    const float2 fxp = cscale(csub(Z0[h + 1], Z1), cg.rdxi);
                    const float2 fxm = cscale(csub(Z1, Z0[h - 1]), cg.rdxim1);
                    const float2 fyp = cscale(csub(Z0[h + kFW], Z1), cg.rdyj);
                    const float2 fym = cscale(csub(Z1, Z0[h - kFW]), cg.rdyjm1);
                    out = cadd(cscale(xx, cg.delYj), cscale(yy, cg.delXi));
                    out = csub(out, cscale(csub(fxp, fxm), pg.dzk * cg.delYj));
                    out = csub(out, cscale(csub(fyp, fym), pg.dzk * cg.delXi));
                    out.x -= dt * Z1.y;
                    out.y += dt * Z1.x;
                    if (gd) out = cadd(out, cscale(csub(P1[hn], P0[hn]), cg.delXi * cg.delYj));
                }
                f(2, 2 * pc + eb, in, out, Z1, az);
            }
            if (k + 1 < k1) load_aux(k + 1);
        }
        __syncthreads();
    }
    return true;
}

// start of a call: r = b - A x0, rt = r; |b|^2, |r|^2
__global__ void __launch_bounds__(kThreads, 4) kct_init(const __grid_constant__ TmaParams tp, KArgs<float> a)
{
    const int r = blockIdx.y;
    if (!a.ost[r].active) return;
    BicgState &st = a.st[r];
    int i0, j0, k0, k1;
    tma_tile(a.cmap, i0, j0);
    tma_range(a.g.nz, k0, k1);
    const size_t off = (size_t)r * a.stride;
    const float2 *b = a.b + off;
    float2 *R = a.r + off, *RT = a.rt + off;
    double u[2] = {0.0, 0.0};
    const bool ok = tma_march(tma_smem(), tp, a.g, a.pl, r, b, a.gd != 0, (float)(a.dsgn * a.ost[r].omega * kMu0),
                              i0, j0, k0, k1, a.err, a.wait_limit, [&](int, int e, bool in, float2 ax, float2, float2 bb) {
                                  float2 res = make_float2(0.f, 0.f);
                                  if (in) {
                                      res = csub(bb, ax);
                                      u[0] += (double)bb.x * bb.x + (double)bb.y * bb.y;
                                      u[1] += (double)res.x * res.x + (double)res.y * res.y;
                                  }
                                  R[e] = res;
                                  RT[e] = res;
                              });
    if (!ok) return;
    double tot[2];
    if (block_reduce_last<2>(u, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0)
        fin_init(st, tot, a.rerr + (size_t)r * a.rerr_stride, a.maxit, a.inner ? a.ost[r].tol_inner : a.ost[r].tol);
}

// v = A ph ; rtv = rt . v ; alpha   (which = 0)
// t = A sh ; ts = t . s, tt = t . t ; omega   (which = 1)
__global__ void __launch_bounds__(kThreads, 4) kct_vt(const __grid_constant__ TmaParams tp, KArgs<float> a, int which)
{
    const int r = blockIdx.y;
    BicgState &st = a.st[r];
    if (st.status != KS_RUNNING || !a.ost[r].active) return;
    if (a.sweeps && threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.z == 0) atomicAdd(a.sweeps, 1ULL);
    int i0, j0, k0, k1;
    tma_tile(a.cmap, i0, j0);
    tma_range(a.g.nz, k0, k1);
    const size_t off = (size_t)r * a.stride;
    const float2 *w = (which ? a.s : a.rt) + off;
    float2 *out = (which ? a.t : a.v) + off;
    double u[3] = {0.0, 0.0, 0.0};
    const bool ok = tma_march(tma_smem(), tp, a.g, a.pl, r, w, a.gd != 0, (float)(a.dsgn * a.ost[r].omega * kMu0),
                              i0, j0, k0, k1, a.err, a.wait_limit, [&](int, int e, bool inn, float2 y, float2, float2 q) {
                                  if (inn) {
                                      if (which == 0) {
                                          u[0] += (double)q.x * y.x + (double)q.y * y.y;  // conj(rt) v
                                          u[1] += (double)q.x * y.y - (double)q.y * y.x;
                                      } else {
                                          u[0] += (double)y.x * q.x + (double)y.y * q.y;  // conj(t) s
                                          u[1] += (double)y.x * q.y - (double)y.y * q.x;
                                          u[2] += (double)y.x * y.x + (double)y.y * y.y;
                                      }
                                  }
                                  out[e] = y;
                              });
    if (!ok) return;
    double tot[3];
    if (block_reduce_last<3>(u, a.parts, a.cnt, r, blockIdx.x + gridDim.x * blockIdx.z, gridDim.x * gridDim.z, tot) &&
        threadIdx.x == 0) {
        if (which == 0) fin_v(st, tot);
        else fin_t(st, tot);
    }
}

// ---------------------------------------------------------------------------
// host side: tensor maps and launches
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

static int encode(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                  const cuuint32_t *box)
{
    auto fn = encode_fn();
    if (!fn) return 1;
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<void *>(base), dims, strides, box, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : 1;
}

TmaMaps *tma_maps_new()
{
    TmaMaps *m = new TmaMaps;
    std::memset(m, 0, sizeof *m);
    return m;
}
void tma_maps_free(TmaMaps *m) { delete m; }

int tma_maps_build(TmaMaps *m, const float2 *x0, const float2 *ph, const float2 *sh, const float2 *pw,
                   const float2 *sw, const float *sig, const float *gdn, PadLayout pl, int nrhs)
{
    m->ok = 0;
    const cuuint64_t Px = pl.Px, Py = pl.Py, Pz = pl.Pz;
    // vectors: floats [nrhs * 3][Pz][Py][2 Px]
    const cuuint64_t vd[4] = {2 * Px, Py, Pz, 3 * (cuuint64_t)nrhs};
    const cuuint64_t vs[3] = {2 * Px * 4, 2 * Px * Py * 4, 2 * Px * Py * Pz * 4};
    const cuuint32_t vb[4] = {2 * kFW, kFR, 1, 3};
    // sigma: floats [3][Pz][Py][Px]; node weights: floats [Pz][Py][Px]
    const cuuint64_t sd[4] = {Px, Py, Pz, 3};
    const cuuint64_t ss[3] = {Px * 4, Px * Py * 4, Px * Py * Pz * 4};
    const cuuint32_t sb[4] = {kSW, kFR, 1, 3};
    const cuuint64_t nd[3] = {Px, Py, Pz};
    const cuuint64_t ns[2] = {Px * 4, Px * Py * 4};
    const cuuint32_t nb[3] = {kNW, kNR, 1};
    if (encode(&m->x0, x0, 4, vd, vs, vb) || encode(&m->ph, ph, 4, vd, vs, vb) || encode(&m->sh, sh, 4, vd, vs, vb) ||
        encode(&m->pw, pw, 4, vd, vs, vb) || encode(&m->sw, sw, 4, vd, vs, vb) ||
        encode(&m->sig, sig, 4, sd, ss, sb) || encode(&m->node, gdn ? gdn : sig, 3, nd, ns, nb))
        return 1;
    m->ok = 1;
    return 0;
}

void launch_tma_init(const KArgs<float> &a, const TmaMaps *m, int nrhs, cudaStream_t s)
{
    counted(1);
    TmaParams tp;
    tp.in = m->x0;
    tp.sig = m->sig;
    tp.node = m->node;
    const size_t sm = sizeof(TmaSmem);
    const int res = tma_resident(kct_init, sm, 0);
    kct_init<<<dim3(a.cmap.tiles, nrhs, stage_chunks(a.g.nz, a.cmap.tiles, res)), kThreads, sm, s>>>(tp, a);
}
void launch_tma_vt(const KArgs<float> &a, const TmaMaps *m, int which, int nrhs, cudaStream_t s)
{
    counted(1);
    TmaParams tp;
    tp.in = which ? m->sh : m->ph;
    tp.sig = m->sig;
    tp.node = m->node;
    const size_t sm = sizeof(TmaSmem);
    const int res = tma_resident(kct_vt, sm, 1);
    kct_vt<<<dim3(a.cmap.tiles, nrhs, stage_chunks(a.g.nz, a.cmap.tiles, res)), kThreads, sm, s>>>(tp, a, which);
}

}  // namespace mt3d

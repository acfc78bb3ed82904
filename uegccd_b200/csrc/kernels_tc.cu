// kernels_tc.cu -- 5th-generation tensor-core (tcgen05 + TMEM) kernels of the
// mixed-precision path.
//
// Particle-particle ladder (CCD.f90:660-681) in the spin-adapted block form
//   G_K^T[a][p] = sum_c v(a - c) t_K[p][c]
// as one MMA per block tile: M = 128 virtuals a, N = o_K rows p (padded to 16, 32
// or 64), K = the block's virtuals c in chunks of 32.  Operands are FP16 with FP32
// accumulation in tensor memory.
//
// Mixed precision as defect correction: the kernel multiplies d = t - t_ref (not t),
// each row p of d scaled by its max |d| before rounding to FP16, and adds the FP64
// ladder of t_ref computed when t_ref was last refreshed.  The ladder is linear in t,
// so the sum is exact up to the FP16 rounding of d and W, an error that shrinks with
// |t - t_ref|; FP64 sweeps at the end remove what is left.
//
// Both FP16 operands are written to global memory already in the MMA's canonical
// shared-memory layout, one 32-wide K chunk after another: the Coulomb slabs once per
// batch (they depend only on the |q|^2 tables; k_w16_build) and the scaled d tiles once
// per iteration (k_delta16).  Each chunk of each operand is then one contiguous range, and
// the MMA kernel streams it into shared memory with one bulk copy of the TMA engine
// (cp.async.bulk, completing on the stage's mbarrier).
//
// Shared-memory operands use the canonical K-major layout without swizzle: 8 x 8
// element core matrices (8 rows of 16 bytes), core matrices adjacent in K 128 bytes
// apart (LBO) and 8-row groups 512 bytes apart (SBO) for a 32-wide K chunk.
// One thread issues the MMAs; tcgen05.commit arrives on an mbarrier per stage.
// Every mbarrier wait is bounded: on expiry the kernel records an error code, still
// frees its tensor memory and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "uegccd_internal.h"

namespace uegccd {

namespace {

constexpr int kTcM = 128;        // MMA M (virtuals per CTA)
constexpr int kTcK = 32;         // K chunk staged per pipeline stage
constexpr int kStages = 3;       // shared-memory stages: two chunk copies in flight beside the MMA
constexpr long long kWaitLimit = 1LL << 26;  // mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: start address, LBO, SBO (all >> 4), version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor, kind::f16: D = F32, A = B = F16, both K-major.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N)
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false when the limit expired
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (long long k = 0; k < kWaitLimit; k++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ int q2_of(int4 x, int4 y)
{
    int d0 = x.x - y.x, d1 = x.y - y.y, d2 = x.z - y.z;
    return d0 * d0 + d1 * d1 + d2 * d2;
}

// offset (in halves) of element (row, k) in a canonical K-major no-swizzle tile
// with 32-wide K: core matrices 8 rows x 8 halves, LBO = 64 halves (128 B),
// SBO = 256 halves (512 B)
__device__ __forceinline__ int cm_off(int row, int k) { return (row & 7) * 8 + (row >> 3) * 256 + (k & 7) + (k >> 3) * 64; }

// The bulk-copy (TMA) engine: one contiguous global range into this CTA's shared memory,
// completing `bytes` of the transaction count of an mbarrier.  Addresses 16-byte aligned,
// sizes multiples of 16; this GPU's own memory only, each CTA fetching its own copy.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

}  // namespace

// FP16 Coulomb slab of (block, 128 virtuals a0..): chunk ch holds A[m][k] = v(n_a - n_c),
// a = a0 + m, c = 32 ch + k, zero outside the block, in the canonical layout.
__global__ void __launch_bounds__(128) k_w16_build(const WSlabDev *__restrict__ slabs,
                                                  const BlockDev *__restrict__ blocks,
                                                  const SolveDev *__restrict__ solves,
                                                  const int16_t *__restrict__ vir, const int4 *__restrict__ nv4,
                                                  const double *__restrict__ vtab, __half *__restrict__ w16)
{
    __shared__ int4 na[kTcM];
    const WSlabDev S = slabs[blockIdx.x];
    const BlockDev B = blocks[S.blk];
    const SolveDev s = solves[B.solve];
    const int tid = threadIdx.x, v = B.v;
    for (int x = tid; x < kTcM; x += blockDim.x) {
        const int a = S.a0 + x;
        na[x] = a < v ? nv4[s.orb0 + vir[B.vir0 + a]] : make_int4(0, 0, 0, 0);
    }
    __syncthreads();
    const int nch = (v + kTcK - 1) / kTcK;
    const int k = tid & (kTcK - 1);
    for (int ch = 0; ch < nch; ch++) {
        const int c = ch * kTcK + k;
        const bool cok = c < v;
        const int4 nc = cok ? nv4[s.orb0 + vir[B.vir0 + c]] : make_int4(0, 0, 0, 0);
        __half *dst = w16 + S.woff + (int64_t)ch * kTcM * kTcK;
        for (int m = tid / kTcK; m < kTcM; m += 128 / kTcK) {
            float w = 0.f;
            if (cok && S.a0 + m < v) {
                const int q2 = q2_of(na[m], nc);
                w = q2 > s.q2max ? 0.f : (float)vtab[s.vtab0 + q2];
            }
            dst[cm_off(m, k)] = __float2half_rn(w);
        }
    }
}

// Scaled FP16 d = t - t_ref of one row tile: the scale of row p is max_c |d[p][c]| (1 if
// zero); chunk ch holds B[n][k] = d[p0 + n][32 ch + k] / scale, in the canonical layout.
__global__ void __launch_bounds__(128) k_delta16(const DTileDev *__restrict__ dt,
                                                const BlockDev *__restrict__ blocks,
                                                const double *__restrict__ t, const double *__restrict__ t_ref,
                                                __half *__restrict__ d16, float *__restrict__ dscale,
                                                const uint8_t *__restrict__ active)
{
    __shared__ float rs[64];
    const DTileDev D = dt[blockIdx.x];
    const BlockDev B = blocks[D.blk];
    if (!active[B.solve]) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, v = B.v, o = B.o, np = D.np;
    for (int pp = warp; pp < np; pp += 4) {
        const int p = D.p0 + pp;
        float m = 0.f;
        if (p < o)
            for (int c = lane; c < v; c += 32) {
                const int64_t idx = B.t0 + (int64_t)p * v + c;
                m = fmaxf(m, fabsf((float)(t[idx] - t_ref[idx])));
            }
        for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
        if (lane == 0) {
            rs[pp] = m > 0.f ? m : 1.f;
            dscale[D.soff + pp] = rs[pp];
        }
    }
    __syncthreads();
    const int nch = (v + kTcK - 1) / kTcK;
    for (int e = tid; e < nch * np * kTcK; e += blockDim.x) {
        const int ch = e / (np * kTcK), r = e - ch * (np * kTcK);
        const int pp = r / kTcK, k = r - pp * kTcK;
        const int p = D.p0 + pp, c = ch * kTcK + k;
        float x = 0.f;
        if (p < o && c < v) {
            const int64_t idx = B.t0 + (int64_t)p * v + c;
            x = (float)((t[idx] - t_ref[idx]) / (double)rs[pp]);
        }
        d16[D.doff + (int64_t)ch * np * kTcK + cm_off(pp, k)] = __float2half_rn(x);
    }
}

// One CTA per (block, 128-virtual tile).  g[...] += g_ref[...] + sum_c v(a-c) (t - t_ref)[p][c]
// for every (p, a) of the tile (g already holds the hole-hole part).
template <int NP>
__global__ void __launch_bounds__(128) k_ladder_tc(const LadderTile *__restrict__ tiles,
                                                  const TcTileDev *__restrict__ tcx,
                                                  const BlockDev *__restrict__ blocks,
                                                  const __half *__restrict__ w16, const __half *__restrict__ d16,
                                                  const float *__restrict__ dscale,
                                                  const double *__restrict__ g_ref, double *__restrict__ g,
                                                  const uint8_t *__restrict__ active, int *__restrict__ err)
{
    constexpr int NCOL = NP < 32 ? 32 : NP;  // tensor-memory columns (power of two, >= 32)
    __shared__ alignas(1024) __half As[kStages][kTcM * kTcK];
    __shared__ alignas(1024) __half Bs[kStages][NP * kTcK];
    __shared__ float rscale[NP];
    __shared__ alignas(8) uint64_t mbar[kStages];   // the MMAs of the stage's chunk are done
    __shared__ alignas(8) uint64_t full[kStages];   // the stage's chunk has landed (bulk copies)
    __shared__ uint32_t tmem_base;
    __shared__ int ok_all;

    const LadderTile T = tiles[blockIdx.x];
    const TcTileDev X = tcx[blockIdx.x];
    const BlockDev B = blocks[T.blk];
    if (!active[B.solve]) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int v = B.v, o = B.o;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int b = 0; b < kStages; b++) {
            mbar_init(&mbar[b], 1);
            mbar_init(&full[b], 1);
        }
        ok_all = 1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int pp = tid; pp < NP; pp += blockDim.x) rscale[pp] = dscale[X.soff + pp];
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem_d = tmem_base;
    const uint32_t idesc = idesc_f16(kTcM, NP);
    const int nchunks = (v + kTcK - 1) / kTcK;
    bool ok = true;
    if (tid == 0) {
        // chunk c of the Coulomb slab (8 KB) and of the d tile (NP x 64 B) into stage c % kStages:
        // one bulk copy each, both completing on full[stage]
        constexpr uint32_t kWBytes = kTcM * kTcK * 2, kDBytes = NP * kTcK * 2;
        int issued = 0;
        auto issue = [&](int c) {
            const int b = c % kStages;
            mbar_expect_tx(&full[b], kWBytes + kDBytes);
            bulk_g2s(&As[b][0], w16 + X.woff + (int64_t)c * kTcM * kTcK, kWBytes, &full[b]);
            bulk_g2s(&Bs[b][0], d16 + X.doff + (int64_t)c * NP * kTcK, kDBytes, &full[b]);
            issued = c + 1;
        };
        for (int c = 0; c < kStages && c < nchunks; c++) issue(c);
        int ch = 0;
        for (; ch < nchunks && ok; ch++) {
            const int st = ch % kStages;
            if (!mbar_wait(&full[st], (ch / kStages) & 1)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(&As[st][0]), b0 = smem_u32(&Bs[st][0]);
#pragma unroll
            for (int j = 0; j < kTcK / 16; j++)
                tc_mma(tmem_d, sdesc(a0 + j * 256, 128, 512), sdesc(b0 + j * 256, 128, 512), idesc,
                       (ch > 0 || j > 0) ? 1u : 0u);
            tc_commit(&mbar[st]);
            // the previous chunk's stage refills once its MMAs are done, while chunk ch's run
            if (ch >= 1 && ch - 1 + kStages < nchunks) {
                const int prev = ch - 1;
                if (!mbar_wait(&mbar[prev % kStages], (prev / kStages) & 1)) {
                    ok = false;
                    ch++;
                    break;
                }
                issue(prev + kStages);
            }
        }
        if (!ok) {
            // let every bulk copy still in flight land before the CTA leaves (bounded)
            for (int c = ch; c < issued; c++) mbar_wait(&full[c % kStages], (c / kStages) & 1);
            ok_all = 0;
        }
    }
    __syncthreads();
    if (!ok_all) ok = false;
    // the last chunk's MMAs (and with them all earlier ones) are done
    if (ok && !mbar_wait(&mbar[(nchunks - 1) % kStages], ((nchunks - 1) / kStages) & 1)) ok = false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // epilogue: warp w holds TMEM lanes 32w..32w+31 = rows a0 + 32w + lane
        const int a = T.a0 + warp * 32 + lane;
#pragma unroll
        for (int c16 = 0; c16 < NP / 16; c16++) {
            float acc[16];
            tc_ld16(tmem_d + ((uint32_t)(warp * 32) << 16) + c16 * 16, acc);
            if (a < v) {
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int pp = c16 * 16 + k;
                    const int p = T.p0 + pp;
                    if (p < o) {
                        const int64_t idx = B.t0 + (int64_t)p * v + a;
                        g[idx] += g_ref[idx] + (double)acc[k] * (double)rscale[pp];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(NCOL));
}

void launch_w16_build(const DevBatch &d, cudaStream_t st)
{
    if (d.nwslabs > 0)
        k_w16_build<<<d.nwslabs, 128, 0, st>>>(d.wslabs, d.blocks, d.solves, d.vir, d.nv4, d.vtab,
                                               static_cast<__half *>(d.w16));
}

void launch_ladder_tc(const DevBatch &d, const double *t_ref, const double *g_ref, int *err, cudaStream_t st)
{
    const __half *w = static_cast<const __half *>(d.w16), *dd = static_cast<const __half *>(d.d16);
    if (d.ndtiles > 0)
        k_delta16<<<d.ndtiles, 128, 0, st>>>(d.dtiles, d.blocks, d.t, t_ref, static_cast<__half *>(d.d16), d.dscale,
                                             d.active);
    if (d.ntc16)
        k_ladder_tc<16><<<d.ntc16, 128, 0, st>>>(d.tctiles, d.tcx, d.blocks, w, dd, d.dscale, g_ref, d.g, d.active,
                                                  err);
    if (d.ntc32)
        k_ladder_tc<32><<<d.ntc32, 128, 0, st>>>(d.tctiles + d.ntc16, d.tcx + d.ntc16, d.blocks, w, dd, d.dscale,
                                                  g_ref, d.g, d.active, err);
    if (d.ntc64)
        k_ladder_tc<64><<<d.ntc64, 128, 0, st>>>(d.tctiles + d.ntc16 + d.ntc32, d.tcx + d.ntc16 + d.ntc32,
                                                  d.blocks, w, dd, d.dscale, g_ref, d.g, d.active, err);
}

}  // namespace uegccd

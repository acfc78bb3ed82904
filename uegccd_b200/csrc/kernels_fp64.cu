// kernels_fp64.cu -- FP64 kernels of the spin-adapted CCD / MP2 / dRPA residual.
//
// Storage (uegccd_internal.h): t(ij,a) = T2abab(i,j,a), block-packed by
// K = n_i + n_j.  The reference's abba and aaaa channels are recovered from
// T2abba(i,j,a) = -t(ij,b) and T2aaaa(i,j,a) = t(ij,a) - t(ij,b), which the
// reference keeps exactly at the MP2 start (MP2.f90:68-70) and which its
// equations preserve when rings and crossed rings are both on.
//
// Notation below: v(x-y) = V(n_x - n_y) is the Coulomb kernel of the reference
// (BaseERI, HEG.f90:969-976), generated from an integer |q|^2 table;
// b = partner of (i,j,a), i.e. n_b = n_i + n_j - n_a.
//
// Every term is derived by substituting the two spin relations into the
// reference loops and re-indexing the sums over the partner bijection a <-> b
// of each K block; each formula cites the loop it replaces.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "kernels.h"
#include "uegccd_internal.h"

namespace uegccd {

// Plane-wave vectors packed one component per byte (x | y << 8 | z << 16, two's complement;
// DevBatch::nvp): the squared length of the difference of two orbitals' vectors is then one
// per-byte subtraction and one 4-way byte dot product.  Every |n_d| <= 63 (checked when the
// batch is made), so each component difference fits a signed byte; modular byte arithmetic
// keeps a difference of differences exact as long as the final one does.
__device__ __forceinline__ int q2p(int a, int c)
{
    const int d = __vsub4(a, c);
    return __dp4a(d, d, 0);
}

__device__ __forceinline__ int q2_of(int4 x, int4 y)
{
    int d0 = x.x - y.x, d1 = x.y - y.y, d2 = x.z - y.z;
    return d0 * d0 + d1 * d1 + d2 * d2;
}

// v(p - q) for orbitals p, q of solve s
__device__ __forceinline__ double vpq(const SolveDev &s, const int4 *__restrict__ nv4,
                                      const double *__restrict__ vtab, int p, int q)
{
    return __ldg(&vtab[s.vtab0 + q2_of(__ldg(&nv4[s.orb0 + p]), __ldg(&nv4[s.orb0 + q]))]);
}

__device__ __forceinline__ int posmap(const SolveDev &s, const int32_t *__restrict__ pos, int i, int j, int a)
{
    return __ldg(&pos[s.pos0 + ((int64_t)i * s.O + j) * s.V + (a - s.O)]);
}

// ----------------------------------------------------------------------------
// Block reductions (fixed order: deterministic for a given launch shape)
// ----------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ void block_reduce3(double &sum, double &mx1, double &mx2)
{
    __shared__ double s_sum[NT / 32], s_m1[NT / 32], s_m2[NT / 32];
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        mx1 = fmax(mx1, __shfl_down_sync(0xffffffffu, mx1, o));
        mx2 = fmax(mx2, __shfl_down_sync(0xffffffffu, mx2, o));
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { s_sum[w] = sum; s_m1[w] = mx1; s_m2[w] = mx2; }
    __syncthreads();
    if (w == 0) {
        sum = (l < NT / 32) ? s_sum[l] : 0.0;
        mx1 = (l < NT / 32) ? s_m1[l] : 0.0;
        mx2 = (l < NT / 32) ? s_m2[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            sum += __shfl_down_sync(0xffffffffu, sum, o);
            mx1 = fmax(mx1, __shfl_down_sync(0xffffffffu, mx1, o));
            mx2 = fmax(mx2, __shfl_down_sync(0xffffffffu, mx2, o));
        }
    }
}

template <int NT>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double s[NT / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) s[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < NT / 32) ? s[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;  // valid in thread 0
}

// ----------------------------------------------------------------------------
// MP2 (MP2.f90:56-74): t = v(i-a)/D, D = e_i + e_j - e_a - e_b.
// E(2) = 1/2 sum [T2aaaa (V_ijab - V_ijba) + T2abab V_ijab - T2abba V_ijba]
//      = sum t(ij,a) (2 v(i-a) - v(i-b))   after the a <-> b re-indexing.
// ----------------------------------------------------------------------------
// The integrals come from the per-amplitude Coulomb factors {v(i-a), v(a-j)} (k_vcoef; the
// same table entries): v(i-b) = v(a-j), since n_i - n_b = n_a - n_j.
__global__ void k_mp2(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                      const AmpInfo *__restrict__ amps, const double2 *__restrict__ vcoef,
                      const double *__restrict__ eigen, double *__restrict__ t,
                      double *__restrict__ part_e, double *__restrict__ part_a, double *__restrict__ part_b)
{
    const ChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    double e = 0.0, mx = 0.0;
    if (loc < s.namp) {
        const int64_t p = s.amp0 + loc;
        const AmpInfo q = amps[p];
        const double *ev = eigen + s.orb0;
        double denom = ev[q.i] + ev[q.j] - ev[q.a] - ev[q.b];
        const double2 vc = vcoef[p];
        double via = vc.x;
        double vib = vc.y;
        // a core pair's integrals are zero (CoreERI), so is its amplitude
        double x = (q.i < s.core_n || q.j < s.core_n) ? 0.0 : via / denom;
        t[p] = x;
        e = x * (2.0 * via - vib);
        mx = fabs(x);
    }
    double dummy = 0.0;
    block_reduce3<kChunk>(e, mx, dummy);
    if (threadIdx.x == 0) { part_e[blockIdx.x] = e; part_a[blockIdx.x] = mx; part_b[blockIdx.x] = 0.0; }
}

// Energy of the current amplitudes and max|t| (the dT before the first iteration).
// kind 0, CCEnergy (CCD.f90:225-227): E = sum t(ij,a) (2 v(i-a) - v(a-j)) after re-indexing;
// kind 1, dRPA CCEnergy (dRPA.f90:206-210): E = sum t (2 v(a-i) - csosex v(b-i)).
// The integrals come from the per-amplitude Coulomb factors {v(i-a), v(a-j)} (k_vcoef):
// v(a-i) = v(i-a), and v(b-i) = v(a-j) since n_b - n_i = n_j - n_a.
__global__ void k_energy(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                         const double2 *__restrict__ vcoef, const double *__restrict__ t, int kind, double csosex,
                         double *__restrict__ part_e, double *__restrict__ part_a, double *__restrict__ part_b)
{
    const ChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    double e = 0.0, mx = 0.0;
    if (loc < s.namp) {
        const int64_t p = s.amp0 + loc;
        double x = t[p];
        const double2 vc = vcoef[p];
        double via = vc.x;
        if (kind == 0) e = x * (2.0 * via - vc.y);
        else e = via * x * 2.0 - vc.y * x * csosex;
        mx = fabs(x);
    }
    double dummy = 0.0;
    block_reduce3<kChunk>(e, mx, dummy);
    if (threadIdx.x == 0) { part_e[blockIdx.x] = e; part_a[blockIdx.x] = mx; part_b[blockIdx.x] = 0.0; }
}

// t'(ij,a) = t(ij,a) - t(ij,b): T2aaaa of spin-adapted amplitudes (MP2.f90:70), the dRPA start.
__global__ void k_to_aaaa(int64_t n, const int32_t *__restrict__ partner, const double *__restrict__ t,
                          double *__restrict__ out)
{
    int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) out[p] = t[p] + (-t[partner[p]]);
}

// Per-solve reduction of the chunk partials in chunk order.
// out[3*s+0] = sum(part_e), out[3*s+1] = max(part_a), out[3*s+2] = max(part_b)
__global__ void k_reduce_solves(const int *__restrict__ chunk_begin, const double *__restrict__ part_e,
                                const double *__restrict__ part_a, const double *__restrict__ part_b,
                                double *__restrict__ out)
{
    const int s = blockIdx.x;
    const int c0 = chunk_begin[s], c1 = chunk_begin[s + 1];
    double e = 0.0, ma = 0.0, mb = 0.0;
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
        e += part_e[c];
        ma = fmax(ma, part_a[c]);
        mb = fmax(mb, part_b[c]);
    }
    block_reduce3<256>(e, ma, mb);
    if (threadIdx.x == 0) { out[3 * s + 0] = e; out[3 * s + 1] = ma; out[3 * s + 2] = mb; }
}

// ----------------------------------------------------------------------------
// Ladders (GetG2Ladders, CCD.f90:588-686), per K block, written as
//   G_K = t_K W_K + H_K t_K
// particle-particle (CCD.f90:660-681): W_K[c][a] = v(c-a) over the block's virtuals;
// hole-hole (CCD.f90:611-657): H_K[p][q] = v(i_p - k_q) + sum_c t_K[p][c] v(c - k_q),
// p = (i,j), q = (k,l), after the pair-swap re-indexing t(kl,b) = t(lk,a).
// k_ladder3 in mode 1 builds H_K; in mode 0 it writes G (overwriting, so it runs first).
// Both run over the rows p = (i,j) with i <= j only: by the pair symmetry
// t(ij,a) = t(ji,b) (T2abab(ij,ab) = T2abab(ji,ba)) the ladder G of the mirror row (j,i)
// at column b = K - a equals that of (i,j) at a, and k_update reads G only on the rows
// i <= j (it updates each mirror from its pair).  The reference forms both rows
// (CCD.f90:617-681); the two agree to rounding.
// ----------------------------------------------------------------------------
constexpr int kVtabSmem = kVtabSmemEntries;  // |q|^2 table entries staged in shared memory

// Ladder tiles v3: FP64 tensor-core MMA (mma.sync m8n8k4 f64; tcgen05 has no f64
// kind).  One warp owns a 32 (a) x NP (p) output tile as 4 x NP/8 fragments of 8x8;
// a CTA of 4 warps covers 128 columns.  Each lane generates its own element of the
// Coulomb fragment, A[a][c] = v(n_a - n_c), from the |q|^2 table, so the Coulomb
// tile never passes through shared memory; the t fragment is read from L1/L2.
//   mode 0: G^T[a][p] = sum_c v(a-c) t[p][c] (+ sum_q t[q][a] H[p][q] when do_hh)
//   mode 1: H^T[q][p] = v(i_p - k_q) + sum_c v(k_q - c) t[p][c]   (columns = pairs)
// Fragment layouts (PTX ISA, m8n8k4 .f64): A row = lane/4, col = lane%4;
// B row (k) = lane%4, col = lane/4; C row = lane/4, cols 2*(lane%4) + {0,1}.
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// The t rows of the tile pass through shared memory in chunks of kLadKC columns,
// double-buffered with cp.async (8-byte copies: rows of odd length are not 16-byte
// aligned); the block's virtual n-vectors and the |q|^2 table are staged once.
constexpr int kLadKC = 32;            // c columns per chunk (mode 0)
constexpr int kLadLd = kLadKC + 4;    // chunk row stride: = 4 mod 16 doubles, conflict-free fragments
// The hole-hole intermediate (mode 1) has little work per column: wider chunks, fewer of the
// round trips that bound it
constexpr int kLadKC1 = 64;   // the default; the launch-shape tuner may pick 32 (DevBatch::hh_kc)

__device__ __forceinline__ void cp_async8(double *dst, const double *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

size_t ladder_smem_bytes(int max_v, int np)
{
    return sizeof(double) * (2 * (size_t)np * kLadLd + kVtabSmem) + sizeof(int) * (size_t)max_v;
}
size_t ladder1_smem_bytes(int max_v, int np, int kc)
{
    return sizeof(double) * (2 * (size_t)np * (kc + 4) + kVtabSmem) + sizeof(int) * (size_t)max_v;
}

// PAIRED (blocks with at most 4 rows i <= j, NP = 8): the fragment's 8 columns hold the
// rows p and, after them, the same rows with the c columns swapped to their partners
// (t[p][pcol c]).  The block's Coulomb kernel is invariant under (a, c) -> (pcol a, pcol c),
// so the second half gives G[p][pcol a] from the same Coulomb fragment: the tile runs over
// the columns a <= pcol a only, half the fragments.  The hole-hole intermediate pairs its
// columns q with their mirror pairs q' the same way (v(k_q' - pcol c) = v(k_q - c)), and the
// hole-hole apply reads H[p][q'] for the second half (t[q][pcol a] = t[q'][a]).
template <int NP, bool KS, bool PAIRED, int KC = kLadKC>
__device__ __forceinline__ void ladder3_tile(const LadderTile &T, const BlockDev &B, const SolveDev &s,
                                             const int16_t *__restrict__ vir, const int16_t *__restrict__ pair_i,
                                             const int *__restrict__ nvp, const double *__restrict__ vtab,
                                             const double *__restrict__ t, const double *__restrict__ H, int mode,
                                             int do_pp, int do_hh, double *__restrict__ out, const double *sv,
                                             bool vsm, double *ts, const int *nvc)
{
    constexpr int NN = NP / 8;  // n fragments
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    const int v = B.v, o = B.o;
    const int orow = B.nd + B.dg;   // rows computed: pairs i < j and the diagonal pair
    const int vc = B.nvd + B.sd;    // columns a <= pcol a
    const int ncol = mode == 0 ? (PAIRED ? vc : v) : (PAIRED ? orow : o);
    // partner column of a virtual column, mirror of a pair row (both involutions)
    auto pcolv = [&](int c) { return c < B.nvd ? c + vc : c < vc ? c : c - vc; };
    auto mirq = [&](int q) { return q < B.nd ? q + orow : q < orow ? q : q - orow; };
    // hole-hole intermediate with at most 32 columns left: the 4 warps share the columns
    // and split the c sum instead (each takes every 4th k step), then reduce
    const bool ksplit = KS && ncol - T.a0 <= 32;
    const int colbase = ksplit ? T.a0 : T.a0 + warp * 32;
    const bool wact = colbase < ncol;  // warps past the last column only help with the copies
    // packed n-vectors of this lane's A-fragment rows (one per m fragment)
    int na[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        int col = colbase + m * 8 + gid;
        na[m] = 0;
        if (col < ncol) na[m] = nvp[s.orb0 + (mode == 0 ? vir[B.vir0 + col] : pair_i[B.pair0 + col])];
    }
    double acc[4][NN][2];
#pragma unroll
    for (int m = 0; m < 4; m++)
#pragma unroll
        for (int n = 0; n < NN; n++) acc[m][n][0] = acc[m][n][1] = 0.0;
    if (do_pp || mode == 1) {
        constexpr int LD = KC + 4;
        const int nchunk = (v + KC - 1) / KC;
        const double *trow0 = t + B.t0;
        // chunk j of the tile's t rows -> buffer b
        auto issue = [&](int j, int b) {
            double *dst = ts + b * (NP * LD);
            const int c0 = j * KC;
            for (int e = threadIdx.x; e < NP * KC; e += blockDim.x) {
                const int r = e / KC, c = e - r * KC;
                const int cc = c0 + c;
                if (PAIRED) {
                    // rows [0, orow): t[p][c]; rows [orow, 2 orow): t[p][pcol c]
                    const bool second = r >= orow;
                    const int p = second ? r - orow : r;
                    if (r < 2 * orow && cc < v)
                        cp_async8(dst + r * LD + c, trow0 + (int64_t)p * v + (second ? pcolv(cc) : cc));
                    else dst[r * LD + c] = 0.0;
                } else {
                    const int p = T.p0 + r;
                    if (p < orow && cc < v) cp_async8(dst + r * LD + c, trow0 + (int64_t)p * v + cc);
                    else dst[r * LD + c] = 0.0;
                }
            }
            cp_async_commit();
        };
        issue(0, 0);
        for (int j = 0; j < nchunk; j++) {
            if (j + 1 < nchunk) {
                issue(j + 1, (j + 1) & 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (wact) {
                const double *tb = ts + (j & 1) * (NP * LD);
                const int c0 = j * KC;
                const int kstart = KS && ksplit ? 4 * warp : 0, kstep = KS && ksplit ? 16 : 4;
#pragma unroll 2
                for (int kk = kstart; kk < KC; kk += kstep) {
                    const int c = min(c0 + kk + tig, v - 1);  // beyond v the t column is zero
                    const int nc = nvc[c];
                    double bf[NN];
#pragma unroll
                    for (int n = 0; n < NN; n++) bf[n] = tb[(n * 8 + gid) * LD + kk + tig];
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int q2 = q2p(na[m], nc);
                        const double af = vsm ? sv[q2] : __ldg(&vtab[s.vtab0 + q2]);
#pragma unroll
                        for (int n = 0; n < NN; n++) dmma_884(acc[m][n][0], acc[m][n][1], af, bf[n]);
                    }
                }
            }
            __syncthreads();
        }
    }
    if (KS && ksplit) {
        // acc of warps 2, 3 into warps 0, 1, then warp 1 into warp 0 (through the idle chunk buffer)
        constexpr int kPart = 4 * NN * 2 * 32;
        for (int round = 0; round < 2; round++) {
            const int lo = round == 0 ? 2 : 1, nw = round == 0 ? 2 : 1;
            if (warp >= lo && warp < lo + nw) {
                double *dst = ts + (warp - lo) * kPart;
#pragma unroll
                for (int m = 0; m < 4; m++)
#pragma unroll
                    for (int n = 0; n < NN; n++)
#pragma unroll
                        for (int h = 0; h < 2; h++) dst[((m * NN + n) * 2 + h) * 32 + lane] = acc[m][n][h];
            }
            __syncthreads();
            if (warp < nw) {
                const double *src = ts + warp * kPart;
#pragma unroll
                for (int m = 0; m < 4; m++)
#pragma unroll
                    for (int n = 0; n < NN; n++)
#pragma unroll
                        for (int h = 0; h < 2; h++) acc[m][n][h] += src[((m * NN + n) * 2 + h) * 32 + lane];
            }
            __syncthreads();
        }
        if (warp != 0) return;
    }
    if (!wact) return;  // no barriers below
    if (mode == 0 && do_hh) {
        // acc[a][p] += sum_q t[q][a] H[p][q]
        for (int q0 = 0; q0 < o; q0 += 4) {
            const int q = q0 + tig;
            const bool qok = q < o;
            double bf[NN];
#pragma unroll
            for (int n = 0; n < NN; n++) {
                if (PAIRED) {
                    const int nn = n * 8 + gid;
                    const bool second = nn >= orow;
                    const int p = second ? nn - orow : nn;
                    bf[n] = (qok && nn < 2 * orow) ? H[(int64_t)p * o + (second ? mirq(q) : q)] : 0.0;
                } else {
                    int p = T.p0 + n * 8 + gid;
                    bf[n] = (qok && p < orow) ? H[(int64_t)p * o + q] : 0.0;
                }
            }
#pragma unroll
            for (int m = 0; m < 4; m++) {
                int col = colbase + m * 8 + gid;
                double af = (qok && col < v) ? __ldg(&t[B.t0 + (int64_t)q * v + col]) : 0.0;
#pragma unroll
                for (int n = 0; n < NN; n++) dmma_884(acc[m][n][0], acc[m][n][1], af, bf[n]);
            }
        }
    }
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int col = colbase + m * 8 + gid;
        if (col >= ncol) continue;
#pragma unroll
        for (int n = 0; n < NN; n++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int p = T.p0 + n * 8 + 2 * tig + h, oc = col;
                int nq = na[m];
                if (PAIRED) {
                    const int nn = n * 8 + 2 * tig + h;
                    if (nn >= 2 * orow) continue;
                    if (nn >= orow) {
                        // the partner column (mode 0) or mirror pair (mode 1); once on self-partners
                        p = nn - orow;
                        oc = mode == 0 ? pcolv(col) : mirq(col);
                        if (oc == col) continue;
                        if (mode == 1) nq = nvp[s.orb0 + pair_i[B.pair0 + oc]];
                    }
                }
                if (p >= orow) continue;
                if (mode == 0) {
                    out[B.t0 + (int64_t)p * v + oc] = acc[m][n][h];
                } else {
                    const int ni = nvp[s.orb0 + pair_i[B.pair0 + p]];
                    const int q2 = q2p(ni, nq);
                    out[(int64_t)p * o + oc] = (vsm ? sv[q2] : vtab[s.vtab0 + q2]) + acc[m][n][h];
                }
            }
    }
}

// One kernel per row tile NP (8, 16, 24, 32 pairs): the small tiles need fewer registers
// and less shared memory, so more CTAs fit on an SM to hide the lookup latency.
// KC1: the hole-hole intermediate's column chunk (mode 1), 64 or 32 (the launch-shape tuner's pick)
template <int NP, bool PAIRED, int KC1 = kLadKC1>
__global__ void __launch_bounds__(128, NP <= 8 ? 8 : NP <= 16 ? 6 : 4)
    k_ladder3(const LadderTile *__restrict__ tiles, const BlockDev *__restrict__ blocks,
              const SolveDev *__restrict__ solves, const int16_t *__restrict__ vir,
              const int16_t *__restrict__ pair_i, const int *__restrict__ nvp,
              const double *__restrict__ vtab, const double *__restrict__ t, const int64_t *__restrict__ hh0,
              double *__restrict__ hh, int mode, int do_pp, int do_hh, double *__restrict__ g,
              const uint8_t *__restrict__ active)
{
    const LadderTile T = tiles[blockIdx.x];
    const BlockDev B = blocks[T.blk];
    if (!active[B.solve]) return;
    const SolveDev s = solves[B.solve];
    extern __shared__ double lsm[];
    double *ts = lsm;                              // 2 x NP x (chunk width + 4)
    double *sv = ts + 2 * NP * (mode == 1 ? KC1 + 4 : kLadLd);   // kVtabSmem
    int *nvc = (int *)(sv + kVtabSmem);            // v_K packed n-vectors of the block's virtuals
    const bool vsm = s.q2max < kVtabSmem;
    if (vsm)
        for (int q = threadIdx.x; q <= s.q2max; q += blockDim.x) sv[q] = vtab[s.vtab0 + q];
    for (int c = threadIdx.x; c < B.v; c += blockDim.x) nvc[c] = nvp[s.orb0 + vir[B.vir0 + c]];
    __syncthreads();
    double *H = hh + hh0[T.blk];
    double *out = mode == 0 ? g : H;
    // the hole-hole intermediate (mode 1) may split its c sum across the warps
    if (mode == 1)
        ladder3_tile<NP, true, PAIRED, KC1>(T, B, s, vir, pair_i, nvp, vtab, t, H, mode, do_pp, do_hh, out, sv,
                                                vsm, ts, nvc);
    else
        ladder3_tile<NP, false, PAIRED>(T, B, s, vir, pair_i, nvp, vtab, t, H, mode, do_pp, do_hh, out, sv, vsm, ts,
                                        nvc);
}

// The dynamic shared-memory limits only grow (batches of different sizes coexist), under
// one lock: batches are created from several host threads while others solve.  Kernel
// attributes belong to a device, so each device keeps its own limits (the caller has made
// the batch's device current).
static std::mutex g_smem_limit_mu;

void set_ladder_smem_limit(int max_v)
{
    std::lock_guard<std::mutex> lock(g_smem_limit_mu);
    static int current_by_dev[kMaxDevices] = {};   // attributes are per device
    const int dev = current_device() % kMaxDevices;
    int &current = current_by_dev[dev];
    if (max_v > current) {
        auto lb = [&](int np) {
            return (int)std::max(ladder_smem_bytes(max_v, np), ladder1_smem_bytes(max_v, np, kLadKC1));
        };
        const int b8 = lb(8);
        cudaFuncSetAttribute(k_ladder3<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b8);
        cudaFuncSetAttribute(k_ladder3<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b8);
        cudaFuncSetAttribute(k_ladder3<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(16));
        cudaFuncSetAttribute(k_ladder3<24, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(24));
        cudaFuncSetAttribute(k_ladder3<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(32));
        cudaFuncSetAttribute(k_ladder3<8, true, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, b8);
        cudaFuncSetAttribute(k_ladder3<8, false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, b8);
        cudaFuncSetAttribute(k_ladder3<16, false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(16));
        cudaFuncSetAttribute(k_ladder3<24, false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(24));
        cudaFuncSetAttribute(k_ladder3<32, false, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, lb(32));
        current = max_v;
    }
}

// Ladder tiles in row-tile classes (sorted: paired 8, then 8, 16, 24, 32 pairs; counts in
// ncls): one launch per non-empty class.  Returns the launches.
static int launch_ladder3(const DevBatch &d, const LadderTile *tiles, const int *ncls, const double *t, int mode,
                          int do_pp, int do_hh, double *g, cudaStream_t st)
{
    int off = 0, n = 0;
    for (int c = 0; c < kLadderClasses; c++) {
        const int cnt = ncls[c];
        if (cnt <= 0) continue;
        const int np = c == 0 ? 8 : 8 * c;
        const bool kc32 = mode == 1 && d.hh_kc == 32;
        const size_t sm = mode == 1 ? ladder1_smem_bytes(d.max_v, np, kc32 ? 32 : kLadKC1) : ladder_smem_bytes(d.max_v, np);
#define UEGCCD_LADDER_ARGS                                                                                  \
    tiles + off, d.blocks, d.solves, d.vir, d.pair_i, d.nvp, d.vtab, t, d.hh0, d.hh, mode, do_pp, do_hh, \
        g, d.active
        if (kc32) {
            switch (c) {
            case 0: k_ladder3<8, true, 32><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 1: k_ladder3<8, false, 32><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 2: k_ladder3<16, false, 32><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 3: k_ladder3<24, false, 32><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            default: k_ladder3<32, false, 32><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            }
        } else {
            switch (c) {
            case 0: k_ladder3<8, true><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 1: k_ladder3<8, false><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 2: k_ladder3<16, false><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            case 3: k_ladder3<24, false><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            default: k_ladder3<32, false><<<cnt, 128, sm, st>>>(UEGCCD_LADDER_ARGS); break;
            }
        }
#undef UEGCCD_LADDER_ARGS
        off += cnt;
        n++;
    }
    return n;
}

// ----------------------------------------------------------------------------
// Mosaics (GetG2Mosaics, CCD.f90:548-582):
//   s(k,l,c) = v(c-k) (T2aaaa + T2abab)(kl,c) - v(c-l) (T2aaaa + T2abba)(kl,c)
//            = v(c-k) (2t(kl,c) - t(kl,d)) - v(c-l) (t(kl,c) - 2t(kl,d))
//   Jvv(c) = sum_{k,l} s(k,l,c),  Joo(k) = sum_{l,c} s(k,l,c)
// dRPA (dRPA.f90:415-431): s(k,l,c) = 2 v(c-k) t(kl,c).
// s lives only in registers: one CTA per K block forms it row by row (d = K - c is
// in the same row) and writes the block's row sums (-> Joo of the row's k) and
// column sums (-> Jvv of the column's c); k_mosaic_sum adds the partials of each
// target in a fixed order.
// ----------------------------------------------------------------------------
constexpr int kMosThreads = 128;

size_t mosaic_smem_bytes(int max_v, int max_o, int vt_n)
{
    return sizeof(double) * ((size_t)vt_n + 2 * (size_t)max_v + (size_t)(kMosThreads / 32) * max_o) +
           sizeof(int) * (2 * (size_t)max_v + 2 * (size_t)max_o);
}

// The threads own the columns (c = tid + k * kMosThreads) and walk the rows: all warps stay
// busy however few rows a block has.  Column sums stay with their thread; row sums are
// reduced per warp, then over the warps in a fixed order.
__global__ void __launch_bounds__(kMosThreads) k_mosaic_blk(const BlockDev *__restrict__ blocks,
                                                           const SolveDev *__restrict__ solves,
                                                           const int16_t *__restrict__ pair_i,
                                                           const int16_t *__restrict__ pair_j,
                                                           const int16_t *__restrict__ vir,
                                                           const int *__restrict__ nvp,
                                                           const double *__restrict__ vtab,
                                                           const double *__restrict__ t,
                                                           const int16_t *__restrict__ pcol, int drpa,
                                                           double *__restrict__ mpart,
                                                           const uint8_t *__restrict__ active, int vt_n)
{
    const BlockDev B = blocks[blockIdx.x];
    if (!active[B.solve]) return;
    const SolveDev s = solves[B.solve];
    const int v = B.v, oc = B.nd + B.dg;
    constexpr int kW = kMosThreads / 32;
    extern __shared__ double msm[];
    double *sv = msm;                          // vt_n: the batch's largest |q|^2 table (at most kVtabSmem)
    double *coff = sv + vt_n;                  // v: column sums over the rows i < j
    double *cdg = coff + v;                    // v: the diagonal pair's row (if any)
    double *wrs = cdg + v;                     // kW x oc: per-warp row sums
    int *nvc = (int *)(wrs + kW * oc);         // v: packed n-vectors of the block's virtuals
    int *nk = nvc + v, *nl = nk + oc;          // oc: packed n-vectors of each row's k and l
    int *pc = nl + oc;                         // v: column of the partner d = K - c
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool vsm = s.q2max < vt_n;
    if (vsm)
        for (int q = tid; q <= s.q2max; q += kMosThreads) sv[q] = vtab[s.vtab0 + q];
    for (int c = tid; c < v; c += kMosThreads) {
        nvc[c] = nvp[s.orb0 + vir[B.vir0 + c]];
        pc[c] = pcol[B.vir0 + c];
        coff[c] = cdg[c] = 0.0;
    }
    for (int r = tid; r < oc; r += kMosThreads) {
        nk[r] = nvp[s.orb0 + pair_i[B.pair0 + r]];
        nl[r] = nvp[s.orb0 + pair_j[B.pair0 + r]];
    }
    __syncthreads();
    auto V = [&](int q2) -> double { return vsm ? sv[q2] : __ldg(&vtab[s.vtab0 + q2]); };
    // Rows i <= j only: by the pair symmetry s(l,k,d) = s(k,l,c) for the mirror (l,k) of a
    // row (k,l) and d = K - c, so the mirror row has the same row sum (Joo of l) and adds
    // the column sums of (k,l) with the columns swapped to their partners.  Four rows at a
    // time: their loads go out together (most blocks have at most four rows), and each column
    // sum still takes the rows in order.
    constexpr int kR = 4;
    for (int r0 = 0; r0 < oc; r0 += kR) {
        const int nr = min(kR, oc - r0);
        const double *row[kR];
        int rk[kR], rl[kR];
        double rs[kR];
#pragma unroll
        for (int q = 0; q < kR; q++) {
            const int r = min(r0 + q, oc - 1);
            row[q] = t + B.t0 + (int64_t)r * v;
            rk[q] = nk[r];
            rl[q] = nl[r];
            rs[q] = 0.0;
        }
        for (int c = tid; c < v; c += kMosThreads) {
            const int ncv = nvc[c];
            const int pcc = drpa ? c : pc[c];
            double x[kR], y[kR];
#pragma unroll
            for (int q = 0; q < kR; q++) {
                x[q] = q < nr ? row[q][c] : 0.0;
                y[q] = (q < nr && !drpa) ? row[q][pcc] : 0.0;   // t(kl, d), same row
            }
#pragma unroll
            for (int q = 0; q < kR; q++) {
                if (q >= nr) continue;
                const double vck = V(q2p(ncv, rk[q]));
                double sval;
                if (drpa) {
                    sval = 2.0 * vck * x[q];
                } else {
                    const double vcl = V(q2p(ncv, rl[q]));
                    sval = vck * (2.0 * x[q] - y[q]) - vcl * (x[q] - 2.0 * y[q]);
                }
                rs[q] += sval;
                if (r0 + q >= B.nd) cdg[c] = sval;
                else coff[c] += sval;
            }
        }
#pragma unroll
        for (int q = 0; q < kR; q++) {
            double v0 = rs[q];
            for (int off = 16; off > 0; off >>= 1) v0 += __shfl_down_sync(0xffffffffu, v0, off);
            if (lane == 0 && q < nr) wrs[warp * oc + r0 + q] = v0;
        }
    }
    __syncthreads();
    for (int r = tid; r < oc; r += kMosThreads) {
        double rs = 0.0;
        for (int w = 0; w < kW; w++) rs += wrs[w * oc + r];
        mpart[B.row0 + r] = rs;
        if (r < B.nd) mpart[B.row0 + r + oc] = rs;   // the mirror row
    }
    for (int c = tid; c < v; c += kMosThreads) mpart[B.col0 + c] = coff[c] + coff[pc[c]] + cdg[c];
}

// One warp per target: targets (s, y < V) are Jvv(c = O + y), (s, y >= V) are Joo(k = y - V).
// The per-target lists k_mosaic_sum adds, built once per batch, one CTA per solve: target y
// < V (the virtual O + y) lists the column partials of every block holding that virtual,
// target V + k the row partials of the pair rows (k, l); both in block order, the order
// k_mosaic_sum then adds them in.  A virtual is one column of a block at most, and an
// occupied k the first index of one row at most (l = K - k), so within a block the targets
// are distinct and the block's entries go in at once.  mt_start[tbase[s] + y] is the first
// entry of target y of solve s (entries from lbase[s] on); the last solve also writes the
// end sentinel.  cnt: V + O ints of dynamic shared memory.
__global__ void k_mosaic_targets(const SolveDev *__restrict__ solves, const BlockDev *__restrict__ blocks,
                                 const int16_t *__restrict__ vir, const int16_t *__restrict__ pair_i,
                                 const int *__restrict__ tbase, const int64_t *__restrict__ lbase,
                                 int32_t *__restrict__ mt_start, int32_t *__restrict__ mt_list)
{
    extern __shared__ int cnt[];
    const int sv = blockIdx.x;
    const SolveDev S = solves[sv];
    const int nt = S.V + S.O, t0 = tbase[sv];
    for (int y = threadIdx.x; y < nt; y += blockDim.x) cnt[y] = 0;
    __syncthreads();
    for (int bi = 0; bi < S.nblk; bi++) {
        const BlockDev B = blocks[S.blk0 + bi];
        for (int c = threadIdx.x; c < B.v; c += blockDim.x) atomicAdd(&cnt[vir[B.vir0 + c] - S.O], 1);
        for (int r = threadIdx.x; r < B.o; r += blockDim.x) atomicAdd(&cnt[S.V + pair_i[B.pair0 + r]], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t run = lbase[sv];
        for (int y = 0; y < nt; y++) {
            mt_start[t0 + y] = (int32_t)run;
            run += cnt[y];
            cnt[y] = 0;
        }
        mt_start[t0 + nt] = (int32_t)run;   // the next solve's first entry, or the end sentinel
    }
    __syncthreads();
    for (int bi = 0; bi < S.nblk; bi++) {
        const BlockDev B = blocks[S.blk0 + bi];
        for (int c = threadIdx.x; c < B.v; c += blockDim.x) {
            const int y = vir[B.vir0 + c] - S.O;
            mt_list[mt_start[t0 + y] + cnt[y]++] = (int32_t)(B.col0 + c);
        }
        for (int r = threadIdx.x; r < B.o; r += blockDim.x) {
            const int y = S.V + pair_i[B.pair0 + r];
            mt_list[mt_start[t0 + y] + cnt[y]++] = (int32_t)(B.row0 + r);
        }
        __syncthreads();
    }
}

void launch_mosaic_targets(const DevBatch &d, const int *tbase, const int64_t *lbase, size_t smem, cudaStream_t st)
{
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_mosaic_targets, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mosaic_targets<<<d.nsolves, 256, smem, st>>>(d.solves, d.blocks, d.vir, d.pair_i, tbase, lbase, d.mt_start,
                                                   d.mt_list);
}

__global__ void __launch_bounds__(256) k_mosaic_sum(const int2 *__restrict__ targets, int ntargets,
                                                   const SolveDev *__restrict__ solves,
                                                   const int32_t *__restrict__ mt_start,
                                                   const int32_t *__restrict__ mt_list,
                                                   const double *__restrict__ mpart, double *__restrict__ jvv,
                                                   double *__restrict__ joo, const uint8_t *__restrict__ active)
{
    const int lane = threadIdx.x & 31;
    const int tix = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (tix >= ntargets) return;
    const int2 tg = targets[tix];
    if (!active[tg.x]) return;
    double a = 0.0;
    for (int e = mt_start[tix] + lane; e < mt_start[tix + 1]; e += 32) a += mpart[mt_list[e]];
    for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
    if (lane == 0) {
        const SolveDev s = solves[tg.x];
        if (tg.y < s.V) jvv[s.jvv0 + tg.y] = a;
        else joo[s.joo0 + tg.y - s.V] = a;
    }
}

void set_mosaic_smem_limit(size_t bytes)
{
    std::lock_guard<std::mutex> lock(g_smem_limit_mu);
    static size_t current_by_dev[kMaxDevices] = {};   // attributes are per device
    size_t &current = current_by_dev[current_device() % kMaxDevices];
    if (current < 48 * 1024) current = 48 * 1024;
    if (bytes > current) {
        cudaFuncSetAttribute(k_mosaic_blk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        current = bytes;
    }
}

// ----------------------------------------------------------------------------
// dRPA ring intermediate (dRPA.f90:517-535), for every (i, x, l) with x virtual:
//   J1 = sum_k 2 t(ik,x) v(i-x).
// The reference skips (i,x,l) when d = n_l + n_x - n_i is not a virtual; the apply
// step in k_update makes the same test, so J1 is formed for every l.
// Layout: J1[ph0 + (i*V + x)*O + l].  (The CCD rings use k_rings.)
// ----------------------------------------------------------------------------
__global__ void k_ring_int(const ChunkDev *__restrict__ rchunks, const SolveDev *__restrict__ solves,
                           const int32_t *__restrict__ pos, const int4 *__restrict__ nv4,
                           const double *__restrict__ vtab, const double *__restrict__ t,
                           double *__restrict__ J1, const uint8_t *__restrict__ active)
{
    const ChunkDev ch = rchunks[blockIdx.x];
    if (!active[ch.solve]) return;
    const SolveDev s = solves[ch.solve];
    const int O = s.O, V = s.V;
    const int e = ch.start + threadIdx.x;
    if (e >= O * V * O) return;
    const int ix = e / O;
    const int x = ix % V + O;
    const int i = ix / V;
    const double vd = vpq(s, nv4, vtab, i, x);
    double j1 = 0.0;
    for (int k = 0; k < O; k++) {
        const int p1 = posmap(s, pos, i, k, x);
        if (p1 >= 0) j1 += 2.0 * t[p1] * vd;
    }
    J1[s.ph0 + e] = j1;
}

// ----------------------------------------------------------------------------
// Rings and crossed rings in particle-hole form (CCD).
// For every ph row (i,x), x virtual, with c = partner of (i,k,x):
//   X[k] = t(ik,x),  Y[k] = t(ik,c)                 (= t(ki,x) by the pair swap)
//   Sx = sum_k X, Sy = sum_k Y
//   Ex[j] = sum_k v(k-j) X[k],  Ey[j] = sum_k v(k-j) Y[k]
//   XW[l] = sum_k X[k] v(i+k-x-l), YW[l] = sum_k Y[k] v(i+k-x-l)
// and the quadratic-ring intermediates of CCD.f90:774-797 / 902-925 become
//   A1 = J1 + J2 = 2 vd (2Sx - Sy) - 2 XW + YW,  A2 = J2 = vd (2Sx - Sy) - XW,  A3 = J3 = YW,
// vd = v(i-x).  Then, for the amplitude (i,j,a) with partner b (rows ia, jb, ib, ja):
//   linear rings   (CCD.f90:716-763): 2 v(i-a)(Sx_ia + Sx_jb) - v(i-a)(Sy_ia + Sy_jb) - Ex_ia[j] - Ex_jb[i]
//   linear xrings  (CCD.f90:845-892): -Ey_ib[j] - Ey_ja[i]
//   quadratic rings  (CCD.f90:801-808): A1_ia . X_jb - A2_ia . Y_jb
//   quadratic xrings (CCD.f90:927-934): A3_ib . Y_ja
// The quadratic products pair the rows of momentum Q with those of -Q, group by
// group; every amplitude receives exactly one ring and one crossed-ring product, so
// no atomics are needed.
// Row layout: row r (local) of solve s: scalars at s.phr0 + r, vectors at s.ph0 + r * O (O entries).
// ----------------------------------------------------------------------------
// ----------------------------------------------------------------------------
// Fused rings: one CTA per pair of ph groups {Q, -Q}.  Everything of the formulas
// above happens in shared memory: X, Y rows of both groups, the exchange kernels
// W_Q[k][l] = v(n_k - n_l - Q) and W_-Q, the direct occupied kernel
// Vocc[j][k] = v(n_k - n_j), the A rows (chunk by chunk) and the products.  Each
// pair of rows (r1 in one group, r2 in the other) owns two amplitudes:
//   ring  amplitude (i1, i2, a = x1):  lin + A1_r1 . X_r2 - A2_r1 . Y_r2
//   xring amplitude (i1, i2, a = x2):  xlin + A3_r1 . Y_r2
// with lin = 2 vd_r1 (Sx_r1 + Sx_r2) - vd_r1 (Sy_r1 + Sy_r2) - Ex_r1[i2] - Ex_r2[i1]
// and xlin = -Ey_r1[i2] - Ey_r2[i1]; Ex/Ey elements are formed where used.
// ----------------------------------------------------------------------------
constexpr int kRingCh = 16;  // A rows per chunk

// The FMA form below serves group pairs too large for k_rings' shared-memory tiles
// (NOcc around 57 and above).
__global__ void __launch_bounds__(256) k_rings_wide(const RingPairDev *__restrict__ pairs,
                                               const SolveDev *__restrict__ solves,
                                               const int16_t *__restrict__ ph_i, const int16_t *__restrict__ ph_x,
                                               const int32_t *__restrict__ pos, const int32_t *__restrict__ partner,
                                               const int4 *__restrict__ nv4, const double *__restrict__ vtab,
                                               const double *__restrict__ t, int do_ring, int do_xring,
                                               double *__restrict__ rx,
                                               const uint8_t *__restrict__ active)
{
    const RingPairDev P = pairs[blockIdx.x];
    if (!active[P.solve]) return;
    const SolveDev s = solves[P.solve];
    const int O = s.O;
    const int R = P.n1 + P.n2;
    const int N2 = (P.n2 + 7) & ~7;   // rx row: ring G of the group-2 columns, then crossed-ring G
    // shared-memory strides are odd so that consecutive threads hit distinct banks
    const int ld = O | 1, lr = R | 1;
    extern __shared__ double smem[];
    double *sv = smem;                                   // kVtabSmem
    double *Vo = sv + kVtabSmem;                         // O x ld : Vo[k*ld + j] = v(n_k - n_j)
    double *W1 = Vo + O * ld;                            // O x ld : W_Q[k][l]
    double *W2 = W1 + O * ld;                            // O x ld : W_-Q[k][l]
    double *XT = W2 + O * ld;                            // O x lr : X[r][k] at k*lr + r
    double *YT = XT + O * lr;                            // O x lr
    double *A1 = YT + O * lr;                            // kRingCh x ld
    double *A2 = A1 + kRingCh * ld;
    double *A3 = A2 + kRingCh * ld;
    double *Sx = A3 + kRingCh * ld;                      // R
    double *Sy = Sx + R;                                 // R
    double *Vd = Sy + R;                                 // R
    int *ri = (int *)(Vd + R);                           // R
    int *rxv = ri + R;                                   // R: the row's virtual
    int4 *no = (int4 *)(((uintptr_t)(rxv + R) + 15) & ~(uintptr_t)15);  // O occupied n-vectors
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool vsm = s.q2max < kVtabSmem;
    if (vsm)
        for (int q = tid; q <= s.q2max; q += nt) sv[q] = vtab[s.vtab0 + q];
    for (int k = tid; k < O; k += nt) no[k] = nv4[s.orb0 + k];
    for (int r = tid; r < R; r += nt) {
        const int64_t row = s.phr0 + (r < P.n1 ? P.r1 + r : P.r2 + r - P.n1);
        ri[r] = ph_i[row];
        rxv[r] = ph_x[row];
    }
    __syncthreads();
    auto V = [&](int q2) -> double { return q2 > s.q2max ? 0.0 : (vsm ? sv[q2] : vtab[s.vtab0 + q2]); };
    // Q of group 1 = n_x - n_i of its first row
    const int4 qa = nv4[s.orb0 + rxv[0]], qb = nv4[s.orb0 + ri[0]];
    const int Qx = qa.x - qb.x, Qy = qa.y - qb.y, Qz = qa.z - qb.z;
    for (int e = tid; e < O * O; e += nt) {
        const int k = e / O, l = e % O;
        const int4 nk = no[k], nl = no[l];
        const int dx = nk.x - nl.x, dy = nk.y - nl.y, dz = nk.z - nl.z;
        Vo[k * ld + l] = V(dx * dx + dy * dy + dz * dz);
        const int ax = dx - Qx, ay = dy - Qy, az = dz - Qz;
        W1[k * ld + l] = V(ax * ax + ay * ay + az * az);
        const int bx = dx + Qx, by = dy + Qy, bz = dz + Qz;
        W2[k * ld + l] = V(bx * bx + by * by + bz * bz);
    }
    // X, Y rows (stored transposed)
    for (int e = tid; e < R * O; e += nt) {
        const int k = e / R, r = e % R;
        const int p = posmap(s, pos, ri[r], k, rxv[r]);
        double xv = 0.0, yv = 0.0;
        if (p >= 0) {
            xv = t[p];
            yv = t[partner[p]];
        }
        XT[k * lr + r] = xv;
        YT[k * lr + r] = yv;
    }
    __syncthreads();
    for (int r = tid; r < R; r += nt) {
        double sx = 0.0, sy = 0.0;
        for (int k = 0; k < O; k++) {
            sx += XT[k * lr + r];
            sy += YT[k * lr + r];
        }
        Sx[r] = sx;
        Sy[r] = sy;
        const int4 ni = nv4[s.orb0 + ri[r]], nx = nv4[s.orb0 + rxv[r]];
        Vd[r] = V(q2_of(ni, nx));
    }
    __syncthreads();
    // rows of group 1 against group 2: the values at (a, b) are the ring G of (i_a, i_b, x_a)
    // and the crossed-ring G of (i_a, i_b, x_b), which k_update reads for each amplitude or
    // its mirror (the reverse direction gives the mirrors' values: not needed)
    for (int dir = 0; dir < 1; dir++) {
        const int a0 = dir == 0 ? 0 : P.n1, na = dir == 0 ? P.n1 : P.n2;
        const int b0 = dir == 0 ? P.n1 : 0, nb = dir == 0 ? P.n2 : P.n1;
        const double *W = dir == 0 ? W1 : W2;
        for (int c0 = 0; c0 < na; c0 += kRingCh) {
            const int nc = min(kRingCh, na - c0);
            // A rows of the chunk: XW, YW with the chunk group's exchange kernel
            for (int e = tid; e < nc * O; e += nt) {
                const int rr = e / O, l = e % O;
                const int r = a0 + c0 + rr;
                double xw = 0.0, yw = 0.0;
                for (int k = 0; k < O; k++) {
                    const double w = W[k * ld + l];
                    xw = fma(XT[k * lr + r], w, xw);
                    yw = fma(YT[k * lr + r], w, yw);
                }
                const double base = Vd[r] * (2.0 * Sx[r] - Sy[r]);
                A1[rr * ld + l] = 2.0 * base - 2.0 * xw + yw;
                A2[rr * ld + l] = base - xw;
                A3[rr * ld + l] = yw;
            }
            __syncthreads();
            for (int e = tid; e < nc * nb; e += nt) {
                const int rr = e / nb, r2 = b0 + e % nb;
                const int r1 = a0 + c0 + rr;
                const int i1 = ri[r1], i2 = ri[r2];
                double quad = 0.0, xquad = 0.0, ex12 = 0.0, ex21 = 0.0, ey12 = 0.0, ey21 = 0.0;
                for (int l = 0; l < O; l++) {
                    const double x2 = XT[l * lr + r2], y2 = YT[l * lr + r2];
                    quad = fma(A1[rr * ld + l], x2, quad);
                    quad = fma(-A2[rr * ld + l], y2, quad);
                    xquad = fma(A3[rr * ld + l], y2, xquad);
                    const double vo12 = Vo[l * ld + i2], vo21 = Vo[l * ld + i1];
                    ex12 = fma(vo12, XT[l * lr + r1], ex12);   // Ex_r1[i2]
                    ey12 = fma(vo12, YT[l * lr + r1], ey12);   // Ey_r1[i2]
                    ex21 = fma(vo21, x2, ex21);                // Ex_r2[i1]
                    ey21 = fma(vo21, y2, ey21);                // Ey_r2[i1]
                }
                double *out = rx + P.xy0 + (int64_t)r1 * 2 * N2;
                if (do_ring) {
                    const double vd = Vd[r1];
                    const double lin = 2.0 * vd * (Sx[r1] + Sx[r2]) - vd * (Sy[r1] + Sy[r2]) - ex12 - ex21;
                    out[r2 - P.n1] = lin + quad;
                }
                if (do_xring) out[N2 + r2 - P.n1] = -ey12 - ey21 + xquad;
            }
            __syncthreads();
        }
    }
}


// ----------------------------------------------------------------------------
// Rings on the FP64 tensor cores (mma.sync m8n8k4 f64), one CTA per {Q, -Q}
// group pair, on compressed matrices.  Rows a of group 1 are (i_a, x_a) with
// n_x - n_i = Q; rows b of group 2 are (i_b, x_b) with -Q.  The amplitude
// t(i_a k, x_a) exists exactly for k in occ2 = {i_b}: its partner is x_b.  So every
// ph row of one group is dense over the occupied indices of the other group:
//   X1[a][b] = t(i_a i_b, x_a)   Y1[a][b] = t(i_b i_a, x_a)   (n1 x n2)
// The rows of group 2 hold the same amplitudes transposed: by the pair symmetry
// t(ij, a) = t(ji, b) (T2abab(ij,ab) = T2abab(ji,ba)),
//   X2[b][a] = t(i_b i_a, x_b) = X1[a][b],   Y2[b][a] = t(i_a i_b, x_b) = Y1[a][b],
// so only X1 and Y1 are gathered.  With
//   W[b][a]  = v(n_{i_b} - n_{i_a} - Q)
//   Vs1[a][a'] = v(n_{i_a'} - n_{i_a}),  Vs2[b][b'] = v(n_{i_b'} - n_{i_b})
//   XW1 = X1 W,  U1 = Y1 W - Vs1
// the fused ring form above becomes, for the amplitude pair (a, b):
//   ring (i_a, i_b, x_a) = lin + base_a (2 Sx_b - Sy_b)
//                          + sum_a' [XW1[a][a'] (Y1 - 2 X1)[a'][b] + U1[a][a'] X1[a'][b]]
//                          - sum_b' X1[a][b'] Vs2[b][b']
//   xring(i_a, i_b, x_b) = sum_a' U1[a][a'] Y1[a'][b] - sum_b' Y1[a][b'] Vs2[b][b']
// (lin, base as above; Sx_b, Sy_b are the column sums of X1, Y1).  The residual
// terms share the pair symmetry (ring and crossed-ring G of (j,i,b) equal those of
// (i,j,a)), and k_update reads G only where the first occupied index is the smaller
// one: the ring value goes to (i_a, i_b, x_a) or to its mirror (i_b, i_a, x_b), the
// crossed-ring value to (i_a, i_b, x_b) or to (i_b, i_a, x_a).  The reference forms
// both halves separately (CCD.f90:716-937); the two agree to rounding.
// Group 1 is the smaller group (the host orders each pair), which minimises both the
// shared memory, 2 N1 (N1 + N2 + 8) doubles, and the work, 5 N1^2 N2 + 2 N1 N2^2 DMMA
// multiply-adds.  Row strides are the padded width + 4 (= 4 or 12 mod 16 doubles):
// fragment loads without bank conflicts, row-wise and transposed.
// ----------------------------------------------------------------------------
__host__ __device__ __forceinline__ int round8(int x) { return (x + 7) & ~7; }

size_t rings_dmma_smem_bytes(int O, int n1, int n2, int q2max)
{
    const size_t N1 = round8(n1), N2 = round8(n2), l1 = N1 + 4, l2 = N2 + 4;
    const size_t nsv = q2max < kVtabSmem ? round8(q2max + 1) : 0;
    const size_t dbl = 2 * N1 * l2 + 2 * N1 * l1 + 3 * (N1 + N2) + nsv;
    return sizeof(double) * dbl + sizeof(int) * ((size_t)O + 4 * (N1 + N2));
}

// Capped at 64 registers (four 256-thread CTAs an SM): a few spill slots, more CTAs resident
// (0.396 -> 0.362 ms per residual on the 100-twist batch, against the 78 registers uncapped).
__global__ void __launch_bounds__(256, 4) k_rings(const RingPairDev *__restrict__ pairs,
                                                        const SolveDev *__restrict__ solves,
                                                        const int16_t *__restrict__ ph_i,
                                                        const int16_t *__restrict__ ph_x,
                                                        const int *__restrict__ nvp,
                                                        const double *__restrict__ vtab,
                                                        const double *__restrict__ xy, int do_ring, int do_xring,
                                                        double *__restrict__ rx,
                                                        const uint8_t *__restrict__ active)
{
    const RingPairDev P = pairs[blockIdx.x];
    if (!active[P.solve]) return;
    const SolveDev s = solves[P.solve];
    const int O = s.O;
    const int n1 = P.n1, n2 = P.n2;
    if (n1 <= 0 || n2 <= 0) return;  // a ring pair always has both groups; whole CTA
    const int N1 = round8(n1), N2 = round8(n2), l1 = N1 + 4, l2 = N2 + 4, R = N1 + N2;
    const bool vsm = s.q2max < kVtabSmem;
    const int nsv = vsm ? round8(s.q2max + 1) : 0;
    extern __shared__ double smem[];
    // W and the direct kernels Vs1, Vs2 are table lookups: generated where the DMMA loops
    // read them (from the rows' n-vectors) instead of stored, for more CTAs per SM
    double *X1 = smem;              // N1 x l2
    double *Y1 = X1 + N1 * l2;      // N1 x l2
    double *XW1 = Y1 + N1 * l2;     // N1 x l1
    double *U1 = XW1 + N1 * l1;     // N1 x l1
    double *Sx = U1 + N1 * l1;      // R: group 1 rows at [0, N1), group 2 rows at [N1, R)
    double *Sy = Sx + R;
    double *Vd = Sy + R;
    double *sv = Vd + R;            // nsv
    int *ri = (int *)(sv + nsv);    // R: occupied index of the row (-1 on padding)
    int *no = ri + R;               // O: packed n-vectors of the occupied orbitals
    int *nx = no + O;               // R: packed n-vector of the row's virtual
    int *nr = nx + R;               // R: packed n-vector of the row's occupied index (0 on padding)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nt = blockDim.x, kWarps = nt >> 5;
    auto V = [&](int q2) -> double {
        return q2 > s.q2max ? 0.0 : (vsm ? sv[q2] : __ldg(&vtab[s.vtab0 + q2]));
    };
    for (int q = tid; q < nsv; q += nt) sv[q] = q <= s.q2max ? vtab[s.vtab0 + q] : 0.0;
    for (int r = tid; r < R; r += nt) {
        int row = -1;
        if (r < n1) row = P.r1 + r;
        else if (r >= N1 && r - N1 < n2) row = P.r2 + (r - N1);
        const int i = row >= 0 ? ph_i[s.phr0 + row] : -1, x = row >= 0 ? ph_x[s.phr0 + row] : -1;
        ri[r] = i;
        nx[r] = x >= 0 ? nvp[s.orb0 + x] : 0;
    }
    for (int k = tid; k < O; k += nt) no[k] = nvp[s.orb0 + k];
    __syncthreads();
    for (int r = tid; r < R; r += nt) nr[r] = ri[r] >= 0 ? no[ri[r]] : 0;
    const int Qp = __vsub4(nx[0], no[ri[0]]);   // Q = n_x - n_i of group 1, packed
    // X1 and Y1: the pair's rows in the particle-hole copy of t (k_ring_stage), 2 N2 doubles
    // a row and 16-byte aligned -- contiguous loads in place of index -> amplitude gathers.
    // Columns n2..N2-1 are zero in memory; rows n1..N1-1 are padding.
    {
        const double2 *src = reinterpret_cast<const double2 *>(xy + P.xy0);
        const int half = N2 / 2;   // double2 per X1 (or Y1) row
        for (int e = tid; e < N1 * N2; e += nt) {
            const int r = e / N2, c2 = e - r * N2;
            const double2 v = r < n1 ? __ldg(&src[(int64_t)r * N2 + c2]) : make_double2(0.0, 0.0);
            double *dst = c2 < half ? X1 + r * l2 + 2 * c2 : Y1 + r * l2 + 2 * (c2 - half);
            dst[0] = v.x;
            dst[1] = v.y;
        }
    }
    __syncthreads();
    // row sums of X1, Y1 for group 1, column sums for group 2 (padding is zero)
    for (int r = tid; r < R; r += nt) {
        double sx = 0.0, sy = 0.0;
        if (r < N1) {
            for (int c = 0; c < n2; c++) {
                sx += X1[r * l2 + c];
                sy += Y1[r * l2 + c];
            }
        } else {
            const int c = r - N1;
            for (int a = 0; a < n1; a++) {
                sx += X1[a * l2 + c];
                sy += Y1[a * l2 + c];
            }
        }
        Sx[r] = sx;
        Sy[r] = sy;
        Vd[r] = ri[r] >= 0 ? V(q2p(no[ri[r]], nx[r])) : 0.0;
    }
    const int g = lane >> 2, tg = lane & 3;
    // phase 1: XW1 = X1 W, U1 = Y1 W - Vs1 (K = N2), with W[b][a] = v(n_{i_b} - n_{i_a} - Q)
    // and Vs1[a][a'] = v(n_{i_a'} - n_{i_a}) generated from the rows' n-vectors (0 on
    // padding).  Tasks: one 8-row fragment row x up to 2 column fragments; X and Y share
    // each generated W fragment.
    {
        const int ngr = (N1 + 15) / 16, ntask = (N1 / 8) * ngr;
        for (int task = warp; task < ntask; task += kWarps) {
            const int mf = task / ngr, ng = task - mf * ngr;
            const double *AX = X1 + (mf * 8 + g) * l2 + tg;
            const double *AY = Y1 + (mf * 8 + g) * l2 + tg;
            const int nbase = ng * 16;
            int cn[2];
            bool cok[2];
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const int n = nbase + f * 8 + g;
                cok[f] = n < n1;
                cn[f] = cok[f] ? __vadd4(nr[n], Qp) : 0;   // n_{i_a'} + Q
            }
            double acc[2][2][2];
#pragma unroll
            for (int f = 0; f < 2; f++) acc[0][f][0] = acc[0][f][1] = acc[1][f][0] = acc[1][f][1] = 0.0;
            for (int k0 = 0; k0 < N2; k0 += 4) {
                const int k = k0 + tg;
                const double ax = AX[k0], ay = AY[k0];
                const bool kok = k < n2;
                const int kn = nr[N1 + k];
#pragma unroll
                for (int f = 0; f < 2; f++) {
                    if (nbase + f * 8 >= N1) break;
                    // B(k = b, n = a') = W[b][a'] = v(n_{i_b} - n_{i_a'} - Q)
                    const double bv = (kok && cok[f]) ? V(q2p(kn, cn[f])) : 0.0;
                    dmma_884(acc[0][f][0], acc[0][f][1], ax, bv);
                    dmma_884(acc[1][f][0], acc[1][f][1], ay, bv);
                }
            }
            const int r = mf * 8 + g;
            const bool rok = r < n1;
            const int rn = rok ? nr[r] : 0;
#pragma unroll
            for (int f = 0; f < 2; f++) {
                if (nbase + f * 8 >= N1) break;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int n = nbase + f * 8 + 2 * tg + h;
                    const double vs = (rok && n < n1) ? V(q2p(nr[n], rn)) : 0.0;
                    XW1[r * l1 + n] = acc[0][f][h];
                    U1[r * l1 + n] = acc[1][f][h] - vs;
                }
            }
        }
    }
    __syncthreads();
    // phase 2: rows a x columns b, tasks of 8 x 16
    const int nng = (N2 + 15) / 16, ntask = (N1 / 8) * nng;
    for (int task = warp; task < ntask; task += kWarps) {
        const int mf = task / nng, ng = task - mf * nng;
        const int m0 = mf * 8;
        double ra[2][2], rb[2][2], xa[2][2], xb[2][2];
#pragma unroll
        for (int f = 0; f < 2; f++)
#pragma unroll
            for (int h = 0; h < 2; h++) ra[f][h] = rb[f][h] = xa[f][h] = xb[f][h] = 0.0;
        // sum over a': A = XW1, U1 rows a; B(k = a', n = b) = X1[a'][b], Y1[a'][b]
        for (int k0 = 0; k0 < N1; k0 += 4) {
            const int k = k0 + tg;
            const double axw = XW1[(m0 + g) * l1 + k], au = U1[(m0 + g) * l1 + k];
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const int n0 = ng * 16 + f * 8;
                if (n0 >= N2) break;
                const double bx = X1[k * l2 + n0 + g], by = Y1[k * l2 + n0 + g];
                dmma_884(ra[f][0], ra[f][1], axw, by - 2.0 * bx);
                dmma_884(rb[f][0], rb[f][1], au, bx);
                dmma_884(xa[f][0], xa[f][1], au, by);
            }
        }
        // sum over b': A = X1, Y1 rows a; B = -Vs2[b][b'], generated
        int bn[2];
        bool bok[2];
#pragma unroll
        for (int f = 0; f < 2; f++) {
            const int bb = ng * 16 + f * 8 + g;
            bok[f] = bb < n2;
            bn[f] = bok[f] ? nr[N1 + bb] : 0;
        }
        for (int k0 = 0; k0 < N2; k0 += 4) {
            const int k = k0 + tg;
            const double ax = X1[(m0 + g) * l2 + k], ay = Y1[(m0 + g) * l2 + k];
            const bool kok = k < n2;
            const int kn = nr[N1 + k];
#pragma unroll
            for (int f = 0; f < 2; f++) {
                const int n0 = ng * 16 + f * 8;
                if (n0 >= N2) break;
                const double bv = (kok && bok[f]) ? -V(q2p(kn, bn[f])) : -0.0;
                dmma_884(rb[f][0], rb[f][1], ax, bv);
                dmma_884(xb[f][0], xb[f][1], ay, bv);
            }
        }
        const int r1 = m0 + g;                          // this lane's row (group 1)
        if (r1 >= n1) continue;
        const double vd = Vd[r1], sx1 = Sx[r1], sy1 = Sy[r1];
        const double base = vd * (2.0 * sx1 - sy1);
        // the ring G of (i_a, i_b, x_a) and the crossed-ring G of (i_a, i_b, x_b) at (a, b) of
        // the pair's rows in rx; k_update picks each amplitude's value there (or its mirror's)
        double *out = rx + P.xy0 + (int64_t)r1 * 2 * N2;
#pragma unroll
        for (int f = 0; f < 2; f++) {
            const int n0 = ng * 16 + f * 8;
            if (n0 >= N2) break;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int n = n0 + 2 * tg + h;
                if (n >= n2) continue;
                const int r2 = N1 + n;
                if (do_ring) {
                    const double lin = 2.0 * vd * (sx1 + Sx[r2]) - vd * (sy1 + Sy[r2]);
                    out[n] = lin + base * (2.0 * Sx[r2] - Sy[r2]) + ra[f][h] + rb[f][h];
                }
                if (do_xring) out[N2 + n] = xa[f][h] + xb[f][h];
            }
        }
    }
}

void set_rings_smem_limit(int wide, size_t bytes)
{
    // keep the largest limit ever requested per kernel: batches of different sizes coexist
    std::lock_guard<std::mutex> lock(g_smem_limit_mu);
    static size_t current_by_dev[kMaxDevices][2] = {};   // attributes are per device
    size_t *current = current_by_dev[current_device() % kMaxDevices];
    if (bytes > current[wide ? 1 : 0]) {
        if (wide) cudaFuncSetAttribute(k_rings_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        else cudaFuncSetAttribute(k_rings, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        current[wide ? 1 : 0] = bytes;
    }
}

size_t rings_smem_bytes(int O, int R)
{
    const int ld = O | 1, lr = R | 1;
    return sizeof(double) * ((size_t)kVtabSmem + 3 * O * ld + 2 * O * lr + 3 * kRingCh * ld + 3 * R) +
           sizeof(int) * 2 * R + 16 + sizeof(int4) * O;
}

// ----------------------------------------------------------------------------
// Fused residual / update / convergence / energy, one thread per amplitude.
//   G = ladders (from k_ladder) + drivers + mosaics + rings + crossed rings
//   R = -G + D t                          (GetRes, CCD.f90:417)
//   t' = (G/D - (1-f) t)/f                (SolveCC, CCD.f90:380)
//   dT = max |t' - t|                     (CnvrgCC, CCD.f90:452-454)
//   E  = sum t' (2 v(i-a) - v(a-j))       (CCEnergy, CCD.f90:225-227 re-indexed)
// mode 0: update (writes t_new, partials e/dT/|R|); mode 1: residual only (|R|).
// ----------------------------------------------------------------------------
struct UpdateArgs {
    const HChunkDev *chunks;
    const SolveDev *solves;
    const AmpInfo *amps;
    const int32_t *partner;
    const int32_t *mirror;
    const int32_t *pos;
    const int4 *nv4;
    const double *eigen;
    const double *vtab;
    const double *t;
    double *t_new;
    const double *g_ladder;
    const double *jvv, *joo;
    const double *J1;             // dRPA ring intermediate
    double *part_e, *part_dt, *part_r;
    double *g_out;            // optional: full G per amplitude (term checks)
    const double *rx;                          // ring and crossed-ring G, particle-hole layout
    const int2 *rpos;                          // where each amplitude's two values sit in it
    const uint8_t *active;
    int do_ladder, do_mosaic, do_ring, do_xring, do_driver, drpa, mode;
    // Pulay DIIS push fused into the update (mode 0, ndiis > 0): the new (t', e) pair
    // goes to the solve's history slot and the chunk partials of e . e_j to dpart
    const IterState *st;
    int ndiis;
    int64_t namp;
    double *hist_t, *dpart;
    float *hist_e;
    const double2 *vcoef;     // per amplitude {v(i-a), v(a-j)}
};

// One CTA per momentum block: for every element (pair r = (i, j), column c = a) the
// amplitude record (i, j, a, b), the position map entry (i, j, a) -> packed index, the
// packed index of the partner (i, j, b), b in column pcol[c] of the same block, and the
// mirror: (j, i, b) in row r + nd + dg for the rows r < nd (i < j); -1 on the diagonal
// pair's row, -2 on the mirror rows.
__global__ void k_block_tables(const BlockDev *__restrict__ blocks, const SolveDev *__restrict__ solves,
                               const int16_t *__restrict__ pair_i, const int16_t *__restrict__ pair_j,
                               const int16_t *__restrict__ vir, const int16_t *__restrict__ pcol,
                               AmpInfo *__restrict__ amps, int32_t *__restrict__ pos, int32_t *__restrict__ partner,
                               int32_t *__restrict__ mirror)
{
    const BlockDev B = blocks[blockIdx.x];
    const SolveDev s = solves[B.solve];
    const int n = B.o * B.v;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int r = e / B.v, c = e - r * B.v;
        const int i = pair_i[B.pair0 + r], j = pair_j[B.pair0 + r];
        const int a = vir[B.vir0 + c], pc = pcol[B.vir0 + c];
        const int64_t p = B.t0 + e;
        amps[p] = AmpInfo{(int16_t)i, (int16_t)j, (int16_t)a, vir[B.vir0 + pc]};
        pos[s.pos0 + ((int64_t)i * s.O + j) * s.V + (a - s.O)] = (int32_t)p;
        partner[p] = (int32_t)(B.t0 + (int64_t)r * B.v + pc);
        const int oc = B.nd + B.dg;
        mirror[p] = r < B.nd ? (int32_t)(B.t0 + (int64_t)(r + oc) * B.v + pc) : r < oc ? -1 : -2;
    }
}

// Ring gather indices per ph row (i, x) and occupied k: t(ik, x) and t(ki, x).
__global__ void k_ring_index(const ChunkDev *__restrict__ rchunks, const SolveDev *__restrict__ solves,
                             const int16_t *__restrict__ ph_i, const int16_t *__restrict__ ph_x,
                             const int32_t *__restrict__ pos, int32_t *__restrict__ ridx_x,
                             int32_t *__restrict__ ridx_y)
{
    const ChunkDev ch = rchunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int e = ch.start + threadIdx.x;
    if (e >= s.O * s.V * s.O) return;
    const int r = e / s.O, k = e - r * s.O;
    const int i = ph_i[s.phr0 + r], x = ph_x[s.phr0 + r];
    ridx_x[s.ph0 + e] = posmap(s, pos, i, k, x);
    ridx_y[s.ph0 + e] = posmap(s, pos, k, i, x);
}

// One CTA per ring pair: where each of its rows (i, x) sits in the particle-hole arrays.
// Group-1 row a: ph_a = xy0 + 2 a N2 (its X1 row; Y1 follows at + N2), ph_b = N2.  Group-2
// row b: ph_a = -1, ph_b = b.  (Rows of groups without a -Q partner keep -1, -1.)
__global__ void k_ph_tables(const RingPairDev *__restrict__ pairs, const SolveDev *__restrict__ solves,
                            const int16_t *__restrict__ ph_i, const int16_t *__restrict__ ph_x,
                            int32_t *__restrict__ ph_a, int32_t *__restrict__ ph_b)
{
    const RingPairDev P = pairs[blockIdx.x];
    const SolveDev s = solves[P.solve];
    const int N2 = (P.n2 + 7) & ~7;
    for (int r = threadIdx.x; r < P.n1 + P.n2; r += blockDim.x) {
        const bool g1 = r < P.n1;
        const int row = g1 ? P.r1 + r : P.r2 + (r - P.n1);
        const int i = ph_i[s.phr0 + row], x = ph_x[s.phr0 + row];
        const int64_t k = s.phr0 + (int64_t)i * s.V + (x - s.O);
        ph_a[k] = g1 ? P.xy0 + 2 * r * N2 : -1;
        ph_b[k] = g1 ? N2 : r - P.n1;
    }
}

// The particle-hole copy of t that k_rings reads, one CTA per {Q, -Q} pair: row a of group
// 1 gets X1[a][c] = t(i_a i_c, x_a) and Y1[a][c] = t(i_c i_a, x_a) for the rows c of group 2,
// through the per-row gather indices (ridx_x, ridx_y).  Each CTA writes its pair's rows
// contiguously; the indexed reads are all this small kernel does, so many of them are in
// flight at once (in k_rings, behind its DMMA phases, they were what the kernel waited on).
__global__ void k_ring_stage(const RingPairDev *__restrict__ pairs, const SolveDev *__restrict__ solves,
                               const int16_t *__restrict__ ph_i, const int32_t *__restrict__ ridx_x,
                               const int32_t *__restrict__ ridx_y, const double *__restrict__ t,
                               double *__restrict__ xy, const uint8_t *__restrict__ active)
{
    const RingPairDev P = pairs[blockIdx.x];
    if (!active[P.solve]) return;
    const SolveDev s = solves[P.solve];
    const int N2 = (P.n2 + 7) & ~7, O = s.O;
    for (int e = threadIdx.x; e < P.n1 * P.n2; e += blockDim.x) {
        const int a = e / P.n2, c = e - a * P.n2;
        const int64_t w = s.ph0 + (int64_t)(P.r1 + a) * O + ph_i[s.phr0 + P.r2 + c];
        const int px = __ldg(&ridx_x[w]), py = __ldg(&ridx_y[w]);
        double *row = xy + P.xy0 + (int64_t)a * 2 * N2;
        row[c] = px >= 0 ? __ldg(&t[px]) : 0.0;
        row[N2 + c] = py >= 0 ? __ldg(&t[py]) : 0.0;
    }
}

// Where k_update finds each amplitude's ring values in rx, once per batch: k_rings leaves at
// (a, b) of a {Q, -Q} pair the ring G of (i_a, i_b, x_a) and the crossed-ring G of
// (i_a, i_b, x_b), a in group 1.  Amplitude (i,j,a) (partner b, i <= j) finds its ring G at
// row (i,a), column (j,b) when (i,a) is in group 1, else at row (j,b), column (i,a) (its
// mirror's place); its crossed-ring G in the second half of row (i,b) at column (j,a), or of
// row (j,a) at column (i,b).
__global__ void k_rx_pos(const HChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                         const AmpInfo *__restrict__ amps, const int32_t *__restrict__ ph_a,
                         const int32_t *__restrict__ ph_b, int2 *__restrict__ rpos)
{
    const HChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= ch.end) return;
    const int64_t p = s.amp0 + loc;
    const AmpInfo q = amps[p];
    const int V = s.V, O = s.O;
    const int32_t *pa = ph_a + s.phr0, *pb = ph_b + s.phr0;
    const int ia = q.i * V + q.a - O, jb = q.j * V + q.b - O, ib = q.i * V + q.b - O, ja = q.j * V + q.a - O;
    const int r = pa[ia] >= 0 ? pa[ia] + pb[jb] : pa[jb] + pb[ia];
    const int x = pa[ib] >= 0 ? pa[ib] + pb[ib] + pb[ja] : pa[ja] + pb[ja] + pb[ib];
    rpos[p] = make_int2(r, x);
}

void launch_block_tables(const DevBatch &d, cudaStream_t st)
{
    if (d.nblocks > 0)
        k_block_tables<<<d.nblocks, 256, 0, st>>>(d.blocks, d.solves, d.pair_i, d.pair_j, d.vir, d.pcol, d.amps,
                                                  d.pos, d.partner, d.mirror);
    if (d.nrpairs > 0) k_ph_tables<<<d.nrpairs, 128, 0, st>>>(d.rpairs, d.solves, d.ph_i, d.ph_x, d.ph_a, d.ph_b);
    if (d.nrpairs > 0 && d.nhchunks > 0)
        k_rx_pos<<<d.nhchunks, kChunk, 0, st>>>(d.hchunks, d.solves, d.amps, d.ph_a, d.ph_b, d.rpos);
    if (d.nrchunks > 0)
        k_ring_index<<<d.nrchunks, kChunk, 0, st>>>(d.rchunks, d.solves, d.ph_i, d.ph_x, d.pos, d.ridx_x,
                                                    d.ridx_y);
}

// Static per-amplitude Coulomb factors of the update: {v(i-a), v(a-j)}.
__global__ void k_vcoef(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                        const AmpInfo *__restrict__ amps, const int4 *__restrict__ nv4,
                        const double *__restrict__ vtab, double2 *__restrict__ vcoef)
{
    const ChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= s.namp) return;
    const int64_t p = s.amp0 + loc;
    const AmpInfo q = amps[p];
    vcoef[p] = make_double2(vpq(s, nv4, vtab, q.i, q.a), vpq(s, nv4, vtab, q.a, q.j));
}

void launch_vcoef(const DevBatch &d, cudaStream_t st)
{
    k_vcoef<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.amps, d.nv4, d.vtab, d.vcoef);
}

// Eight CTAs per SM (32 registers, a few spilled): the kernel waits on scattered loads, and
// full occupancy hides them better than the spills cost (0.70 -> 0.50 ms per residual at
// 100 twists of N=54, against the 64-register form).
__global__ void __launch_bounds__(kChunk, 8) k_update(UpdateArgs A)
{
    const HChunkDev ch = A.chunks[blockIdx.x];
    double esum = 0.0, dtmax = 0.0, rmax = 0.0;
    const bool on = A.active[ch.solve];
    const SolveDev s = A.solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    // The chunks cover the amplitudes i <= j only: by the pair symmetry t(ij,a) = t(ji,b)
    // each amplitude with i < j also updates its mirror (j,i,b); every term of G shares the
    // symmetry.
    const bool valid = loc < ch.end;
    const int32_t mirv = valid ? A.mirror[s.amp0 + loc] : -2;
    if (!on && A.mode == 0 && valid) {
        A.t_new[s.amp0 + loc] = A.t[s.amp0 + loc];
        if (mirv >= 0) A.t_new[mirv] = A.t[mirv];
    }
    const int32_t mir = on ? mirv : -2;
    const double wgt = mir >= 0 ? 2.0 : 1.0;   // energy and DIIS dot weight: this amplitude and its mirror
    if (mir != -2) {
        const int64_t p = s.amp0 + loc;
        const AmpInfo q = A.amps[p];
        const int i = q.i, j = q.j, a = q.a, b = q.b;
        const int O = s.O;
        const double told = A.t[p];
        const double2 vc = A.vcoef[p];
        const double via = vc.x;
        double g = A.do_ladder ? A.g_ladder[p] : 0.0;
        if (A.do_driver) g += via;  // GetG2Drivers: G2abab = V(n_i - n_a)
        if (A.do_mosaic)
            g -= 0.5 * (A.jvv[s.jvv0 + a - O] + A.jvv[s.jvv0 + b - O] + A.joo[s.joo0 + i] + A.joo[s.joo0 + j]) * told;
        if (A.drpa) {
            if (A.do_ring) {
                // linear (dRPA.f90:476-513): 2 v(i-a) sum_k t(ik,a) + 2 v(j-b) sum_k t(jk,b)
                double s1 = 0.0, s2 = 0.0;
                for (int k = 0; k < O; k++) {
                    int p1 = posmap(s, A.pos, i, k, a);
                    if (p1 >= 0) s1 += A.t[p1];
                    int p2 = posmap(s, A.pos, j, k, b);
                    if (p2 >= 0) s2 += A.t[p2];
                }
                g += 2.0 * via * s1 + 2.0 * vpq(s, A.nv4, A.vtab, j, b) * s2;
                // quadratic (dRPA.f90:539-545): sum_l 2 J(i,a,l) t(lj,d), d = n_l + n_a - n_i
                const double *Jr = A.J1 + s.ph0 + ((int64_t)i * s.V + (a - O)) * O;
                for (int l = 0; l < O; l++) {
                    int pb = posmap(s, A.pos, l, j, b);  // exists iff d is a virtual
                    if (pb < 0) continue;
                    g += 2.0 * Jr[l] * A.t[A.partner[pb]];
                }
            }
        } else if (A.do_ring || A.do_xring) {
            // the ring G (rings, linear + quadratic, CCD.f90:716-811) and the crossed-ring G
            // (CCD.f90:845-937) of this amplitude, where k_rings left them (k_rx_pos)
            const int2 ro = A.rpos[p];
            if (A.do_ring) g += A.rx[ro.x];
            if (A.do_xring) g += A.rx[ro.y];
        }
        {   // core pair: every term has a zero factor (CoreN read on its own: taken from the
            // solve record above, it costs this kernel registers)
            const int cn = __ldg(&A.solves[ch.solve].core_n);
            if (i < cn || j < cn) g = 0.0;
        }
        if (A.g_out) {
            A.g_out[p] = g;
            if (mir >= 0) A.g_out[mir] = g;
        }
        const double *ev = A.eigen + s.orb0;
        const double denom = ev[i] + ev[j] - ev[a] - ev[b];
        const double r = -g + denom * told;
        rmax = fabs(r);
        if (A.mode == 0) {
            const double f = s.denom_factor;
            const double tn = (g / denom - (1.0 - f) * told) / f;
            if (A.ndiis == 0) {  // with DIIS the history slot holds t'
                A.t_new[p] = tn;
                if (mir >= 0) A.t_new[mir] = tn;
            }
            dtmax = fabs(tn - told);
            if (A.drpa) esum = via * tn * 2.0;  // SOSEX part added by k_drpa_energy at the end
            else esum = tn * (2.0 * via - vc.y);
            esum *= wgt;
            if (!(fabs(tn) < 1e300)) dtmax = __longlong_as_double(0x7ff0000000000000LL);  // +Inf marks NaN/Inf
            if (A.ndiis > 0) {
                const int slot = (A.st[ch.solve].niter - 1) % A.ndiis;
                const float e = (float)(tn - told);
                // the mirrors' history entries are never read: k_diis_extrap2 and the dot
                // products go through the amplitudes i <= j
                A.hist_t[(int64_t)slot * A.namp + p] = tn;
                A.hist_e[(int64_t)slot * A.namp + p] = e;
            }
        }
    }
    if (A.mode == 0 && A.ndiis > 0 && on) {
        // e . e_j of every stored j (the chunk belongs to one solve: the loop is uniform)
        const int nb = A.st[ch.solve].niter;
        const int slot = (nb - 1) % A.ndiis, nvec = min(nb, A.ndiis);
        const bool mine = mir != -2;   // the mirrors count through their pair (weight 2)
        const int64_t p = s.amp0 + loc;
        const double e0 = mine ? (double)A.hist_e[(int64_t)slot * A.namp + p] : 0.0, e = wgt * e0;
        __shared__ double sd[kChunk / 32][kDiisMax];
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        for (int jv = 0; jv < nvec; jv++) {
            double d = mine ? e * (jv == slot ? e0 : (double)A.hist_e[(int64_t)jv * A.namp + p]) : 0.0;
            for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
            if (l == 0) sd[w][jv] = d;
        }
        __syncthreads();
        if (threadIdx.x < nvec) {
            double d = 0.0;
            for (int k = 0; k < kChunk / 32; k++) d += sd[k][threadIdx.x];
            A.dpart[(int64_t)blockIdx.x * kDiisMax + threadIdx.x] = d;
        }
    }
    block_reduce3<kChunk>(esum, dtmax, rmax);
    if (threadIdx.x == 0) {
        A.part_e[blockIdx.x] = esum;
        A.part_dt[blockIdx.x] = dtmax;
        A.part_r[blockIdx.x] = rmax;
    }
}

// ----------------------------------------------------------------------------
// Pulay DIIS (new in this library; the reference's GetTFromDIIS, DIISCC.f90:52-131,
// builds a singular matrix and never extrapolates).  Error vector e = t' - t of
// the (damped) Jacobi step; history of ndiis (t', e) pairs per solve.
// k_update stores the solve's current slot and forms the dot products e . e_j of
// every stored j (per-chunk partials); k_diis_rows2 reduces them per solve in chunk order.
// ----------------------------------------------------------------------------
constexpr int kMaxDiis = 16;
// ----------------------------------------------------------------------------
// Device-side iteration control.  Every solve of a batch carries its own state;
// one iteration is a fixed sequence of launches (residual terms -> update ->
// per-solve reduction -> [DIIS push] -> k_control -> commit -> k_active_swap),
// so it can be captured once as a CUDA graph and replayed.  Converged solves stop
// being updated (their CTAs return at once) while the others continue.
// ----------------------------------------------------------------------------
// Pulay system [B 1; 1 0][c; l] = [0; 1] over nvec vectors, B scaled by its max
// diagonal; Gaussian elimination with partial pivoting.  Returns false if singular.
__device__ bool pulay_device(const double *B, int nvec, double *c)
{
    constexpr int N = kMaxDiis + 1;
    double A[N][N + 1];
    const int n = nvec + 1;
    double scale = 0.0;
    for (int j = 0; j < nvec; j++) scale = fmax(scale, B[j * kMaxDiis + j]);
    if (!(scale > 0.0) || !isfinite(scale)) return false;
    for (int j = 0; j < n; j++)
        for (int k = 0; k <= n; k++) A[j][k] = 0.0;
    for (int j = 0; j < nvec; j++) {
        for (int k = 0; k < nvec; k++) A[j][k] = B[j * kMaxDiis + k] / scale;
        A[j][nvec] = 1.0;
        A[nvec][j] = 1.0;
    }
    A[nvec][n] = 1.0;
    for (int k = 0; k < n; k++) {
        int piv = k;
        for (int i = k + 1; i < n; i++)
            if (fabs(A[i][k]) > fabs(A[piv][k])) piv = i;
        if (fabs(A[piv][k]) < 1e-14) return false;
        if (piv != k)
            for (int j = 0; j <= n; j++) {
                double tmp = A[k][j];
                A[k][j] = A[piv][j];
                A[piv][j] = tmp;
            }
        for (int i = k + 1; i < n; i++) {
            const double f = A[i][k] / A[k][k];
            for (int j = k; j <= n; j++) A[i][j] -= f * A[k][j];
        }
    }
    for (int k = n - 1; k >= 0; k--) {
        double x = A[k][n];
        for (int j = k + 1; j < n; j++) x -= A[k][j] * A[j][n];
        A[k][n] = x / A[k][k];
    }
    for (int j = 0; j < nvec; j++) {
        if (!isfinite(A[j][n])) return false;
        c[j] = A[j][n];
    }
    return true;
}

// One thread per solve.  init = 1: record the start energy and decide whether to iterate.
__global__ void k_control(int nsolves, const double *__restrict__ red, const double *__restrict__ brow,
                          IterState *__restrict__ st, double *__restrict__ Bm, double *__restrict__ coef,
                          double *__restrict__ rec_e, double *__restrict__ rec_dt, int max_rec,
                          const uint8_t *__restrict__ active, uint8_t *__restrict__ active_next, double tol,
                          int max_iter, int ndiis, int init)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsolves) return;
    IterState S = st[s];
    if (!init && !active[s]) {
        active_next[s] = 0;
        return;
    }
    const double e = red[3 * s], dt = red[3 * s + 1];
    if (!init) S.niter += 1;
    const int r = S.niter - 1;
    if (r >= 0 && r < max_rec) {
        rec_e[(int64_t)s * max_rec + r] = e;
        rec_dt[(int64_t)s * max_rec + r] = dt;
    }
    S.e = e;
    S.dt = dt;
    const bool finite = isfinite(e) && isfinite(dt);
    const bool go = finite && dt >= tol && S.niter < max_iter;
    if (!finite) S.status = 3;
    if (!init && ndiis > 0) {
        // this iteration pushed slot (niter_before - 1) % ndiis with nvec = min(niter_before, ndiis)
        const int nb = S.niter - 1;
        const int slot = (nb - 1) % ndiis, nvec = min(nb, ndiis);
        double *B = Bm + (int64_t)s * kMaxDiis * kMaxDiis;
        for (int j = 0; j < nvec; j++) B[slot * kMaxDiis + j] = B[j * kMaxDiis + slot] = brow[s * kMaxDiis + j];
        double *c = coef + s * kMaxDiis;
        for (int j = 0; j < kMaxDiis; j++) c[j] = 0.0;
        if (!go || nvec < 2 || !pulay_device(B, nvec, c)) {
            for (int j = 0; j < kMaxDiis; j++) c[j] = 0.0;
            c[slot] = 1.0;
        }
    }
    if (!go && S.status == 0) S.status = (finite && dt >= tol) ? 2 : 1;
    active_next[s] = go ? 1 : 0;
    st[s] = S;
}

// active <- active_next; count of active solves for the host's poll.
__global__ void k_active_swap(int nsolves, uint8_t *__restrict__ active, const uint8_t *__restrict__ active_next,
                              int *__restrict__ count)
{
    int c = 0;
    for (int s = threadIdx.x; s < nsolves; s += blockDim.x) {
        const uint8_t a = active_next[s];
        active[s] = a;
        c += a;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ int w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += w[k];
        *count = tot;
    }
}

// t <- t_new for the solves still iterating this round (replay mode)
__global__ void k_commit(const HChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                         const int32_t *__restrict__ mirror, const double *__restrict__ t_new,
                         double *__restrict__ t, const uint8_t *__restrict__ active)
{
    const HChunkDev ch = chunks[blockIdx.x];
    if (!active[ch.solve]) return;
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= ch.end) return;
    const int64_t p = s.amp0 + loc;
    const double x = t_new[p];
    t[p] = x;
    const int32_t mir = mirror[p];
    if (mir >= 0) t[mir] = x;
}

__global__ void k_diis_rows2(const int *__restrict__ chunk_begin, const IterState *__restrict__ st, int ndiis,
                             const double *__restrict__ part, double *__restrict__ brow,
                             const uint8_t *__restrict__ active)
{
    const int s = blockIdx.x;
    if (!active[s]) return;
    const int nvec = min(st[s].niter, ndiis);
    const int c0 = chunk_begin[s], c1 = chunk_begin[s + 1];
    for (int jv = 0; jv < nvec; jv++) {
        double acc = 0.0;
        for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) acc += part[(int64_t)c * kMaxDiis + jv];
        acc = block_sum<256>(acc);
        if (threadIdx.x == 0) brow[s * kMaxDiis + jv] = acc;
        __syncthreads();
    }
}

// t = sum_j c_j t'_j over the amplitudes i <= j, each also written to its mirror (j,i,b)
__global__ void k_diis_extrap2(const HChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                               int64_t namp, const double *__restrict__ hist_t, const double *__restrict__ coef,
                               int ndiis, const int32_t *__restrict__ mirror, double *__restrict__ t,
                               const uint8_t *__restrict__ active)
{
    const HChunkDev ch = chunks[blockIdx.x];
    if (!active[ch.solve]) return;
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= ch.end) return;
    const int64_t p = s.amp0 + loc;
    const int32_t mir = mirror[p];
    const double *c = coef + ch.solve * kMaxDiis;
    double x = 0.0;
    for (int jv = 0; jv < ndiis; jv++) {
        const double cj = c[jv];
        if (cj != 0.0) x = fma(cj, hist_t[(int64_t)jv * namp + p], x);
    }
    t[p] = x;
    if (mir >= 0) t[mir] = x;
}

__global__ void k_copy(int64_t n, const double *__restrict__ src, double *__restrict__ dst)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) dst[p] = src[p];
}

void launch_refresh(const DevBatch &d, cudaStream_t st)
{
    k_copy<<<(unsigned)((d.namp + 255) / 256), 256, 0, st>>>(d.namp, d.t, d.t_ref);
    launch_ladder3(d, d.tiles, d.ntile_cls, d.t_ref, 0, 1, 0, d.g_ref, st);
}

void launch_control(const DevBatch &d, const CtlBuffers &c, double tol, int max_iter, int ndiis, int init,
                    cudaStream_t st)
{
    k_control<<<(d.nsolves + 127) / 128, 128, 0, st>>>(d.nsolves, d.red, c.brow, c.state, c.Bm, c.coef, c.rec_e,
                                                       c.rec_dt, c.max_rec, d.active, c.active_next, tol,
                                                       max_iter, ndiis, init);
}

void launch_active_swap(const DevBatch &d, const CtlBuffers &c, cudaStream_t st)
{
    k_active_swap<<<1, 1024, 0, st>>>(d.nsolves, d.active, c.active_next, c.count);
}

// One iteration: residual + update, reduction, [DIIS], control, commit, swap.  Returns launches.
int launch_iteration(const DevBatch &d, const CtlBuffers &c, const TermFlags &f, double tol, int max_iter,
                     int ndiis, cudaStream_t st, KernelTimer *kt)
{
    // the DIIS push (history slot and e . e_j partials) happens inside k_update
    int n = launch_residual(d, f, 0, nullptr, st, kt, &c, ndiis);
    if (ndiis > 0) {
        k_diis_rows2<<<d.nsolves, 256, 0, st>>>(d.hchunk_begin, c.state, ndiis, c.part, c.brow, d.active);
        n += 1;
    }
    launch_control(d, c, tol, max_iter, ndiis, 0, st);
    if (ndiis > 0)
        k_diis_extrap2<<<d.nhchunks, kChunk, 0, st>>>(d.hchunks, d.solves, d.namp, c.hist_t, c.coef, ndiis, d.mirror,
                                                     d.t, d.active);
    else
        k_commit<<<d.nhchunks, kChunk, 0, st>>>(d.hchunks, d.solves, d.mirror, d.t_new, d.t, d.active);
    launch_active_swap(d, c, st);
    return n + 3;
}

// ----------------------------------------------------------------------------
// Layout conversion between the packed amplitudes and the reference's
// T(NOcc,NOcc,NOcc+1:NAO) column-major arrays (one solve).
// ----------------------------------------------------------------------------
__global__ void k_pack(const SolveDev *__restrict__ solves, int sidx, const AmpInfo *__restrict__ amps,
                       const double *__restrict__ dense, double *__restrict__ t)
{
    const SolveDev s = solves[sidx];
    int loc = blockIdx.x * blockDim.x + threadIdx.x;
    if (loc >= s.namp) return;
    int64_t p = s.amp0 + loc;
    AmpInfo q = amps[p];
    // core pairs are held at zero (their integrals are zero; see uegccd_internal.h)
    t[p] = (q.i < s.core_n || q.j < s.core_n) ? 0.0 : dense[q.i + (int64_t)s.O * q.j + (int64_t)s.O * s.O * (q.a - s.O)];
}

// writes T2abab, T2abba = -t(ij,b), T2aaaa = t(ij,a) - t(ij,b) (any may be null);
// the dense arrays must be zeroed before (entries of forbidden (i,j,a) stay 0).
__global__ void k_unpack(const SolveDev *__restrict__ solves, int sidx, const AmpInfo *__restrict__ amps,
                         const int32_t *__restrict__ partner, const double *__restrict__ t,
                         double *__restrict__ d_abab, double *__restrict__ d_abba, double *__restrict__ d_aaaa)
{
    const SolveDev s = solves[sidx];
    int loc = blockIdx.x * blockDim.x + threadIdx.x;
    if (loc >= s.namp) return;
    int64_t p = s.amp0 + loc;
    AmpInfo q = amps[p];
    int64_t x = q.i + (int64_t)s.O * q.j + (int64_t)s.O * s.O * (q.a - s.O);
    double ta = t[p], tb = t[partner[p]];
    if (d_abab) d_abab[x] = ta;
    if (d_abba) d_abba[x] = -tb;
    if (d_aaaa) d_aaaa[x] = ta + (-tb);
}

// T2abab of every solve in the reference layout, solve after solve (dense_off[s]).
__global__ void k_unpack_all(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                             const int64_t *__restrict__ dense_off, const AmpInfo *__restrict__ amps,
                             const double *__restrict__ t, double *__restrict__ out)
{
    const ChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= s.namp) return;
    const int64_t p = s.amp0 + loc;
    const AmpInfo q = amps[p];
    out[dense_off[ch.solve] + q.i + (int64_t)s.O * q.j + (int64_t)s.O * s.O * (q.a - s.O)] = t[p];
}

void launch_unpack_all(const DevBatch &d, const int64_t *dense_off, const double *t, double *out, cudaStream_t st)
{
    k_unpack_all<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, dense_off, d.amps, t, out);
}

// ----------------------------------------------------------------------------
// Structure factors on the momentum-transfer grid (CCEnergyAndSF, CCD.f90:290-331;
// DrvMBPT, MP2.f90:86-95).  For every stored (i,j,a) the reference adds
//   at q = n_a - n_i:  SfSum += T2aaaa + T2abab,  SfDSum += 2 T2abab,  SfXSum += T2aaaa - T2abab
//   at q = n_a - n_j:  SfSum -= T2aaaa + T2abba,  SfDSum -= 2 T2abba,  SfXSum -= T2aaaa - T2abba
// with T2abba(i,j,a) = -t(ij,b) and T2aaaa = T2abab + T2abba (CCD.f90:90).
// Particle-hole row (i,x) of group Q = n_x - n_i, with occupied k, holds the direct
// transfer of t(ik,x) and the exchange transfer of t(ki,x): every contribution to grid
// point Q comes from the rows of group Q.  One CTA per group therefore owns its grid
// point and writes it without atomics, summing in a fixed order.
// ----------------------------------------------------------------------------
constexpr int kSfThreads = 128;

__global__ void __launch_bounds__(kSfThreads)
    k_sf(const int2 *__restrict__ groups, const SolveDev *__restrict__ solves, int solve,
         const int16_t *__restrict__ ph_i, const int16_t *__restrict__ ph_x, const int4 *__restrict__ nv4,
         const int32_t *__restrict__ ridx_x, const int32_t *__restrict__ ridx_y,
         const int32_t *__restrict__ partner, const double *__restrict__ t, int S, double *__restrict__ grid,
         int *__restrict__ err)
{
    const int2 G = groups[blockIdx.x];   // rows [G.x, G.x + G.y) of the solve
    const SolveDev s = solves[solve];
    const int O = s.O, V = s.V;
    double sum = 0.0, dsum = 0.0, xsum = 0.0, cnt = 0.0;
    // position of the last contribution in the reference's loop order (I, J, A, then
    // direct before exchange): its SfV assignment is the one that stays
    long long last = -1;
    const int n = G.y * O;
    for (int e = threadIdx.x; e < n; e += kSfThreads) {
        const int r = G.x + e / O, k = e - (e / O) * O;
        const int64_t ri = s.ph0 + (int64_t)r * O + k;
        const int ir = ph_i[s.phr0 + r], xr = ph_x[s.phr0 + r] - O;
        const int pd = __ldg(&ridx_x[ri]);
        if (pd >= 0) {  // direct: (I,J,A) = (i,k,x)
            const double tab = __ldg(&t[pd]), tba = -__ldg(&t[__ldg(&partner[pd])]);
            const double taa = tab + tba;
            sum += taa + tab;
            dsum += 2.0 * tab;
            xsum += taa - tab;
            cnt += 1.0;
            last = max(last, (((long long)ir * O + k) * V + xr) * 2);
        }
        const int px = __ldg(&ridx_y[ri]);
        if (px >= 0) {  // exchange: (I,J,A) = (k,i,x)
            const double tab = __ldg(&t[px]), tba = -__ldg(&t[__ldg(&partner[px])]);
            const double taa = tab + tba;
            sum -= taa + tba;
            dsum -= 2.0 * tba;
            xsum -= taa - tba;
            cnt += 1.0;
            last = max(last, (((long long)k * O + ir) * V + xr) * 2 + 1);
        }
    }
    __shared__ double red[4][kSfThreads / 32];
    __shared__ long long red_last[kSfThreads / 32];
    double v[4] = {sum, dsum, xsum, cnt};
#pragma unroll
    for (int q = 0; q < 4; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    for (int o = 16; o > 0; o >>= 1) last = max(last, __shfl_down_sync(0xffffffffu, last, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int q = 0; q < 4; q++) red[q][w] = v[q];
        red_last[w] = last;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double tot[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        tot[q] = red[q][0];
        for (int k = 1; k < kSfThreads / 32; k++) tot[q] += red[q][k];
    }
    for (int k = 1; k < kSfThreads / 32; k++) last = max(last, red_last[k]);
    last = max(last, red_last[0]);
    if (tot[3] == 0.0) return;   // no stored amplitude reaches this transfer
    // the last tuple (I,J): a core pair leaves SfV = 0 (its integral is zero under CoreN)
    const long long ij = (last >> 1) / V;
    const bool last_core = (int)(ij / O) < s.core_n || (int)(ij % O) < s.core_n;
    const int i = ph_i[s.phr0 + G.x], x = ph_x[s.phr0 + G.x];
    const int4 a = nv4[s.orb0 + x], b = nv4[s.orb0 + i];
    const int q0 = a.x - b.x, q1 = a.y - b.y, q2 = a.z - b.z;
    if (q0 < -S || q0 > S || q1 < -S || q1 > S || q2 < -S || q2 > S) {
        atomicExch(err, 1);
        return;
    }
    const int64_t W = 2 * S + 1, W3 = W * W * W;
    const int64_t c = (q0 + S) + W * ((q1 + S) + W * (int64_t)(q2 + S));
    grid[c] = tot[0];
    grid[W3 + c] = tot[1];
    grid[2 * W3 + c] = tot[2];
    grid[3 * W3 + c] = tot[3];
    grid[4 * W3 + c] = last_core ? 1.0 : 0.0;
}

void launch_sf(const DevBatch &d, const int2 *groups, int ngroups, int solve, int S, double *grid, int *err,
               cudaStream_t st)
{
    if (ngroups > 0)
        k_sf<<<ngroups, kSfThreads, 0, st>>>(groups, d.solves, solve, d.ph_i, d.ph_x, d.nv4, d.ridx_x, d.ridx_y,
                                            d.partner, d.t, S, grid, err);
}

// ----------------------------------------------------------------------------
// Launch wrappers
// ----------------------------------------------------------------------------
void launch_mp2(const DevBatch &d, cudaStream_t st)
{
    k_mp2<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.amps, d.vcoef, d.eigen, d.t, d.part_e, d.part_dt,
                                        d.part_r);
}

void launch_reduce(const DevBatch &d, cudaStream_t st)
{
    k_reduce_solves<<<d.nsolves, 256, 0, st>>>(d.chunk_begin, d.part_e, d.part_dt, d.part_r, d.red);
}

void launch_energy(const DevBatch &d, int kind, double csosex, cudaStream_t st)
{
    k_energy<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.vcoef, d.t, kind, csosex, d.part_e, d.part_dt,
                                           d.part_r);
}

void launch_to_aaaa(const DevBatch &d, cudaStream_t st)
{
    k_to_aaaa<<<(unsigned)((d.namp + 255) / 256), 256, 0, st>>>(d.namp, d.partner, d.t, d.t_new);
}

const char *kKernelNames[KID_COUNT] = {"k_mp2",      "k_energy",   "k_ladder_hh", "k_ladder",
                                      "k_mosaic_blk", "k_mosaic_sum", "k_ring_int", "k_update",
                                      "k_reduce_solves", "k_rings",
                                      "k_ladder_tc", "k_ring_stage"};

int tune_rings(DevBatch &d, cudaStream_t st)
{
    static const int kCand[] = {32, 64, 128, 256};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    int off = 0;
    for (int c = 0; c < kRingClasses && err == cudaSuccess; c++) {
        if (d.nring[c] > 0) {
            float best = 1e30f;
            int pick = d.ring_threads[c];
            for (int th : kCand) {
                auto run = [&]() {
                    k_rings<<<d.nring[c], th, d.ring_smem[c], st>>>(d.rpairs + off, d.solves, d.ph_i, d.ph_x,
                                                                    d.nvp, d.vtab, d.xy, 1, 1, d.rx, d.active);
                };
                run();  // warm
                cudaEventRecord(e0, st);
                run();
                run();
                cudaEventRecord(e1, st);
                if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) {
                    best = ms;
                    pick = th;
                }
            }
            d.ring_threads[c] = pick;
        }
        off += d.nring[c];
    }
    // the staging kernel's CTA size
    if (err == cudaSuccess && d.nrpairs > 0) {
        float best = 1e30f;
        for (int th : {64, 128, 256}) {
            auto run = [&]() {
                k_ring_stage<<<d.nrpairs, th, 0, st>>>(d.spairs, d.solves, d.ph_i, d.ridx_x, d.ridx_y, d.t, d.xy,
                                                       d.active);
            };
            run();
            cudaEventRecord(e0, st);
            run();
            run();
            cudaEventRecord(e1, st);
            if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                d.stage_threads = th;
            }
        }
    }
    // the ladder tiles' order (particle-particle part alone; it writes only d.g)
    if (err == cudaSuccess && d.nblocks > 0 && d.tiles_lpt) {
        float best = 1e30f;
        for (int sched = 0; sched < 2 && err == cudaSuccess; sched++) {
            const LadderTile *tl = sched ? d.tiles_lpt : d.tiles;
            launch_ladder3(d, tl, d.ntile_cls, d.t, 0, 1, 0, d.g, st);
            cudaEventRecord(e0, st);
            launch_ladder3(d, tl, d.ntile_cls, d.t, 0, 1, 0, d.g, st);
            launch_ladder3(d, tl, d.ntile_cls, d.t, 0, 1, 0, d.g, st);
            cudaEventRecord(e1, st);
            if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                d.ladder_sched = sched;
            }
        }
    }
    // the hole-hole intermediate's column chunk (mode 1 alone; it writes only d.hh)
    if (err == cudaSuccess && d.nblocks > 0) {
        float best = 1e30f;
        int pick = 64;
        const LadderTile *tl = d.ladder_sched ? d.htiles_lpt : d.htiles;
        for (int kc : {64, 32}) {
            d.hh_kc = kc;
            launch_ladder3(d, tl, d.nhtile_cls, d.t, 1, 1, 1, d.g, st);
            cudaEventRecord(e0, st);
            launch_ladder3(d, tl, d.nhtile_cls, d.t, 1, 1, 1, d.g, st);
            launch_ladder3(d, tl, d.nhtile_cls, d.t, 1, 1, 1, d.g, st);
            cudaEventRecord(e1, st);
            if ((err = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                pick = kc;
            }
        }
        d.hh_kc = pick;
    }
    if (err == cudaSuccess) err = cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return (int)err;
}

int launch_residual(const DevBatch &d, const TermFlags &f, int mode, double *g_out, cudaStream_t st,
                    KernelTimer *kt, const CtlBuffers *diis, int ndiis)
{
    KernelTimer dummy;
    if (!kt) kt = &dummy;
    int n = 0;
    if (f.do_ladder && d.nblocks > 0) {
        if (f.do_hh) {
            kt->begin(KID_HH_W, st);
            n += launch_ladder3(d, d.ladder_sched ? d.htiles_lpt : d.htiles, d.nhtile_cls, d.t, 1, f.do_pp, f.do_hh,
                                d.g, st);
            kt->end(st);
        }
        const int pp64 = (f.do_pp && !f.mixed) ? 1 : 0;
        kt->begin(KID_LADDER, st);
        n += launch_ladder3(d, d.ladder_sched ? d.tiles_lpt : d.tiles, d.ntile_cls, d.t, 0, pp64, f.do_hh, d.g, st);
        kt->end(st);
        if (f.do_pp && f.mixed) {
            kt->begin(KID_LADDER_TC, st);
            launch_ladder_tc(d, d.t_ref, d.g_ref, d.tc_err, st);
            kt->end(st);
            n += (d.ntc16 > 0) + (d.ntc32 > 0) + (d.ntc64 > 0);
        }
    }
    if (f.do_mosaic) {
        kt->begin(KID_MOSAIC_S, st);
        k_mosaic_blk<<<d.nblocks, kMosThreads, d.mosaic_smem, st>>>(d.blocks, d.solves, d.pair_i, d.pair_j, d.vir,
                                                                   d.nvp, d.vtab, d.t, d.pcol, f.drpa, d.mpart,
                                                                   d.active, d.mosaic_vt);
        kt->end(st);
        kt->begin(KID_MOSAIC_RED, st);
        k_mosaic_sum<<<(d.ntargets + 7) / 8, 256, 0, st>>>(d.targets, d.ntargets, d.solves, d.mt_start, d.mt_list,
                                                           d.mpart, d.jvv, d.joo, d.active);
        kt->end(st);
        n += 2;
    }
    if ((f.do_ring || f.do_xring) && f.drpa) {
        kt->begin(KID_RING_INT, st);
        k_ring_int<<<d.nrchunks, kChunk, 0, st>>>(d.rchunks, d.solves, d.pos, d.nv4, d.vtab, d.t, d.J1, d.active);
        kt->end(st);
        n++;
    }
    if ((f.do_ring || f.do_xring) && !f.drpa) {
        kt->begin(KID_RING_STAGE, st);
        k_ring_stage<<<d.nrpairs, d.stage_threads, 0, st>>>(d.spairs, d.solves, d.ph_i, d.ridx_x, d.ridx_y, d.t, d.xy,
                                                            d.active);
        kt->end(st);
        n++;
        kt->begin(KID_RINGS, st);
        // pair classes (sorted in this order): DMMA tiles in two shared-memory sizes, then the FMA form
        int off = 0;
        for (int c = 0; c < kRingClasses; c++) {
            if (d.nring[c] > 0) {
                k_rings<<<d.nring[c], d.ring_threads[c], d.ring_smem[c], st>>>(
                    d.rpairs + off, d.solves, d.ph_i, d.ph_x, d.nvp, d.vtab, d.xy, f.do_ring, f.do_xring, d.rx,
                    d.active);
                n++;
            }
            off += d.nring[c];
        }
        if (d.nring[kRingClasses] > 0) {
            k_rings_wide<<<d.nring[kRingClasses], 256, d.ring_smem[kRingClasses], st>>>(d.rpairs + off, d.solves, d.ph_i, d.ph_x, d.pos,
                                                                 d.partner, d.nv4, d.vtab, d.t, f.do_ring,
                                                                 f.do_xring, d.rx, d.active);
            n++;
        }
        kt->end(st);
    }
    UpdateArgs A;
    A.chunks = d.hchunks; A.solves = d.solves; A.amps = d.amps; A.partner = d.partner; A.mirror = d.mirror; A.pos = d.pos;
    A.nv4 = d.nv4; A.eigen = d.eigen; A.vtab = d.vtab; A.t = d.t; A.t_new = d.t_new; A.g_ladder = d.g;
    A.jvv = d.jvv; A.joo = d.joo; A.J1 = d.J1;
    A.part_e = d.part_e; A.part_dt = d.part_dt; A.part_r = d.part_r; A.g_out = g_out; A.active = d.active;
    A.do_ladder = f.do_ladder; A.do_mosaic = f.do_mosaic; A.do_ring = f.do_ring; A.do_xring = f.do_xring;
    A.do_driver = f.do_driver; A.drpa = f.drpa; A.mode = mode;
    A.rx = d.rx; A.rpos = d.rpos;
    A.st = diis ? diis->state : nullptr; A.ndiis = (diis && mode == 0) ? ndiis : 0; A.namp = d.namp;
    A.hist_t = diis ? diis->hist_t : nullptr; A.hist_e = diis ? diis->hist_e : nullptr;
    A.dpart = diis ? diis->part : nullptr;
    A.vcoef = d.vcoef;
    kt->begin(KID_UPDATE, st);
    k_update<<<d.nhchunks, kChunk, 0, st>>>(A);
    kt->end(st);
    n++;
    kt->begin(KID_REDUCE, st);
    k_reduce_solves<<<d.nsolves, 256, 0, st>>>(d.hchunk_begin, d.part_e, d.part_dt, d.part_r, d.red);
    kt->end(st);
    n++;
    return n;
}

void launch_pack(const DevBatch &d, int s, int namp, const double *dense, cudaStream_t st)
{
    k_pack<<<(namp + 255) / 256, 256, 0, st>>>(d.solves, s, d.amps, dense, d.t);
}

void launch_unpack(const DevBatch &d, int s, int namp, const double *t, double *ab, double *ba, double *aa,
                   cudaStream_t st)
{
    k_unpack<<<(namp + 255) / 256, 256, 0, st>>>(d.solves, s, d.amps, d.partner, t, ab, ba, aa);
}

}  // namespace uegccd

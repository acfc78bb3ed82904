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

#include "kernels.h"
#include "uegccd_internal.h"

namespace uegccd {

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
__global__ void k_mp2(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                      const AmpInfo *__restrict__ amps, const int4 *__restrict__ nv4,
                      const double *__restrict__ eigen, const double *__restrict__ vtab, double *__restrict__ t,
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
        double via = vpq(s, nv4, vtab, q.i, q.a);
        double vib = vpq(s, nv4, vtab, q.i, q.b);
        double x = via / denom;
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
__global__ void k_energy(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                         const AmpInfo *__restrict__ amps, const int4 *__restrict__ nv4,
                         const double *__restrict__ vtab, const double *__restrict__ t, int kind, double csosex,
                         double *__restrict__ part_e, double *__restrict__ part_a, double *__restrict__ part_b)
{
    const ChunkDev ch = chunks[blockIdx.x];
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    double e = 0.0, mx = 0.0;
    if (loc < s.namp) {
        const int64_t p = s.amp0 + loc;
        const AmpInfo q = amps[p];
        double x = t[p];
        double via = vpq(s, nv4, vtab, q.a, q.i);
        if (kind == 0) e = x * (2.0 * via - vpq(s, nv4, vtab, q.a, q.j));
        else e = via * x * 2.0 - vpq(s, nv4, vtab, q.b, q.i) * x * csosex;
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
// k_hh_w builds H_K; k_ladder writes G (it overwrites, so it runs first).
// ----------------------------------------------------------------------------
constexpr int kHhC = 32;
__global__ void k_hh_w(const BlockDev *__restrict__ blocks, const SolveDev *__restrict__ solves,
                       const int16_t *__restrict__ pair_i, const int16_t *__restrict__ vir,
                       const int4 *__restrict__ nv4, const double *__restrict__ vtab,
                       const double *__restrict__ t, const int64_t *__restrict__ hh0, double *__restrict__ hh,
                       const uint8_t *__restrict__ active)
{
    const BlockDev B = blocks[blockIdx.x];
    if (!active[B.solve]) return;
    const SolveDev s = solves[B.solve];
    extern __shared__ double sm[];
    const int o = B.o, v = B.v;
    double *Ts = sm;                    // o x kHhC
    double *Us = Ts + o * kHhC;         // kHhC x o
    int4 *nk = (int4 *)(Us + kHhC * o); // o
    for (int q = threadIdx.x; q < o; q += blockDim.x) nk[q] = nv4[s.orb0 + pair_i[B.pair0 + q]];
    const int nent = o * o;
    constexpr int kPer = 16;  // entries per thread (o <= 64 -> 4096 entries <= 256*16)
    double acc[kPer];
#pragma unroll
    for (int r = 0; r < kPer; r++) acc[r] = 0.0;
    __syncthreads();
    for (int c0 = 0; c0 < v; c0 += kHhC) {
        for (int e = threadIdx.x; e < o * kHhC; e += blockDim.x) {
            int pp = e / kHhC, cc = e % kHhC;
            Ts[pp * kHhC + cc] = (c0 + cc < v) ? t[B.t0 + (int64_t)pp * v + c0 + cc] : 0.0;
        }
        for (int e = threadIdx.x; e < o * kHhC; e += blockDim.x) {
            int cc = e / o, qq = e % o;
            double u = 0.0;
            if (c0 + cc < v) {
                int4 nc = nv4[s.orb0 + vir[B.vir0 + c0 + cc]];
                u = vtab[s.vtab0 + q2_of(nc, nk[qq])];
            }
            Us[cc * o + qq] = u;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kPer; r++) {
            int e = threadIdx.x + r * blockDim.x;
            if (e < nent) {
                int pp = e / o, qq = e % o;
                double a = acc[r];
                for (int cc = 0; cc < kHhC; cc++) a += Ts[pp * kHhC + cc] * Us[cc * o + qq];
                acc[r] = a;
            }
        }
        __syncthreads();
    }
    double *H = hh + hh0[blockIdx.x];
#pragma unroll
    for (int r = 0; r < kPer; r++) {
        int e = threadIdx.x + r * blockDim.x;
        if (e < nent) {
            int pp = e / o, qq = e % o;
            int ip = pair_i[B.pair0 + pp];
            int4 ni = nv4[s.orb0 + ip];
            H[pp * o + qq] = vtab[s.vtab0 + q2_of(ni, nk[qq])] + acc[r];
        }
    }
}

// G tile [a0, a0+64) x [p0, p0+32) of block blk.  128 threads, 4 (a) x 4 (p) each.
constexpr int kLA = 64, kLP = 32, kLC = 16;
__global__ void __launch_bounds__(128) k_ladder(const LadderTile *__restrict__ tiles,
                                               const BlockDev *__restrict__ blocks,
                                               const SolveDev *__restrict__ solves,
                                               const int16_t *__restrict__ vir, const int4 *__restrict__ nv4,
                                               const double *__restrict__ vtab, const double *__restrict__ t,
                                               const int64_t *__restrict__ hh0, const double *__restrict__ hh,
                                               int do_pp, int do_hh, double *__restrict__ g,
                                               const uint8_t *__restrict__ active)
{
    const LadderTile T = tiles[blockIdx.x];
    const BlockDev B = blocks[T.blk];
    if (!active[B.solve]) return;
    const SolveDev s = solves[B.solve];
    __shared__ double Ws[kLC][kLA + 2];
    __shared__ double Ts[kLC][kLP + 2];
    __shared__ int4 na[kLA];
    __shared__ int4 nc[kLC];
    const int tid = threadIdx.x;
    const int ta = tid >> 3;  // 0..15 -> a = 4*ta..4*ta+3
    const int tp = tid & 7;   // 0..7  -> p = 4*tp..4*tp+3
    const int v = B.v, o = B.o;
    for (int x = tid; x < kLA; x += blockDim.x) {
        int a = T.a0 + x;
        na[x] = (a < v) ? nv4[s.orb0 + vir[B.vir0 + a]] : make_int4(0, 0, 0, 0);
    }
    double acc[4][4];
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
    __syncthreads();
    if (do_pp) {
        for (int c0 = 0; c0 < v; c0 += kLC) {
            if (tid < kLC) {
                int c = c0 + tid;
                nc[tid] = (c < v) ? nv4[s.orb0 + vir[B.vir0 + c]] : make_int4(0, 0, 0, 0);
            }
            __syncthreads();
            for (int e = tid; e < kLC * kLA; e += blockDim.x) {
                int cc = e / kLA, aa = e % kLA;
                bool ok = (c0 + cc < v) && (T.a0 + aa < v);
                Ws[cc][aa] = ok ? vtab[s.vtab0 + q2_of(nc[cc], na[aa])] : 0.0;
            }
            for (int e = tid; e < kLC * kLP; e += blockDim.x) {
                int pp = e / kLC, cc = e % kLC;
                int p = T.p0 + pp, c = c0 + cc;
                Ts[cc][pp] = (p < o && c < v) ? t[B.t0 + (int64_t)p * v + c] : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int cc = 0; cc < kLC; cc++) {
                double wa[4], tp4[4];
#pragma unroll
                for (int x = 0; x < 4; x++) wa[x] = Ws[cc][ta * 4 + x];
#pragma unroll
                for (int y = 0; y < 4; y++) tp4[y] = Ts[cc][tp * 4 + y];
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] = fma(wa[x], tp4[y], acc[x][y]);
            }
            __syncthreads();
        }
    }
    if (do_hh) {
        // acc[a][p] += sum_q t[q][a] * H[p][q]
        const double *H = hh + hh0[T.blk];
        for (int q0 = 0; q0 < o; q0 += kLC) {
            for (int e = tid; e < kLC * kLA; e += blockDim.x) {
                int qq = e / kLA, aa = e % kLA;
                int q = q0 + qq, a = T.a0 + aa;
                Ws[qq][aa] = (q < o && a < v) ? t[B.t0 + (int64_t)q * v + a] : 0.0;
            }
            for (int e = tid; e < kLC * kLP; e += blockDim.x) {
                int pp = e / kLC, qq = e % kLC;
                int p = T.p0 + pp, q = q0 + qq;
                Ts[qq][pp] = (p < o && q < o) ? H[p * o + q] : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int qq = 0; qq < kLC; qq++) {
                double wa[4], tp4[4];
#pragma unroll
                for (int x = 0; x < 4; x++) wa[x] = Ws[qq][ta * 4 + x];
#pragma unroll
                for (int y = 0; y < 4; y++) tp4[y] = Ts[qq][tp * 4 + y];
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] = fma(wa[x], tp4[y], acc[x][y]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int y = 0; y < 4; y++) {
        int p = T.p0 + tp * 4 + y;
        if (p >= o) continue;
#pragma unroll
        for (int x = 0; x < 4; x++) {
            int a = T.a0 + ta * 4 + x;
            if (a < v) g[B.t0 + (int64_t)p * v + a] = acc[x][y];
        }
    }
}

// ----------------------------------------------------------------------------
// Mosaics (GetG2Mosaics, CCD.f90:548-582):
//   s(k,l,c) = v(c-k) (T2aaaa + T2abab)(kl,c) - v(c-l) (T2aaaa + T2abba)(kl,c)
//            = v(c-k) (2t(kl,c) - t(kl,d)) - v(c-l) (t(kl,c) - 2t(kl,d))
//   Jvv(c) = sum_{k,l} s(k,l,c),  Joo(k) = sum_{l,c} s(k,l,c)
// dRPA (dRPA.f90:415-431): s(k,l,c) = 2 v(c-k) t(kl,c).
// ----------------------------------------------------------------------------
__global__ void k_mosaic_s(const ChunkDev *__restrict__ chunks, const SolveDev *__restrict__ solves,
                           const AmpInfo *__restrict__ amps, const int32_t *__restrict__ partner,
                           const int4 *__restrict__ nv4, const double *__restrict__ vtab,
                           const double *__restrict__ t, int drpa, double *__restrict__ S,
                           const uint8_t *__restrict__ active)
{
    const ChunkDev ch = chunks[blockIdx.x];
    if (!active[ch.solve]) return;
    const SolveDev s = solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (loc >= s.namp) return;
    const int64_t p = s.amp0 + loc;
    const AmpInfo q = amps[p];
    double x = t[p];
    double vck = vpq(s, nv4, vtab, q.a, q.i);
    if (drpa) {
        S[p] = 2.0 * vck * x;
    } else {
        double y = t[partner[p]];
        double vcl = vpq(s, nv4, vtab, q.a, q.j);
        S[p] = vck * (2.0 * x - y) - vcl * (x - 2.0 * y);
    }
}

// One CTA per mosaic target: targets [0, V) are Jvv(c = O + x), [V, V+O) are Joo(k).
__global__ void k_mosaic_reduce(const int2 *__restrict__ targets, const SolveDev *__restrict__ solves,
                                const int32_t *__restrict__ pos, const double *__restrict__ S,
                                double *__restrict__ jvv, double *__restrict__ joo,
                                const uint8_t *__restrict__ active)
{
    const int2 tg = targets[blockIdx.x];
    if (!active[tg.x]) return;
    const SolveDev s = solves[tg.x];
    const int O = s.O, V = s.V;
    double acc = 0.0;
    if (tg.y < V) {
        const int cx = tg.y;
        for (int kl = threadIdx.x; kl < O * O; kl += blockDim.x) {
            int p = pos[s.pos0 + (int64_t)kl * V + cx];
            if (p >= 0) acc += S[p];
        }
    } else {
        const int k = tg.y - V;
        const int64_t base = s.pos0 + (int64_t)k * O * V;
        for (int lc = threadIdx.x; lc < O * V; lc += blockDim.x) {
            int p = pos[base + lc];
            if (p >= 0) acc += S[p];
        }
    }
    acc = block_sum<256>(acc);
    if (threadIdx.x == 0) {
        if (tg.y < V) jvv[s.jvv0 + tg.y] = acc;
        else joo[s.joo0 + tg.y - V] = acc;
    }
}

// ----------------------------------------------------------------------------
// Ring intermediates (quadratic rings CCD.f90:771-797, quadratic crossed rings
// CCD.f90:899-925), for every (i, x, l) with x virtual:
//   c = partner of (i,k,x); vd = v(i-x); ve = v(c-l) = v(i+k-x-l)
//   J1 = sum_k (2t(ik,x) - t(ik,c)) vd - (t(ik,x) - t(ik,c)) ve
//   J2 = sum_k (2t(ik,x) - t(ik,c)) vd - t(ik,x) ve
//   J3 = sum_k ve t(ki,x)
// dRPA (dRPA.f90:517-535): J1 = sum_k 2 t(ik,x) vd.
// The reference skips (i,x,l) when d = n_l + n_x - n_i is not a virtual; the apply
// step below makes the same test, so J is formed for every l.
// Layout: J[ph0 + (i*V + x)*O + l].
// ----------------------------------------------------------------------------
__global__ void k_ring_int(const ChunkDev *__restrict__ rchunks, const SolveDev *__restrict__ solves,
                           const AmpInfo *__restrict__ amps, const int32_t *__restrict__ partner,
                           const int32_t *__restrict__ pos, const int4 *__restrict__ nv4,
                           const double *__restrict__ vtab, const double *__restrict__ t, int drpa,
                           double *__restrict__ J1, double *__restrict__ J2, double *__restrict__ J3,
                           const uint8_t *__restrict__ active)
{
    const ChunkDev ch = rchunks[blockIdx.x];
    if (!active[ch.solve]) return;
    const SolveDev s = solves[ch.solve];
    const int O = s.O, V = s.V;
    const int e = ch.start + threadIdx.x;
    if (e >= O * V * O) return;
    const int l = e % O;
    const int ix = e / O;
    const int x = ix % V + O;
    const int i = ix / V;
    const double vd = vpq(s, nv4, vtab, i, x);
    const int4 nl = nv4[s.orb0 + l];
    double j1 = 0.0, j2 = 0.0, j3 = 0.0;
    for (int k = 0; k < O; k++) {
        int p1 = posmap(s, pos, i, k, x);
        if (p1 < 0) continue;
        double tx = t[p1];
        if (drpa) {
            j1 += 2.0 * tx * vd;
            continue;
        }
        int c = amps[p1].b;
        double ty = t[partner[p1]];
        double ve = vtab[s.vtab0 + q2_of(nv4[s.orb0 + c], nl)];
        j1 += (2.0 * tx - ty) * vd - (tx - ty) * ve;
        j2 += (2.0 * tx - ty) * vd - tx * ve;
        int p3 = posmap(s, pos, k, i, x);  // same partner c as (i,k,x): always allowed
        if (p3 >= 0) j3 += ve * t[p3];
    }
    const int64_t off = s.ph0 + e;
    J1[off] = j1;
    if (!drpa) { J2[off] = j2; J3[off] = j3; }
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
    const ChunkDev *chunks;
    const SolveDev *solves;
    const AmpInfo *amps;
    const int32_t *partner;
    const int32_t *pos;
    const int4 *nv4;
    const double *eigen;
    const double *vtab;
    const double *t;
    double *t_new;
    const double *g_ladder;
    const double *jvv, *joo;
    const double *J1, *J2, *J3;
    double *part_e, *part_dt, *part_r;
    double *g_out;            // optional: full G per amplitude (term checks)
    const uint8_t *active;
    int do_ladder, do_mosaic, do_ring, do_xring, do_driver, drpa, mode;
};

__global__ void __launch_bounds__(kChunk) k_update(UpdateArgs A)
{
    const ChunkDev ch = A.chunks[blockIdx.x];
    double esum = 0.0, dtmax = 0.0, rmax = 0.0;
    const bool on = A.active[ch.solve];
    const SolveDev s = A.solves[ch.solve];
    const int loc = ch.start + threadIdx.x;
    if (!on && A.mode == 0 && loc < s.namp) A.t_new[s.amp0 + loc] = A.t[s.amp0 + loc];
    if (on && loc < s.namp) {
        const int64_t p = s.amp0 + loc;
        const AmpInfo q = A.amps[p];
        const int i = q.i, j = q.j, a = q.a, b = q.b;
        const int O = s.O;
        const double told = A.t[p];
        const double via = vpq(s, A.nv4, A.vtab, i, a);
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
        } else {
            if (A.do_ring) {
                // linear rings (CCD.f90:716-763), c = partner of (i,k,a) / (j,k,b):
                //   (2v(i-a) - v(k-j)) t(ik,a) - v(i-a) t(ik,c)
                // + (2v(a-i) - v(k-i)) t(jk,b) - v(a-i) t(jk,c')
                double acc = 0.0;
                for (int k = 0; k < O; k++) {
                    int p1 = posmap(s, A.pos, i, k, a);
                    if (p1 >= 0) {
                        double tx = A.t[p1], ty = A.t[A.partner[p1]];
                        acc += (2.0 * via - vpq(s, A.nv4, A.vtab, k, j)) * tx - via * ty;
                    }
                    int p2 = posmap(s, A.pos, j, k, b);
                    if (p2 >= 0) {
                        double tx = A.t[p2], ty = A.t[A.partner[p2]];
                        acc += (2.0 * via - vpq(s, A.nv4, A.vtab, k, i)) * tx - via * ty;
                    }
                }
                // quadratic rings (CCD.f90:801-808): sum_l (J1+J2)(i,a,l) t(lj,d) - J2(i,a,l) t(lj,b)
                const int64_t jr = s.ph0 + ((int64_t)i * s.V + (a - O)) * O;
                for (int l = 0; l < O; l++) {
                    int pb = posmap(s, A.pos, l, j, b);  // (l,j,b) exists iff d is a virtual
                    if (pb < 0) continue;
                    double tb = A.t[pb], td = A.t[A.partner[pb]];
                    double j2 = A.J2[jr + l];
                    acc += (A.J1[jr + l] + j2) * td - j2 * tb;
                }
                g += acc;
            }
            if (A.do_xring) {
                // linear crossed rings (CCD.f90:851-889): -v(j-k) t(ki,b) - v(i-k) t(kj,a)
                double acc = 0.0;
                for (int k = 0; k < O; k++) {
                    int p3 = posmap(s, A.pos, k, i, b);
                    if (p3 >= 0) acc -= vpq(s, A.nv4, A.vtab, j, k) * A.t[p3];
                    int p4 = posmap(s, A.pos, k, j, a);
                    if (p4 >= 0) acc -= vpq(s, A.nv4, A.vtab, i, k) * A.t[p4];
                }
                // quadratic crossed rings (CCD.f90:927-934): sum_l J3(i,b,l) t(lj,a)
                const int64_t jr = s.ph0 + ((int64_t)i * s.V + (b - O)) * O;
                for (int l = 0; l < O; l++) {
                    int pa = posmap(s, A.pos, l, j, a);
                    if (pa < 0) continue;
                    acc += A.J3[jr + l] * A.t[pa];
                }
                g += acc;
            }
        }
        if (A.g_out) A.g_out[p] = g;
        const double *ev = A.eigen + s.orb0;
        const double denom = ev[i] + ev[j] - ev[a] - ev[b];
        const double r = -g + denom * told;
        rmax = fabs(r);
        if (A.mode == 0) {
            const double f = s.denom_factor;
            const double tn = (g / denom - (1.0 - f) * told) / f;
            A.t_new[p] = tn;
            dtmax = fabs(tn - told);
            if (A.drpa) esum = via * tn * 2.0;  // SOSEX part added by k_drpa_energy at the end
            else esum = tn * (2.0 * via - vpq(s, A.nv4, A.vtab, a, j));
            if (!(fabs(tn) < 1e300)) dtmax = __longlong_as_double(0x7ff0000000000000LL);  // +Inf marks NaN/Inf
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
    t[p] = dense[q.i + (int64_t)s.O * q.j + (int64_t)s.O * s.O * (q.a - s.O)];
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

// ----------------------------------------------------------------------------
// Launch wrappers
// ----------------------------------------------------------------------------
void launch_mp2(const DevBatch &d, cudaStream_t st)
{
    k_mp2<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.amps, d.nv4, d.eigen, d.vtab, d.t, d.part_e,
                                        d.part_dt, d.part_r);
}

void launch_reduce(const DevBatch &d, cudaStream_t st)
{
    k_reduce_solves<<<d.nsolves, 256, 0, st>>>(d.chunk_begin, d.part_e, d.part_dt, d.part_r, d.red);
}

void launch_energy(const DevBatch &d, int kind, double csosex, cudaStream_t st)
{
    k_energy<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.amps, d.nv4, d.vtab, d.t, kind, csosex, d.part_e,
                                           d.part_dt, d.part_r);
}

void launch_to_aaaa(const DevBatch &d, cudaStream_t st)
{
    k_to_aaaa<<<(unsigned)((d.namp + 255) / 256), 256, 0, st>>>(d.namp, d.partner, d.t, d.t_new);
}

const char *kKernelNames[KID_COUNT] = {"k_mp2", "k_energy", "k_hh_w", "k_ladder", "k_mosaic_s",
                                      "k_mosaic_reduce", "k_ring_int", "k_update", "k_reduce_solves", "k_pack"};

int launch_residual(const DevBatch &d, const TermFlags &f, int mode, double *g_out, cudaStream_t st,
                    KernelTimer *kt)
{
    KernelTimer dummy;
    if (!kt) kt = &dummy;
    int n = 0;
    if (f.do_ladder && d.nblocks > 0) {
        if (f.do_hh) {
            size_t smem = (size_t)(2 * d.max_o * kHhC) * sizeof(double) + (size_t)d.max_o * sizeof(int4);
            kt->begin(KID_HH_W, st);
            k_hh_w<<<d.nblocks, 256, smem, st>>>(d.blocks, d.solves, d.pair_i, d.vir, d.nv4, d.vtab, d.t, d.hh0,
                                                 d.hh, d.active);
            kt->end(st);
            n++;
        }
        kt->begin(KID_LADDER, st);
        k_ladder<<<d.ntiles, 128, 0, st>>>(d.tiles, d.blocks, d.solves, d.vir, d.nv4, d.vtab, d.t, d.hh0, d.hh,
                                           f.do_pp, f.do_hh, d.g, d.active);
        kt->end(st);
        n++;
    }
    if (f.do_mosaic) {
        kt->begin(KID_MOSAIC_S, st);
        k_mosaic_s<<<d.nchunks, kChunk, 0, st>>>(d.chunks, d.solves, d.amps, d.partner, d.nv4, d.vtab, d.t, f.drpa,
                                                 d.S, d.active);
        kt->end(st);
        kt->begin(KID_MOSAIC_RED, st);
        k_mosaic_reduce<<<d.ntargets, 256, 0, st>>>(d.targets, d.solves, d.pos, d.S, d.jvv, d.joo, d.active);
        kt->end(st);
        n += 2;
    }
    if (f.do_ring || f.do_xring) {
        kt->begin(KID_RING_INT, st);
        k_ring_int<<<d.nrchunks, kChunk, 0, st>>>(d.rchunks, d.solves, d.amps, d.partner, d.pos, d.nv4, d.vtab, d.t,
                                                  f.drpa, d.J1, d.J2, d.J3, d.active);
        kt->end(st);
        n++;
    }
    UpdateArgs A;
    A.chunks = d.chunks; A.solves = d.solves; A.amps = d.amps; A.partner = d.partner; A.pos = d.pos;
    A.nv4 = d.nv4; A.eigen = d.eigen; A.vtab = d.vtab; A.t = d.t; A.t_new = d.t_new; A.g_ladder = d.g;
    A.jvv = d.jvv; A.joo = d.joo; A.J1 = d.J1; A.J2 = d.J2; A.J3 = d.J3;
    A.part_e = d.part_e; A.part_dt = d.part_dt; A.part_r = d.part_r; A.g_out = g_out; A.active = d.active;
    A.do_ladder = f.do_ladder; A.do_mosaic = f.do_mosaic; A.do_ring = f.do_ring; A.do_xring = f.do_xring;
    A.do_driver = f.do_driver; A.drpa = f.drpa; A.mode = mode;
    kt->begin(KID_UPDATE, st);
    k_update<<<d.nchunks, kChunk, 0, st>>>(A);
    kt->end(st);
    n++;
    kt->begin(KID_REDUCE, st);
    k_reduce_solves<<<d.nsolves, 256, 0, st>>>(d.chunk_begin, d.part_e, d.part_dt, d.part_r, d.red);
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

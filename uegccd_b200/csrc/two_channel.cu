// two_channel.cu -- the two-channel form of the CCD residual and the general-flag dRPA
// residual: per-term integral flags and Do Rings without Do XRings.
//
// The spin-adapted kernels (kernels_fp64.cu) store T2abab alone and use
// T2abba(i,j,a) = -T2abab(i,j,b).  The reference keeps that relation only while each term's
// direct and exchange integrals are the same function and rings and crossed rings are both
// on or both off.  Here both channels, T2abab and T2abba, are iterated as DrvCCD does
// (CCD.f90:18-183), and every integral takes the flag the reference gives it: the Max(...)
// of its term's flags (CCD.f90:620-937).  dRPA keeps its one channel (DrvdRPA,
// dRPA.f90:23-174) with the flags of its terms.
//
// Layout: the reference's own, T(i,j,a) at i + O*j + O*O*(a-O) (0-based), FP64, on the
// device for the whole solve.  FindIndex(i,j,p) (HEG.f90:357-404) -- the orbital with
// n = n_i + n_j - n_p -- is one int32 table F over the occupied pairs and every orbital (all
// its calls in the terms have two occupied arguments).  An integral ERI(a,b,i,j,flag) is a
// table lookup: it depends on |n_a - n_i|^2, the flag and whether an index is a core orbital;
// the host fills the table of the routine SetPointers picks (Main.f90:274-318) with that
// routine's filters in their order.
//
// Kernels of one residual:
//   k2_mosaic   the mosaic sums Jvv(c) and Joo(k) (CCD.f90:507-585; dRPA.f90:377-446)
//   k2_hh       the hole-hole ladder sums j2, j3 of every (i,j,k) (CCD.f90:597-631)
//   k2_ringq    the quadratic ring sums of every (i,a,l) (CCD.f90:771-811; dRPA.f90:520-551)
//   k2_xringq   the quadratic crossed-ring sums of every (i,b,l) (CCD.f90:899-937)
//   k2_assemble every term of one amplitude (i,j,a) in the reference's order: drivers,
//               mosaics, hole-hole then particle-particle ladder, rings, crossed rings
// and per iteration k2_update (GetRes, SolveCC, CnvrgCC and CCEnergy).  Each sum has a fixed
// order and every reduction a fixed tree, so results do not depend on the launch.
#include "two_channel.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

namespace uegccd {
int set_last_error(int code, const char *msg);

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDiis = 16;

int tfail(int code, const std::string &m) { return set_last_error(code, m.c_str()); }

#define TCU(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return tfail(UEGCCD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

struct View2 {
    int O, M, V, nq, core_n;
    int n;                  // O*O*V amplitudes per channel
    const int *F;
    const int4 *nv;
    const double *vt;       // [core 0/1][flag 0..3][|q|^2]
    const double *eig;
    TcFlags f;
};

__device__ __forceinline__ int fnd(const View2 &D, int i, int j, int p)
{
    return __ldg(D.F + (i + D.O * (j + D.O * p))) - 1;
}

// ERI(a,b,i,j,flag) of the selected routine: momentum transfer n_a - n_i.
__device__ __forceinline__ double eri(const View2 &D, int a, int b, int i, int j, int flag)
{
    const int4 na = __ldg(D.nv + a), ni = __ldg(D.nv + i);
    const int dx = na.x - ni.x, dy = na.y - ni.y, dz = na.z - ni.z;
    const int core = min(min(a, b), min(i, j)) < D.core_n ? 1 : 0;
    return __ldg(D.vt + ((core * 4 + flag) * D.nq + dx * dx + dy * dy + dz * dz));
}

// The reference's "If (Min(V1,V2) < -80) Cycle" (the -100 of an excluded integral).
__device__ __forceinline__ bool excluded(double v1, double v2) { return fmin(v1, v2) < -80.0; }

__device__ __forceinline__ double nanmax(double a, double b) { return (a > b || a != a) ? a : b; }

// Fixed-tree block reductions (result in thread 0); sh holds kThreads/32 doubles.
__device__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ double block_max(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    return v;
}

// FindIndex table: F[i + O*(j + O*p)] = 1 + the orbital of n_i + n_j - n_p, 0 when that
// vector is not in the basis.  cube: 1 + orbital of each n in [-R, R]^3, 0 elsewhere.
__global__ void k2_find(View2 D, const int *__restrict__ cube, int R, int *F)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)D.O * D.O * D.M;
    if (e >= total) return;
    const int i = (int)(e % D.O), j = (int)((e / D.O) % D.O), p = (int)(e / ((int64_t)D.O * D.O));
    const int4 a = D.nv[i], b = D.nv[j], c = D.nv[p];
    const int x = a.x + b.x - c.x, y = a.y + b.y - c.y, z = a.z + b.z - c.z;
    int r = 0;
    if (abs(x) <= R && abs(y) <= R && abs(z) <= R) {
        const int S = 2 * R + 1;
        r = cube[(x + R) + S * ((y + R) + S * (z + R))];
    }
    F[e] = r;
}

// Mosaic sums (GetG2Mosaics, CCD.f90:507-585; dRPA.f90:377-446).  Blocks [0, V): Jvv(c),
// over (k,l); blocks [V, V+O): Joo(k), over (l,c).  CCD: w = V_cdkl (Taaaa + Tabab) -
// V_cdlk (Taaaa + Tabba); dRPA: w = 2 V_cdkl T.
template <bool DRPA>
__global__ void __launch_bounds__(kThreads) k2_mosaic(View2 D, const double *__restrict__ tab,
                                                      const double *__restrict__ tba, double *jvv, double *joo)
{
    __shared__ double sh[kThreads / 32];
    const int O = D.O;
    const bool vv = (int)blockIdx.x < D.V;
    const int fixed = vv ? blockIdx.x : blockIdx.x - D.V;
    const int cnt = vv ? O * O : O * D.V;
    double s = 0.0;
    for (int p = threadIdx.x; p < cnt; p += blockDim.x) {
        int k, l, va;
        if (vv) {
            va = fixed, k = p % O, l = p / O;
        } else {
            k = fixed, l = p % O, va = p / O;
        }
        const int c = O + va;
        const int d = fnd(D, k, l, c);
        if (d < O) continue;
        const double v1 = eri(D, c, d, k, l, D.f.mosaic);
        const int x = k + O * (l + O * va);
        if (DRPA) {
            if (v1 < -80.0) continue;
            s += 2.0 * v1 * tab[x];
        } else {
            const double v2 = eri(D, c, d, l, k, D.f.mosaic);
            if (excluded(v1, v2)) continue;
            const double ta = tab[x] + tba[x];
            s += v1 * (ta + tab[x]) - v2 * (ta + tba[x]);
        }
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) (vv ? jvv : joo)[fixed] = s;
}

// Hole-hole ladder sums (GetG2Ladders, CCD.f90:597-631), one warp per (i,j,k), l the
// momentum partner: j2 = V_ijkl + 1/2 sum_c (V_cdkl Tabab(ijc) - V_cdlk Tabba(ijc)),
// j3 = -V_ijlk + 1/2 sum_c (V_cdkl Tabba(ijc) - V_cdlk Tabab(ijc)); 0 when excluded.
__global__ void __launch_bounds__(kThreads) k2_hh(View2 D, const double *__restrict__ tab,
                                                  const double *__restrict__ tba, double *h2, double *h3)
{
    const int O = D.O;
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (w >= O * O * O) return;   // whole warps
    const int i = w % O, j = (w / O) % O, k = w / (O * O);
    const int l = fnd(D, i, j, k);
    bool on = l >= 0 && l < O;
    double e2 = 0.0, e3 = 0.0, j2 = 0.0, j3 = 0.0;
    if (on) {
        e2 = eri(D, i, j, k, l, D.f.lad_lin_d);
        e3 = -eri(D, i, j, l, k, D.f.lad_lin_x);
        on = !(fmin(e2, -e3) < -80.0);
    }
    if (on) {
        for (int c = O + lane; c < D.M; c += 32) {
            const int d = fnd(D, i, j, c);
            if (d < O) continue;
            const double v1 = eri(D, c, d, k, l, D.f.lad_quad_d), v2 = eri(D, c, d, l, k, D.f.lad_quad_x);
            if (excluded(v1, v2)) continue;
            const int y = i + O * (j + O * (c - O));
            j2 += 0.5 * (v1 * tab[y] - v2 * tba[y]);
            j3 += 0.5 * (v1 * tba[y] - v2 * tab[y]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            j2 += __shfl_xor_sync(0xffffffffu, j2, o);
            j3 += __shfl_xor_sync(0xffffffffu, j3, o);
        }
    }
    if (lane == 0) {
        h2[w] = on ? e2 + j2 : 0.0;
        h3[w] = on ? e3 + j3 : 0.0;
    }
}

// Quadratic ring sums (GetG2Rings, CCD.f90:771-790; dRPA.f90:520-536) of (i,a,l) at
// r = i + O*(l + O*(a-O)), over k with c = FindIndex(i,k,a), d = FindIndex(k,l,c).
template <bool DRPA>
__global__ void __launch_bounds__(kThreads) k2_ringq(View2 D, const double *__restrict__ tab,
                                                     const double *__restrict__ tba, double *r1, double *r2,
                                                     double *r3)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= D.n) return;
    const int O = D.O;
    const int i = r % O, l = (r / O) % O, va = r / (O * O), a = O + va;
    double j1 = 0.0, j2 = 0.0, j3 = 0.0;
    for (int k = 0; k < O; k++) {
        const int c = fnd(D, i, k, a);
        if (c < O) continue;
        const int d = fnd(D, k, l, c);
        if (d < O) continue;
        const double v1 = eri(D, c, d, k, l, D.f.ring_quad_d);
        const int y = i + O * (k + O * va);
        if (DRPA) {
            if (v1 < -80.0) continue;
            j1 += 2.0 * tab[y] * v1;
        } else {
            const double v2 = eri(D, c, d, l, k, D.f.ring_quad_x);
            if (excluded(v1, v2)) continue;
            const double ta = tab[y] + tba[y];
            j1 += ta * (v1 - v2) + tab[y] * v1;
            j2 += tab[y] * (v1 - v2) + ta * v1;
            j3 -= tba[y] * v2;
        }
    }
    r1[r] = j1;
    if (!DRPA) {
        r2[r] = j2;
        r3[r] = j3;
    }
}

// Quadratic crossed-ring sums (GetG2XRings, CCD.f90:899-922) of (i,b,l) at
// r = i + O*(l + O*(b-O)), over k with c = FindIndex(i,k,b), d = FindIndex(k,l,c).
__global__ void __launch_bounds__(kThreads) k2_xringq(View2 D, const double *__restrict__ tab,
                                                      const double *__restrict__ tba, double *x1, double *x2,
                                                      double *x3)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= D.n) return;
    const int O = D.O;
    const int i = r % O, l = (r / O) % O, vb = r / (O * O), b = O + vb;
    double j1 = 0.0, j2 = 0.0, j3 = 0.0;
    for (int k = 0; k < O; k++) {
        const int c = fnd(D, i, k, b);
        if (c < O) continue;
        const int d = fnd(D, k, l, c);
        if (d < O) continue;
        const double v1 = eri(D, c, d, k, l, D.f.xr_quad_d), v2 = eri(D, c, d, l, k, D.f.xr_quad_x);
        if (excluded(v1, v2)) continue;
        const int y = k + O * (i + O * vb);
        const double ta = tab[y] + tba[y];
        j1 += ta * (v1 - v2) + tba[y] * v1;
        j2 += tba[y] * (v1 - v2) + ta * v1;
        j3 += tab[y] * v2;
    }
    x1[r] = j1;
    x2[r] = j2;
    x3[r] = j3;
}

struct Inter {
    const double *jvv, *joo, *h2, *h3, *r1, *r2, *r3, *x1, *x2, *x3;
};

// Every term of one amplitude x = (i,j,a), b its momentum partner, in the reference's order
// (TermsWrapper, CCD.f90:146-181): drivers (CCD.f90:465-504; dRPA.f90:339-374), mosaics,
// ladders (hole-hole, then particle-particle, CCD.f90:588-686), rings (CCD.f90:689-814;
// dRPA.f90:453-551), crossed rings (CCD.f90:817-940).  Amplitudes without a virtual partner
// get G = 0.
template <bool DRPA>
__global__ void __launch_bounds__(kThreads) k2_assemble(View2 D, int mask, const double *__restrict__ tab,
                                                        const double *__restrict__ tba, Inter J, double *gab,
                                                        double *gba)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= D.n) return;
    const int O = D.O;
    const int i = x % O, j = (x / O) % O, va = x / (O * O), a = O + va;
    const int b = fnd(D, i, j, a);
    if (b < O) {
        gab[x] = 0.0;
        if (!DRPA) gba[x] = 0.0;
        return;
    }
    const int vb = b - O;
    const TcFlags &f = D.f;
    const double t1 = tab[x], t2 = DRPA ? 0.0 : tba[x];
    double g1 = 0.0, g2 = 0.0;
    if (mask & 1) {
        if (DRPA) {
            const double v = eri(D, i, j, a, b, f.drv_d);
            if (!(v < -80.0)) g1 = v;
        } else {
            const double v1 = eri(D, i, j, a, b, f.drv_d), v2 = eri(D, i, j, b, a, f.drv_x);
            if (!excluded(v1, v2)) {
                g1 = v1;
                g2 = -v2;
            }
        }
    }
    if (mask & 2) {
        const double ja = J.jvv[va], jb = J.jvv[vb], ji = J.joo[i], jj = J.joo[j];
        g1 = g1 - 0.5 * (ja * t1 + jb * t1);
        g1 = g1 - 0.5 * (ji * t1 + jj * t1);
        if (!DRPA) {
            g2 = g2 - 0.5 * (ja * t2 + jb * t2);
            g2 = g2 - 0.5 * (ji * t2 + jj * t2);
        }
    }
    if (!DRPA && (mask & 4)) {
        for (int k = 0; k < O; k++) {
            const int l = fnd(D, i, j, k);
            if (l < 0 || l >= O) continue;
            const int w = i + O * (j + O * k), y = k + O * (l + O * va);
            const double h2 = J.h2[w], h3 = J.h3[w];
            g1 += 0.5 * (h2 * tab[y] + h3 * tba[y]);
            g2 += 0.5 * (h2 * tba[y] + h3 * tab[y]);
        }
        // the particle-particle sum over c, the largest loop of the form: ERI(c,d,a,b) and
        // ERI(c,d,b,a) (momentum transfers n_c - n_a and n_c - n_b) with the vectors of a and b,
        // the table rows of both flags and the row (i,j) of FindIndex taken out of the loop
        const int4 na = __ldg(D.nv + a), nb = __ldg(D.nv + b);
        const bool core_ab = min(a, b) < D.core_n;
        const double *vd0 = D.vt + f.lad_lin_d * D.nq, *vd1 = vd0 + 4 * D.nq;
        const double *vx0 = D.vt + f.lad_lin_x * D.nq, *vx1 = vx0 + 4 * D.nq;
        const int OO = O * O, x0 = i + O * j;
        const int *Fij = D.F + x0;
        for (int c = O; c < D.M; c++) {
            const int d = __ldg(Fij + OO * c) - 1;
            if (d < O) continue;
            const int4 nc = __ldg(D.nv + c);
            const int ax = nc.x - na.x, ay = nc.y - na.y, az = nc.z - na.z;
            const int bx = nc.x - nb.x, by = nc.y - nb.y, bz = nc.z - nb.z;
            const bool core = core_ab || min(c, d) < D.core_n;
            const double v1 = __ldg((core ? vd1 : vd0) + (ax * ax + ay * ay + az * az));
            const double v2 = __ldg((core ? vx1 : vx0) + (bx * bx + by * by + bz * bz));
            if (excluded(v1, v2)) continue;
            const int y = x0 + OO * (c - O);
            g1 += 0.5 * (v1 * tab[y] - v2 * tba[y]);
            g2 += 0.5 * (v1 * tba[y] - v2 * tab[y]);
        }
    }
    if (mask & 8) {
        for (int k = 0; k < O; k++) {
            const int c = fnd(D, i, k, a);
            if (c < O) continue;
            const int y = i + O * (k + O * va);
            if (DRPA) {
                const double v = eri(D, c, j, k, b, f.ring_lin_d);
                if (v < -80.0) continue;
                g1 += 2.0 * v * tab[y];
            } else {
                const double v1 = eri(D, c, j, k, b, f.ring_lin_d), v2 = eri(D, c, j, b, k, f.ring_lin_x);
                if (excluded(v1, v2)) continue;
                g1 += (v1 - v2) * tab[y] + v1 * (tab[y] + tba[y]);
                g2 -= v2 * tba[y];
            }
        }
        for (int k = 0; k < O; k++) {
            const int c = fnd(D, j, k, b);
            if (c < O) continue;
            const int y = j + O * (k + O * vb);
            if (DRPA) {
                const double v = eri(D, c, i, k, a, f.ring_lin_d);
                if (v < -80.0) continue;
                g1 += 2.0 * v * tab[y];
            } else {
                const double v1 = eri(D, c, i, k, a, f.ring_lin_d), v2 = eri(D, c, i, a, k, f.ring_lin_x);
                if (excluded(v1, v2)) continue;
                g1 += (v1 - v2) * tab[y] + v1 * (tab[y] + tba[y]);
                g2 -= v2 * tba[y];
            }
        }
        for (int l = 0; l < O; l++) {
            const int d = fnd(D, j, l, b);
            if (d < O) continue;
            const int y = l + O * (j + O * (d - O)), r = i + O * (l + O * va);
            if (DRPA) {
                g1 += 2.0 * J.r1[r] * tab[y];
            } else {
                g1 += J.r2[r] * (tab[y] + tba[y]) + J.r1[r] * tab[y];
                g2 += J.r3[r] * tba[y];
            }
        }
    }
    if (!DRPA && (mask & 16)) {
        for (int k = 0; k < O; k++) {
            const int c = fnd(D, k, i, b);
            if (c < O) continue;
            const double v1 = eri(D, j, c, k, a, f.xr_lin_x), v2 = eri(D, j, c, a, k, f.xr_lin_d);
            if (excluded(v1, v2)) continue;
            const int y = k + O * (i + O * vb);
            g1 -= v1 * tab[y];
            g2 += (v2 - v1) * tba[y] + v2 * (tab[y] + tba[y]);
        }
        for (int k = 0; k < O; k++) {
            const int c = fnd(D, k, j, a);
            if (c < O) continue;
            const double v1 = eri(D, i, c, k, b, f.xr_lin_x), v2 = eri(D, i, c, b, k, f.xr_lin_d);
            if (excluded(v1, v2)) continue;
            const int y = k + O * (j + O * va);
            g1 -= v1 * tab[y];
            g2 += (v2 - v1) * tba[y] + v2 * (tab[y] + tba[y]);
        }
        for (int l = 0; l < O; l++) {
            const int d = fnd(D, l, j, a);
            if (d < O) continue;
            const int y = l + O * (j + O * va), r = i + O * (l + O * vb);
            g2 = g2 - J.x1[r] * tba[y] - J.x2[r] * (tab[y] + tba[y]);
            g1 += J.x3[r] * tab[y];
        }
    }
    gab[x] = g1;
    if (!DRPA) gba[x] = g2;
}

// One iteration's update of every amplitude with a virtual partner: GetRes into the DIIS
// history (CCD.f90:389-424), SolveCC (CCD.f90:354-386), max|dT| (CnvrgCC, CCD.f90:427-462)
// and the energy of the new amplitudes (CCEnergy, CCD.f90:186-237; dRPA.f90:181-216, csosex
// 0).  part[2*block] = max|dT|, part[2*block+1] = energy of the block.
template <bool DRPA>
__global__ void __launch_bounds__(kThreads) k2_update(View2 D, double df, double *tab, double *tba,
                                                      const double *__restrict__ gab, const double *__restrict__ gba,
                                                      double *rab, double *rba, double *hab, double *hba, double *part)
{
    __shared__ double sh[kThreads / 32];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    double dmax = 0.0, e = 0.0;
    if (x < D.n) {
        const int O = D.O;
        const int i = x % O, j = (x / O) % O, a = O + x / (O * O);
        const int b = fnd(D, i, j, a);
        if (b < O) {
            // no virtual partner: the amplitude stays as it is, and its history entries are
            // that value and a zero residual, so that the dot products and the extrapolation
            // read defined values everywhere
            if (rab) rab[x] = 0.0;
            if (hab) hab[x] = tab[x];
            if (!DRPA) {
                if (rba) rba[x] = 0.0;
                if (hba) hba[x] = tba[x];
            }
        } else {
            const double denom = D.eig[i] + D.eig[j] - D.eig[a] - D.eig[b];
            const double o1 = tab[x], q1 = gab[x];
            if (rab) rab[x] = -q1 + denom * o1;
            const double n1 = (q1 / denom - (1.0 - df) * o1) / df;
            tab[x] = n1;
            if (hab) hab[x] = n1;
            dmax = fabs(n1 - o1);
            if (DRPA) {
                const double v1 = eri(D, a, b, i, j, 0), v2 = eri(D, b, a, i, j, 0);
                e = v1 * n1 * 2.0 - v2 * n1 * 0.0;
            } else {
                const double o2 = tba[x], q2 = gba[x];
                if (rba) rba[x] = -q2 + denom * o2;
                const double n2 = (q2 / denom - (1.0 - df) * o2) / df;
                tba[x] = n2;
                if (hba) hba[x] = n2;
                dmax = nanmax(dmax, fabs(n2 - o2));
                const double v1 = eri(D, a, b, i, j, D.f.energy), v2 = eri(D, a, b, j, i, D.f.energy);
                if (!excluded(v1, v2)) {
                    const double ta = n1 + n2;
                    e = 0.5 * (v1 * (ta + n1) - v2 * (ta + n2));
                }
            }
        }
    }
    const double m = block_max(dmax, sh);
    const double s = block_sum(e, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = m;
        part[2 * blockIdx.x + 1] = s;
    }
}

// Statistics of the amplitudes as they are: max|T| over both channels (every element, as
// MaxVal(Abs(T)) reads them, CCD.f90:63) and the energy (dRPA: with csosex), or, when g is
// given, max|R| of GetRes (CCD.f90:103-107).  part as in k2_update.
template <bool DRPA>
__global__ void __launch_bounds__(kThreads) k2_stats(View2 D, double csosex, const double *__restrict__ tab,
                                                     const double *__restrict__ tba, const double *__restrict__ gab,
                                                     const double *__restrict__ gba, double *part)
{
    __shared__ double sh[kThreads / 32];
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0, e = 0.0;
    if (x < D.n) {
        const int O = D.O;
        const int i = x % O, j = (x / O) % O, a = O + x / (O * O);
        const int b = fnd(D, i, j, a);
        const double t1 = tab[x], t2 = DRPA ? 0.0 : tba[x];
        if (!gab) m = nanmax(fabs(t1), fabs(t2));
        if (b >= O) {
            if (gab) {
                const double denom = D.eig[i] + D.eig[j] - D.eig[a] - D.eig[b];
                m = fabs(-gab[x] + denom * t1);
                if (!DRPA) m = nanmax(m, fabs(-gba[x] + denom * t2));
            }
            if (DRPA) {
                const double v1 = eri(D, a, b, i, j, 0), v2 = eri(D, b, a, i, j, 0);
                e = v1 * t1 * 2.0 - v2 * t1 * csosex;
            } else {
                const double v1 = eri(D, a, b, i, j, D.f.energy), v2 = eri(D, a, b, j, i, D.f.energy);
                if (!excluded(v1, v2)) {
                    const double ta = t1 + t2;
                    e = 0.5 * (v1 * (ta + t1) - v2 * (ta + t2));
                }
            }
        }
    }
    const double mm = block_max(m, sh);
    const double s = block_sum(e, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = mm;
        part[2 * blockIdx.x + 1] = s;
    }
}

// out[0] = max of part[2b], out[1] = sum of part[2b+1], over nb blocks, in a fixed order.
__global__ void __launch_bounds__(kThreads) k2_finish(const double *part, int nb, double *out)
{
    __shared__ double sh[kThreads / 32];
    double m = 0.0, s = 0.0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        m = nanmax(m, part[2 * k]);
        s += part[2 * k + 1];
    }
    m = block_max(m, sh);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        out[0] = m;
        out[1] = s;
    }
}

// DIIS: the dot products of the newest residual pair (slot s) with every slot q < nd, over
// both channels: part[blk*nd + q].
__global__ void __launch_bounds__(kThreads) k2_dots(int n, int nd, int s, const double *__restrict__ rab,
                                                    const double *__restrict__ rba, double *part)
{
    __shared__ double sh[kThreads / 32];
    double acc[kMaxDiis];
#pragma unroll
    for (int q = 0; q < kMaxDiis; q++) acc[q] = 0.0;
    const double *ns_ab = rab + (int64_t)s * n, *ns_ba = rba ? rba + (int64_t)s * n : nullptr;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
        const double u = ns_ab[x], w = ns_ba ? ns_ba[x] : 0.0;
#pragma unroll
        for (int q = 0; q < kMaxDiis; q++)
            if (q < nd) {
                acc[q] += u * rab[(int64_t)q * n + x];
                if (ns_ba) acc[q] += w * rba[(int64_t)q * n + x];
            }
    }
    for (int q = 0; q < nd; q++) {
        const double v = block_sum(acc[q], sh);
        if (threadIdx.x == 0) part[blockIdx.x * nd + q] = v;
    }
}

__global__ void k2_dots_finish(const double *part, int nb, int nd, double *out)
{
    __shared__ double sh[kThreads / 32];
    for (int q = 0; q < nd; q++) {
        double s = 0.0;
        for (int k = threadIdx.x; k < nb; k += blockDim.x) s += part[k * nd + q];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[q] = s;
    }
}

struct Coef {
    double c[kMaxDiis];
};

// T = sum_q c_q T_q over the history (GetTFromDIIS's extrapolation, DIISCC.f90:118-125).
__global__ void __launch_bounds__(kThreads) k2_extrap(int n, int nd, Coef c, const double *__restrict__ hab,
                                                      const double *__restrict__ hba, double *tab, double *tba)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    double s1 = 0.0, s2 = 0.0;
    for (int q = 0; q < nd; q++) {
        s1 += c.c[q] * hab[(int64_t)q * n + x];
        if (hba) s2 += c.c[q] * hba[(int64_t)q * n + x];
    }
    tab[x] = s1;
    if (hba) tba[x] = s2;
}

// [B 1; 1 0] [c; y] = [0; 1] by LU with partial pivoting; false when a pivot is exactly 0.
bool pulay_solve(int nd, const std::vector<double> &B, std::vector<double> &c)
{
    const int n = nd + 1;
    std::vector<double> m((size_t)n * n, 0.0), v(n, 0.0);
    for (int p = 0; p < nd; p++) {
        for (int q = 0; q < nd; q++) m[p * n + q] = B[p * nd + q];
        m[p * n + nd] = 1.0;
        m[nd * n + p] = 1.0;
    }
    v[nd] = 1.0;
    for (int k = 0; k < n; k++) {
        int piv = k;
        for (int r = k + 1; r < n; r++)
            if (std::fabs(m[r * n + k]) > std::fabs(m[piv * n + k])) piv = r;
        if (m[piv * n + k] == 0.0) return false;
        if (piv != k) {
            for (int q = 0; q < n; q++) std::swap(m[k * n + q], m[piv * n + q]);
            std::swap(v[k], v[piv]);
        }
        for (int r = k + 1; r < n; r++) {
            const double l = m[r * n + k] / m[k * n + k];
            for (int q = k; q < n; q++) m[r * n + q] -= l * m[k * n + q];
            v[r] -= l * v[k];
        }
    }
    for (int k = n - 1; k >= 0; k--) {
        double s = v[k];
        for (int q = k + 1; q < n; q++) s -= m[k * n + q] * v[q];
        v[k] = s / m[k * n + k];
    }
    c.assign(v.begin(), v.begin() + nd);
    for (double x : c)
        if (!std::isfinite(x)) return false;
    return true;
}

inline int blocks_of(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

// BaseERI's value (HEG.f90:969-976) and CasedERI's before its filters (HEG.f90:725-762).
double base_value(double L, double mad, int q2) { return q2 == 0 ? -mad : 1.0 / (L * kPi * (double)q2); }
double cased_value(double L, double mad, double sd, int flag, int q2)
{
    if (q2 == 0) {
        switch (flag) {
        case 0: return -mad;
        case 1: return (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / std::pow(sd, 2.0);
        case 2: return -mad - (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / std::pow(sd, 2.0);
        default: return 0.0;
        }
    }
    const double q2s = (double)q2 * std::pow(2.0 * kPi / L, 2.0);
    switch (flag) {
    case 0: return 1.0 / (L * kPi * (double)q2);
    case 1: return (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / (std::pow(sd, 2.0) + q2s);
    case 2: return (1.0 / std::pow(L, 3.0)) * 4.0 * kPi / (std::pow(sd, 2.0) + q2s) * std::pow(sd, 2.0) / q2s;
    default: return 0.0;
    }
}

// One integral of a routine with its filters in the routine's order: CasedERI / NoCaseERI
// zero a core integral before "< 0 -> -100" and the GapII filter (HEG.f90:763-772,
// 822-831); CoreERI applies "< 0 -> -100" first (HEG.f90:880-885); GapERI and BaseERI have
// no core test.
double routine_value(int routine, bool core, int flag, double L, double mad, double sd, double gapii, int q2)
{
    double v = routine == TC_CASED ? cased_value(L, mad, sd, flag, q2) : base_value(L, mad, q2);
    switch (routine) {
    case TC_BASE: return v;
    case TC_CORE:
        if (v < 0.0) return -100.0;
        return core ? 0.0 : v;
    case TC_GAP:
        if (v < 0.0) return -100.0;
        if (v > gapii && gapii > 0.0) return 0.0;
        return v;
    default:   // TC_NOCASE, TC_CASED
        if (core) v = 0.0;
        if (v < 0.0) return -100.0;
        if (v > gapii && gapii > 0.0) return 0.0;
        return v;
    }
}

}  // namespace

int tc_pick_routine(const UegccdRangeTerms &fl, int safe_eri, int core_n, double gapii)
{
    const int32_t *p = &fl.ring;
    int s = 0;
    for (int k = 0; k < 15; k++) s += std::abs(p[k]);
    if ((s > 0 && gapii > 0.0 && core_n > 0) || safe_eri) return TC_CASED;
    if (gapii > 0.0 && core_n > 0) return TC_NOCASE;
    if (core_n > 0) return TC_CORE;
    if (gapii > 0.0) return TC_GAP;
    return TC_BASE;
}

TwoChannel::~TwoChannel()
{
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
}

int TwoChannel::alloc(void **p, size_t bytes)
{
    const int rc = al_.get(p, bytes);
    if (rc == 0) bytes_ += (bytes + 255) & ~(size_t)255;
    return rc;
}

int TwoChannel::init(const SystemHost &sys, cudaStream_t stream, TcAlloc al)
{
    O_ = sys.O;
    M_ = sys.M;
    V_ = M_ - O_;
    L_ = sys.L;
    madelung_ = sys.madelung;
    st_ = stream;
    al_ = std::move(al);
    const int64_t n = (int64_t)O_ * O_ * V_, nf = (int64_t)O_ * O_ * M_;
    if (nf >= (int64_t)1 << 31 || (int64_t)O_ * O_ * O_ * 32 >= (int64_t)1 << 31)
        return tfail(UEGCCD_ERR_UNSUPPORTED, "system too large for the two-channel form");
    n_ = n;
    int R = 0;
    for (const auto &v : sys.n)
        for (int d = 0; d < 3; d++) R = std::max(R, std::abs(v[d]));
    if (R > 63) return tfail(UEGCCD_ERR_UNSUPPORTED, "plane-wave components beyond +-63");
    nq_ = 3 * (2 * R) * (2 * R) + 1;
    const int S = 2 * R + 1;
    std::vector<int> cube((size_t)S * S * S, 0);
    std::vector<int4> nv(M_);
    for (int p = 0; p < M_; p++) {
        const auto &v = sys.n[p];
        nv[p] = make_int4(v[0], v[1], v[2], 0);
        int &c = cube[(v[0] + R) + S * ((v[1] + R) + (size_t)S * (v[2] + R))];
        if (c == 0) c = p + 1;   // the first orbital with this vector
    }
    nblk_ = blocks_of(n_);
    int *cube_d = nullptr;
    int rc = 0;
    al_.begin();
    if ((rc = alloc((void **)&F_, nf * sizeof(int))) || (rc = alloc((void **)&nv_, M_ * sizeof(int4))) ||
        (rc = alloc((void **)&vt_, (size_t)8 * nq_ * sizeof(double))) ||
        (rc = alloc((void **)&eig_, M_ * sizeof(double))) || (rc = alloc((void **)&cube_d, cube.size() * sizeof(int))) ||
        (rc = alloc((void **)&jvv_, V_ * sizeof(double))) || (rc = alloc((void **)&joo_, O_ * sizeof(double))) ||
        (rc = alloc((void **)&part_, (size_t)2 * std::max(nblk_, 1) * kMaxDiis * sizeof(double))) ||
        (rc = alloc((void **)&out_, 2 * kMaxDiis * sizeof(double)))) {
        al_.rollback();
        return rc;
    }
    for (int c = 0; c < 2; c++)
        if ((rc = alloc((void **)&t_[c], n_ * sizeof(double))) || (rc = alloc((void **)&g_[c], n_ * sizeof(double)))) {
            al_.rollback();
            return rc;
        }
    for (int c = 0; c < 2; c++)
        if ((rc = alloc((void **)&h_[c], (size_t)O_ * O_ * O_ * sizeof(double)))) {
            al_.rollback();
            return rc;
        }
    for (int c = 0; c < 3; c++)
        if ((rc = alloc((void **)&r_[c], n_ * sizeof(double))) || (rc = alloc((void **)&x_[c], n_ * sizeof(double)))) {
            al_.rollback();
            return rc;
        }
    TCU(cudaMemcpyAsync(nv_, nv.data(), M_ * sizeof(int4), cudaMemcpyHostToDevice, st_));
    TCU(cudaMemcpyAsync(cube_d, cube.data(), cube.size() * sizeof(int), cudaMemcpyHostToDevice, st_));
    TCU(cudaMemcpyAsync(eig_, sys.eigen.data(), M_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    View2 D{};
    D.O = O_, D.M = M_, D.V = V_, D.n = (int)n_, D.nv = nv_;
    k2_find<<<blocks_of(nf), kThreads, 0, st_>>>(D, cube_d, R, F_);
    TCU(cudaGetLastError());
    TCU(cudaStreamSynchronize(st_));
    if (!ev0_) TCU(cudaEventCreate(&ev0_));
    if (!ev1_) TCU(cudaEventCreate(&ev1_));
    UegccdRangeTerms none{};
    return set_integrals(TC_BASE, none, 0, 0.0, 0.0);
}

int TwoChannel::set_integrals(int routine, const UegccdRangeTerms &fl, int core_n, double gapii, double screening)
{
    const int32_t *p = &fl.ring;
    for (int k = 0; k < 15; k++)
        if (p[k] < 0 || p[k] > 3) return tfail(UEGCCD_ERR_ARG, "range flags must be 0, 1, 2 or 3");
    if (core_n < 0 || core_n > O_) return tfail(UEGCCD_ERR_ARG, "CoreN must be in [0, NOcc]");
    if (routine == TC_CASED) {
        bool need = false;
        for (int k = 0; k < 15; k++) need = need || p[k] == 1 || p[k] == 2;
        if (need && !(screening > 0.0)) return tfail(UEGCCD_ERR_ARG, "screening distance must be > 0");
    }
    const double g = gapii > 0.0 ? gapii : 0.0;
    std::vector<double> vt((size_t)8 * nq_);
    for (int core = 0; core < 2; core++)
        for (int flag = 0; flag < 4; flag++)
            for (int q2 = 0; q2 < nq_; q2++)
                vt[(size_t)(core * 4 + flag) * nq_ + q2] =
                    routine_value(routine, core != 0, flag, L_, madelung_, screening, g, q2);
    TCU(cudaMemcpyAsync(vt_, vt.data(), vt.size() * sizeof(double), cudaMemcpyHostToDevice, st_));
    TCU(cudaStreamSynchronize(st_));
    routine_ = routine;
    core_n_ = core_n;
    // The Max(...) of each integral's flags (CCD.f90:620-642, 726-750, 782-786, 855-879, 910-914).
    auto m3 = [](int a, int b, int c) { return std::max(a, std::max(b, c)); };
    TcFlags &f = f_;
    f.drv_d = fl.driver_direct;
    f.drv_x = fl.driver_exchange;
    f.mosaic = fl.mosaic;
    f.energy = fl.energy;
    f.lad_lin_d = m3(fl.ladder, fl.direct_ladders, fl.lin_ladders);
    f.lad_lin_x = m3(fl.ladder, fl.exchange_ladders, fl.lin_ladders);
    f.lad_quad_d = m3(fl.ladder, fl.direct_ladders, fl.quad_ladders);
    f.lad_quad_x = m3(fl.ladder, fl.exchange_ladders, fl.quad_ladders);
    f.ring_lin_d = m3(fl.ring, fl.direct_rings, fl.lin_rings);
    f.ring_lin_x = m3(fl.ring, fl.exchange_rings, fl.lin_rings);
    f.ring_quad_d = m3(fl.ring, fl.direct_rings, fl.quad_rings);
    f.ring_quad_x = m3(fl.ring, fl.exchange_rings, fl.quad_rings);
    f.xr_lin_d = m3(fl.xring, fl.direct_rings, fl.lin_rings);
    f.xr_lin_x = m3(fl.xring, fl.exchange_rings, fl.lin_rings);
    f.xr_quad_d = m3(fl.xring, fl.direct_rings, fl.quad_rings);
    f.xr_quad_x = m3(fl.xring, fl.exchange_rings, fl.quad_rings);
    return 0;
}

int TwoChannel::upload_t(const double *h, double *d)
{
    TCU(cudaMemcpyAsync(d, h, n_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    return 0;
}

int TwoChannel::read_out(int k, double *h)
{
    TCU(cudaMemcpyAsync(h, out_, k * sizeof(double), cudaMemcpyDeviceToHost, st_));
    TCU(cudaStreamSynchronize(st_));
    return 0;
}

// One residual G of the terms in mask from t_ into g_.
int TwoChannel::residual(bool drpa, int mask)
{
    View2 D{O_, M_, V_, nq_, core_n_, (int)n_, F_, nv_, vt_, eig_, f_};
    Inter J{jvv_, joo_, h_[0], h_[1], r_[0], r_[1], r_[2], x_[0], x_[1], x_[2]};
    if (mask & 2) {
        if (drpa)
            k2_mosaic<true><<<V_ + O_, kThreads, 0, st_>>>(D, t_[0], t_[1], jvv_, joo_);
        else
            k2_mosaic<false><<<V_ + O_, kThreads, 0, st_>>>(D, t_[0], t_[1], jvv_, joo_);
        launches_++;
    }
    if (!drpa && (mask & 4)) {
        k2_hh<<<blocks_of((int64_t)O_ * O_ * O_ * 32), kThreads, 0, st_>>>(D, t_[0], t_[1], h_[0], h_[1]);
        launches_++;
    }
    if (mask & 8) {
        if (drpa)
            k2_ringq<true><<<nblk_, kThreads, 0, st_>>>(D, t_[0], t_[1], r_[0], r_[1], r_[2]);
        else
            k2_ringq<false><<<nblk_, kThreads, 0, st_>>>(D, t_[0], t_[1], r_[0], r_[1], r_[2]);
        launches_++;
    }
    if (!drpa && (mask & 16)) {
        k2_xringq<<<nblk_, kThreads, 0, st_>>>(D, t_[0], t_[1], x_[0], x_[1], x_[2]);
        launches_++;
    }
    if (drpa)
        k2_assemble<true><<<nblk_, kThreads, 0, st_>>>(D, mask, t_[0], t_[1], J, g_[0], g_[1]);
    else
        k2_assemble<false><<<nblk_, kThreads, 0, st_>>>(D, mask, t_[0], t_[1], J, g_[0], g_[1]);
    launches_++;
    TCU(cudaGetLastError());
    return 0;
}

int TwoChannel::ccd_g2(const double *t_abab, const double *t_abba, int mask, double *g_abab, double *g_abba)
{
    int rc;
    if ((rc = upload_t(t_abab, t_[0])) || (rc = upload_t(t_abba, t_[1])) || (rc = residual(false, mask))) return rc;
    TCU(cudaMemcpyAsync(g_abab, g_[0], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    TCU(cudaMemcpyAsync(g_abba, g_[1], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    TCU(cudaStreamSynchronize(st_));
    return 0;
}

int TwoChannel::drpa_g2(const double *t2, int mask, double *g2)
{
    int rc;
    if ((rc = upload_t(t2, t_[0])) || (rc = residual(true, mask))) return rc;
    TCU(cudaMemcpyAsync(g2, g_[0], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    TCU(cudaStreamSynchronize(st_));
    return 0;
}

int TwoChannel::diis_alloc(int ndiis)
{
    if (ndiis <= ndiis_cap_) return 0;
    al_.begin();
    double *p[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < 4; k++) {
        const int rc = alloc((void **)&p[k], (size_t)ndiis * n_ * sizeof(double));
        if (rc) {
            al_.rollback();
            return rc;
        }
    }
    ht_[0] = p[0], ht_[1] = p[1], hr_[0] = p[2], hr_[1] = p[3];
    ndiis_cap_ = ndiis;
    return 0;
}

int TwoChannel::solve(const UegccdOptions &opt, bool drpa, const std::vector<double> &eigen, double *t_aaaa,
                      double *t_abab, double *t_abba, UegccdResult &res)
{
    int rc = 0;
    std::memset(&res, 0, sizeof(res));
    launches_ = 0;
    TCU(cudaMemcpyAsync(eig_, eigen.data(), M_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    if ((rc = upload_t(t_abab, t_[0]))) return rc;
    if (!drpa) {
        if (t_abba) {
            if ((rc = upload_t(t_abba, t_[1]))) return rc;
        } else {
            // the MP2 relation T2abba(i,j,a) = -T2abab(i,j,b) (MP2.f90:68-69)
            std::vector<int> F((size_t)O_ * O_ * M_);
            TCU(cudaMemcpyAsync(F.data(), F_, F.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
            TCU(cudaStreamSynchronize(st_));
            std::vector<double> ba(n_, 0.0);
            for (int va = 0; va < V_; va++)
                for (int j = 0; j < O_; j++)
                    for (int i = 0; i < O_; i++) {
                        const int b = F[i + O_ * (j + (size_t)O_ * (O_ + va))] - 1;
                        if (b < O_) continue;
                        ba[i + O_ * (j + (size_t)O_ * va)] = -t_abab[i + O_ * (j + (size_t)O_ * (b - O_))];
                    }
            if ((rc = upload_t(ba.data(), t_[1]))) return rc;
        }
    }
    // DIIS depth: SetUpDIISCC steps NDIIS down until its Allocate succeeds (DIISCC.f90:22-29)
    int nd = opt.scheme == UEGCCD_DIIS ? opt.ndiis : 0;
    if (nd > 0) {
        while ((rc = diis_alloc(nd)) == UEGCCD_ERR_ALLOC && nd > 2) nd--;
        if (rc) return rc;
    }
    View2 D{O_, M_, V_, nq_, core_n_, (int)n_, F_, nv_, vt_, eig_, f_};
    const int mask = drpa ? (1 | (opt.do_mosaic ? 2 : 0) | (opt.do_ring ? 8 : 0))
                          : (1 | (opt.do_mosaic ? 2 : 0) | (opt.do_ladder ? 4 : 0) | (opt.do_ring ? 8 : 0) |
                             (opt.do_xring ? 16 : 0));
    const double df = opt.denom_factor;
    TCU(cudaEventRecord(ev0_, st_));
    // dT = max|T| and the energy of the start amplitudes (CCD.f90:63-64; dRPA.f90:68-69)
    if (drpa)
        k2_stats<true><<<nblk_, kThreads, 0, st_>>>(D, 0.0, t_[0], t_[1], nullptr, nullptr, part_);
    else
        k2_stats<false><<<nblk_, kThreads, 0, st_>>>(D, 0.0, t_[0], t_[1], nullptr, nullptr, part_);
    k2_finish<<<1, kThreads, 0, st_>>>(part_, nblk_, out_);
    launches_ += 2;
    double o[2];
    if ((rc = read_out(2, o))) return rc;
    double dt = o[0], e = o[1];
    const int max_rec = opt.energies || opt.dts ? opt.max_rec : 0;
    int nrec = 0;
    auto record = [&]() {
        if (nrec < max_rec) {
            if (opt.energies) opt.energies[nrec] = e;
            if (opt.dts) opt.dts[nrec] = dt;
            nrec++;
        }
    };
    record();
    int niter = 1, status = 0;
    // DIIS history: slot of iteration m is m % nd; B over slots, by slot
    std::vector<double> B((size_t)kMaxDiis * kMaxDiis, 0.0);
    int pushed = 0;
    while (dt >= opt.tol && niter < opt.max_iter) {
        if (!std::isfinite(dt) || !std::isfinite(e)) {
            status = UEGCCD_ERR_NUMERIC;
            break;
        }
        if (nd > 0 && niter >= nd + 5 && pushed >= nd) {
            // GetTFromDIIS with a working solve (DIISCC.f90:52-131): one set of coefficients
            // for both channels
            std::vector<double> Bs((size_t)nd * nd), c;
            for (int p = 0; p < nd; p++)
                for (int q = 0; q < nd; q++) Bs[p * nd + q] = B[p * kMaxDiis + q];
            if (pulay_solve(nd, Bs, c)) {
                Coef cf{};
                for (int q = 0; q < nd; q++) cf.c[q] = c[q];
                k2_extrap<<<nblk_, kThreads, 0, st_>>>((int)n_, nd, cf, ht_[0], drpa ? nullptr : ht_[1], t_[0], t_[1]);
                launches_++;
            }
        }
        if ((rc = residual(drpa, mask))) return rc;
        const int slot = nd > 0 ? pushed % nd : 0;
        double *rab = nd > 0 ? hr_[0] + (int64_t)slot * n_ : nullptr;
        double *rba = nd > 0 && !drpa ? hr_[1] + (int64_t)slot * n_ : nullptr;
        double *hab = nd > 0 ? ht_[0] + (int64_t)slot * n_ : nullptr;
        double *hba = nd > 0 && !drpa ? ht_[1] + (int64_t)slot * n_ : nullptr;
        if (drpa)
            k2_update<true><<<nblk_, kThreads, 0, st_>>>(D, df, t_[0], t_[1], g_[0], g_[1], rab, rba, hab, hba, part_);
        else
            k2_update<false><<<nblk_, kThreads, 0, st_>>>(D, df, t_[0], t_[1], g_[0], g_[1], rab, rba, hab, hba, part_);
        k2_finish<<<1, kThreads, 0, st_>>>(part_, nblk_, out_);
        launches_ += 2;
        if (nd > 0) {
            const int nb = std::min(nblk_, 2 * 148);
            k2_dots<<<nb, kThreads, 0, st_>>>((int)n_, nd, slot, hr_[0], drpa ? nullptr : hr_[1], part_ + 2 * nblk_);
            k2_dots_finish<<<1, kThreads, 0, st_>>>(part_ + 2 * nblk_, nb, nd, out_ + 2);
            launches_ += 2;
        }
        double ob[2 + kMaxDiis];
        if ((rc = read_out(2 + nd, ob))) return rc;
        dt = ob[0];
        e = ob[1];
        if (nd > 0) {
            for (int q = 0; q < nd; q++) B[slot * kMaxDiis + q] = B[q * kMaxDiis + slot] = ob[2 + q];
            pushed++;
        }
        niter++;
        record();
    }
    if (status == 0 && (!std::isfinite(dt) || !std::isfinite(e))) status = UEGCCD_ERR_NUMERIC;
    // the final residual (CCD.f90:103-107; dRPA.f90:98-101)
    if ((rc = residual(drpa, mask))) return rc;
    if (drpa)
        k2_stats<true><<<nblk_, kThreads, 0, st_>>>(D, 1.0, t_[0], t_[1], g_[0], g_[1], part_);
    else
        k2_stats<false><<<nblk_, kThreads, 0, st_>>>(D, 0.0, t_[0], t_[1], g_[0], g_[1], part_);
    k2_finish<<<1, kThreads, 0, st_>>>(part_, nblk_, out_);
    launches_ += 2;
    if ((rc = read_out(2, o))) return rc;
    const double maxres = o[0];
    TCU(cudaEventRecord(ev1_, st_));
    TCU(cudaEventSynchronize(ev1_));
    float ms = 0.f;
    TCU(cudaEventElapsedTime(&ms, ev0_, ev1_));
    // amplitudes back in the reference layout
    TCU(cudaMemcpyAsync(t_abab, t_[0], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    if (!drpa && t_abba) TCU(cudaMemcpyAsync(t_abba, t_[1], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
    TCU(cudaStreamSynchronize(st_));
    if (!drpa && t_aaaa) {
        if (t_abba) {
            for (int64_t x = 0; x < n_; x++) t_aaaa[x] = t_abab[x] + t_abba[x];
        } else {
            std::vector<double> ba(n_);
            TCU(cudaMemcpyAsync(ba.data(), t_[1], n_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
            TCU(cudaStreamSynchronize(st_));
            for (int64_t x = 0; x < n_; x++) t_aaaa[x] = t_abab[x] + ba[x];
        }
    }
    res.ecorr = e;
    res.max_res = maxres;
    res.last_dt = dt;
    res.niter = niter;
    res.fail = maxres > opt.fail_ratio * opt.tol;
    // Ec(SOSEX) only when the dRPA solve did not fail (dRPA.f90:102-107)
    res.ecorr_sosex = drpa && !res.fail ? o[1] : 0.0;
    res.n_recorded = nrec;
    res.kernel_launches = launches_;
    res.gpu_ms = ms;
    res.ndiis = nd;
    if (status == UEGCCD_ERR_NUMERIC || !std::isfinite(maxres)) {
        res.status = UEGCCD_ERR_NUMERIC;
        return tfail(UEGCCD_ERR_NUMERIC, "non-finite amplitudes or energy");
    }
    res.status = (res.fail || (dt >= opt.tol && niter >= opt.max_iter)) ? UEGCCD_NOT_CONVERGED : UEGCCD_OK;
    return res.status;
}

}  // namespace uegccd

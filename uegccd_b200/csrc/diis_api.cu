// diis_api.cu -- the DIIS entry points of the reference's DIISCC module
// (SetUpDIISCC, GetTFromDIIS, ShutDownDIISCC; DIISCC.f90:10-155) for a host that
// keeps its own iteration loop.  The history of NDIIS (T, R) pairs lives on the
// device; the host passes each new pair in and receives the next T.
//
// Two schemes, as in the solve options:
//   REPLAY  the reference's behaviour.  Its B-matrix block is overwritten with ones
//           (DIISCC.f90:110-111), so DGESV meets a singular matrix, C stays
//           (0,...,0,1) and the next T is the newest OldT2 (DIISCC.f90:114-125).
//           No dot products are formed.
//   DIIS    the Pulay extrapolation the routine's comments describe
//           (DIISCC.f90:66-88): B(i,j) = R(i).R(j), [B 1; 1 0][c; y] = [0; 1],
//           T = sum c(i) T(i), over the pairs pushed so far.
// Dot products and the extrapolation run on the device in a fixed order
// (deterministic); the (NDIIS+1)^2 solve runs on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/uegccd.h"
#include "kernels.h"

namespace uegccd {
int set_last_error(int code, const char *msg);
int device_ok();
}

namespace {

constexpr int kDiisCap = 16;
constexpr int kDotThreads = 256;
constexpr int kDotBlocks = 148 * 4;

int fail(int code, const std::string &m) { return uegccd::set_last_error(code, m.c_str()); }

#define CUD(call)                                                                                       \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// part[blk * kDiisCap + k] = sum over this block's grid-stride share of r[slot] . r[k],
// for the k in use; fixed order per block (deterministic for a fixed grid).
__global__ void __launch_bounds__(kDotThreads)
    k_diis_dots(const double *__restrict__ r, int64_t n, int slot, int nuse, double *__restrict__ part)
{
    __shared__ double red[kDotThreads / 32][kDiisCap];
    const double *rs = r + (int64_t)slot * n;
    double acc[kDiisCap];
#pragma unroll
    for (int k = 0; k < kDiisCap; k++) acc[k] = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * kDotThreads + threadIdx.x; e < n; e += (int64_t)gridDim.x * kDotThreads) {
        const double x = rs[e];
#pragma unroll
        for (int k = 0; k < kDiisCap; k++)
            if (k < nuse) acc[k] += x * r[(int64_t)k * n + e];
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < kDiisCap; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (l == 0) red[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < nuse) {
        double v = 0.0;
        for (int q = 0; q < kDotThreads / 32; q++) v += red[q][threadIdx.x];
        part[(int64_t)blockIdx.x * kDiisCap + threadIdx.x] = v;
    }
}

// row[k] = sum over blocks of part[blk * kDiisCap + k], blocks in order
__global__ void k_diis_rows(const double *__restrict__ part, int nblk, int nuse, double *__restrict__ row)
{
    const int k = threadIdx.x;
    if (k >= nuse) return;
    double v = 0.0;
    for (int b = 0; b < nblk; b++) v += part[(int64_t)b * kDiisCap + k];
    row[k] = v;
}

// out = sum_k c[k] t[slot_k], k in the order given
__global__ void k_diis_combine(const double *__restrict__ t, int64_t n, int nuse, const int *__restrict__ slots,
                               const double *__restrict__ c, double *__restrict__ out)
{
    __shared__ double cs[kDiisCap];
    __shared__ int ss[kDiisCap];
    if (threadIdx.x < nuse) {
        cs[threadIdx.x] = c[threadIdx.x];
        ss[threadIdx.x] = slots[threadIdx.x];
    }
    __syncthreads();
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int k = 0; k < nuse; k++) v += cs[k] * t[(int64_t)ss[k] * n + e];
        out[e] = v;
    }
}

// [B 1; 1 0][c; y] = [0; 1] with B scaled by its largest diagonal; Gaussian
// elimination with partial pivoting.  False if singular.
bool pulay_solve(const std::vector<double> &B, int m, std::vector<double> &c)
{
    const int n = m + 1;
    double scale = 0.0;
    for (int i = 0; i < m; i++) scale = std::max(scale, B[i * kDiisCap + i]);
    if (!(scale > 0.0) || !std::isfinite(scale)) return false;
    std::vector<double> A((size_t)n * (n + 1), 0.0);
    auto a = [&](int i, int j) -> double & { return A[(size_t)i * (n + 1) + j]; };
    for (int i = 0; i < m; i++) {
        for (int j = 0; j < m; j++) a(i, j) = B[i * kDiisCap + j] / scale;
        a(i, m) = 1.0;
        a(m, i) = 1.0;
    }
    a(m, n) = 1.0;
    for (int k = 0; k < n; k++) {
        int p = k;
        for (int i = k + 1; i < n; i++)
            if (std::fabs(a(i, k)) > std::fabs(a(p, k))) p = i;
        if (std::fabs(a(p, k)) < 1e-14) return false;
        if (p != k)
            for (int j = 0; j <= n; j++) std::swap(a(k, j), a(p, j));
        for (int i = k + 1; i < n; i++) {
            const double f = a(i, k) / a(k, k);
            for (int j = k; j <= n; j++) a(i, j) -= f * a(k, j);
        }
    }
    for (int k = n - 1; k >= 0; k--) {
        double x = a(k, n);
        for (int j = k + 1; j < n; j++) x -= a(k, j) * a(j, n);
        a(k, n) = x / a(k, k);
    }
    c.assign(m, 0.0);
    for (int i = 0; i < m; i++) c[i] = a(i, n);
    return true;
}

}  // namespace

struct UegccdDiis {
    int64_t n = 0;
    int ndiis = 0, scheme = 0;
    int count = 0;        // pairs pushed, at most ndiis kept
    int newest = -1;      // slot of the newest T (the start amplitudes before any push)
    double *t = nullptr, *r = nullptr;          // ndiis slots of n doubles each
    double *part = nullptr, *row = nullptr, *c = nullptr, *out = nullptr;
    int *slots = nullptr;
    std::vector<double> B;                      // kDiisCap x kDiisCap, by slot
    cudaStream_t stream = nullptr;
    int dev = -1;                               // the device the history lives on
    ~UegccdDiis()
    {
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : {(void *)t, (void *)r, (void *)part, (void *)row, (void *)c, (void *)out, (void *)slots})
            if (p) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

int uegccd_diis_create(int64_t n, int32_t ndiis, int32_t scheme, const double *t0, UegccdDiis **out)
{
    if (!out) return fail(UEGCCD_ERR_ARG, "null out");
    *out = nullptr;
    if (n <= 0 || ndiis < 1 || ndiis > kDiisCap) return fail(UEGCCD_ERR_ARG, "n must be > 0 and ndiis in [1, 16]");
    if (scheme != UEGCCD_REPLAY && scheme != UEGCCD_DIIS) return fail(UEGCCD_ERR_ARG, "unknown scheme");
    if (int rc = uegccd::device_ok()) return rc;
    auto *d = new UegccdDiis;
    cudaGetDevice(&d->dev);   // the history stays on the device current now
    d->n = n;
    d->ndiis = ndiis;
    d->scheme = scheme;
    d->B.assign(kDiisCap * kDiisCap, 0.0);
    cudaError_t e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    const size_t bytes = (size_t)ndiis * n * sizeof(double);
    if (e == cudaSuccess) e = cudaMalloc(&d->t, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d->r, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d->part, (size_t)kDotBlocks * kDiisCap * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d->row, kDiisCap * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d->c, kDiisCap * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d->slots, kDiisCap * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d->out, n * sizeof(double));
    if (e != cudaSuccess) {
        delete d;
        return fail(UEGCCD_ERR_ALLOC, std::string("DIIS history: ") + cudaGetErrorString(e));
    }
    if (t0) {  // SetUpDIISCC: OldT2(:,:,:,NDIIS) = T2
        e = cudaMemcpyAsync(d->t, t0, n * sizeof(double), cudaMemcpyHostToDevice, d->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
        if (e != cudaSuccess) {
            delete d;
            return fail(UEGCCD_ERR_CUDA, std::string("DIIS start amplitudes: ") + cudaGetErrorString(e));
        }
        d->newest = 0;
    }
    *out = d;
    return UEGCCD_OK;
}

int uegccd_diis_push(UegccdDiis *d, const double *t, const double *r)
{
    if (!d || !t || !r) return fail(UEGCCD_ERR_ARG, "null argument");
    uegccd::DeviceScope on_dev(d->dev);
    if (on_dev.rc != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(on_dev.rc));
    // the start amplitudes (no residual) hold slot 0 until the first push replaces them
    const int slot = d->count == 0 ? 0 : (d->newest + 1) % d->ndiis;
    const size_t bytes = d->n * sizeof(double);
    CUD(cudaMemcpyAsync(d->t + (int64_t)slot * d->n, t, bytes, cudaMemcpyHostToDevice, d->stream));
    CUD(cudaMemcpyAsync(d->r + (int64_t)slot * d->n, r, bytes, cudaMemcpyHostToDevice, d->stream));
    d->newest = slot;
    d->count = std::min(d->count + 1, d->ndiis);
    if (d->scheme == UEGCCD_DIIS) {
        // B row of the new residual against every slot in use (slots 0..count-1)
        const int nuse = d->count;
        k_diis_dots<<<kDotBlocks, kDotThreads, 0, d->stream>>>(d->r, d->n, slot, nuse, d->part);
        k_diis_rows<<<1, 32, 0, d->stream>>>(d->part, kDotBlocks, nuse, d->row);
        CUD(cudaGetLastError());
        double row[kDiisCap];
        CUD(cudaMemcpyAsync(row, d->row, nuse * sizeof(double), cudaMemcpyDeviceToHost, d->stream));
        CUD(cudaStreamSynchronize(d->stream));
        for (int k = 0; k < nuse; k++) d->B[slot * kDiisCap + k] = d->B[k * kDiisCap + slot] = row[k];
    } else {
        CUD(cudaStreamSynchronize(d->stream));
    }
    return UEGCCD_OK;
}

int uegccd_diis_get_t(UegccdDiis *d, int32_t niter, double *t2)
{
    if (!d || !t2) return fail(UEGCCD_ERR_ARG, "null argument");
    uegccd::DeviceScope on_dev(d->dev);
    if (on_dev.rc != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(on_dev.rc));
    if (d->newest < 0) return fail(UEGCCD_ERR_ARG, "no amplitudes: pass t0 or push a pair first");
    const size_t bytes = d->n * sizeof(double);
    std::vector<double> c;
    const int m = d->count;
    // slots oldest first: the combination runs in age order
    std::vector<int> order(m);
    for (int k = 0; k < m; k++) order[k] = (d->newest + 1 + k + (d->ndiis - m)) % d->ndiis;
    // the reference extrapolates from NIter >= NDIIS + IWait, IWait = 5 (DIISCC.f90:59,94)
    if (d->scheme == UEGCCD_DIIS && niter >= d->ndiis + 5 && m >= 2) {
        std::vector<double> Bm(kDiisCap * kDiisCap, 0.0);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < m; j++) Bm[i * kDiisCap + j] = d->B[order[i] * kDiisCap + order[j]];
        if (pulay_solve(Bm, m, c)) {
            CUD(cudaMemcpyAsync(d->c, c.data(), m * sizeof(double), cudaMemcpyHostToDevice, d->stream));
            CUD(cudaMemcpyAsync(d->slots, order.data(), m * sizeof(int), cudaMemcpyHostToDevice, d->stream));
            k_diis_combine<<<148 * 4, 256, 0, d->stream>>>(d->t, d->n, m, d->slots, d->c, d->out);
            CUD(cudaGetLastError());
            CUD(cudaMemcpyAsync(t2, d->out, bytes, cudaMemcpyDeviceToHost, d->stream));
            CUD(cudaStreamSynchronize(d->stream));
            return UEGCCD_OK;
        }
    }
    // REPLAY (the reference's singular solve), too few pairs, or a singular B: the newest T
    CUD(cudaMemcpyAsync(t2, d->t + (int64_t)d->newest * d->n, bytes, cudaMemcpyDeviceToHost, d->stream));
    CUD(cudaStreamSynchronize(d->stream));
    return UEGCCD_OK;
}

int uegccd_diis_destroy(UegccdDiis *d)
{
    if (!d) return UEGCCD_OK;
    uegccd::DeviceScope on_dev(d->dev);
    delete d;
    return UEGCCD_OK;
}

}  // extern "C"

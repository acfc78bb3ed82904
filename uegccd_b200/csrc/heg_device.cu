// heg_device.cu -- the plane-wave set-up of many twists at once on the device: for every
// twist k_s the reference's ChangeTwist (HEG.f90:551-578), i.e. SetupBasis (HEG.f90:150-324:
// the candidates |n|^2 <= MaxKPoint sorted by the twisted |n + k_s|^2 with a stable sort,
// truncated by fcut and corefcut), the HF eigenvalues (HEG.f90:581-603) and the HF energy
// (print_HF, HEG.f90:605-615), at the set-up's current rS.
//
// One CTA per twist.  The stable sort is a bitonic sort of (key, candidate index) pairs: with
// the index breaking ties the order is total, so the result is the stable order the
// reference's bubble sort leaves (equal keys keep their loop order).  Every floating-point
// expression is written with explicitly rounded operations (__dmul_rn, __dadd_rn, ...) in
// the host code's evaluation order, so no multiply-add is contracted and the keys, wave
// vectors, eigenvalues and energies are bit-equal to heg_host.cpp's.
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/uegccd.h"
#include "../../include/uegccd_host.h"
#include "heg_device.h"

namespace uegccd {
int set_last_error(int code, const char *msg);
int device_ok();
}

namespace {

constexpr int kMaxCand = 4096;   // candidates a twist sorts in shared memory
constexpr int kThreads = 512;
constexpr double kFourPi = 4.0 * 3.1415926535897932384626433833;   // 4.0 * kPi (Constants.f90:7)

int fail(int code, const std::string &m) { return uegccd::set_last_error(code, m.c_str()); }

struct TwistArgs {
    const int4 *cand;       // ncand untwisted n vectors
    int ncand, npow2;       // npow2: sort length (power of two >= ncand)
    int nao, mcore, nocc;
    double kscale, inv_omega, madelung, gap, xf, half_nel_madelung;
    const double *twists;   // 3 per twist
    int32_t *nvec;          // per twist NAO x 3, column-major (HEGData%nVec)
    double *eigen;          // per twist NAO
    double *kvec;           // per twist NAO x 3, row-major (scratch of the eigenvalue pass)
    double *ehf;            // per twist: E_HF as the set-up stores it (hf_energy)
};

__global__ void __launch_bounds__(kThreads) k_twist_setup(TwistArgs A)
{
    __shared__ double key[kMaxCand];
    __shared__ int idx[kMaxCand];
    const int tw = blockIdx.x;
    const double t0 = A.twists[3 * tw], t1 = A.twists[3 * tw + 1], t2 = A.twists[3 * tw + 2];
    // keys: nt = n + k_s, |nt|^2 = (nt0 nt0 + nt1 nt1) + nt2 nt2 (SetupBasis's expression)
    for (int c = threadIdx.x; c < A.npow2; c += blockDim.x) {
        if (c < A.ncand) {
            const int4 n = A.cand[c];
            const double a = __dadd_rn((double)n.x, t0), b = __dadd_rn((double)n.y, t1), d = __dadd_rn((double)n.z, t2);
            key[c] = __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(d, d));
            idx[c] = c;
        } else {
            key[c] = __longlong_as_double(0x7ff0000000000000LL);   // +Inf: padding sorts last
            idx[c] = c;
        }
    }
    __syncthreads();
    // bitonic sort, ascending by (key, idx)
    for (int size = 2; size <= A.npow2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < A.npow2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool up = (i & size) == 0;
                    const double ki = key[i], kj = key[j];
                    const int ii = idx[i], ij = idx[j];
                    const bool gt = ki > kj || (ki == kj && ii > ij);
                    if (gt == up) {
                        key[i] = kj;
                        key[j] = ki;
                        idx[i] = ij;
                        idx[j] = ii;
                    }
                }
            }
            __syncthreads();
        }
    }
    // the basis: sorted entries 0 .. nocc-1, then (past the core shell) from mcore on
    int32_t *nv = A.nvec + (int64_t)tw * A.nao * 3;
    double *kv = A.kvec + (int64_t)tw * A.nao * 3;
    for (int p = threadIdx.x; p < A.nao; p += blockDim.x) {
        const int off = (p + 1 > A.nocc) ? A.mcore - A.nocc : 0;
        const int4 n = A.cand[idx[p + off]];
        nv[p] = n.x;
        nv[p + A.nao] = n.y;
        nv[p + 2 * A.nao] = n.z;
        kv[3 * p] = __dmul_rn(__dadd_rn((double)n.x, t0), A.kscale);
        kv[3 * p + 1] = __dmul_rn(__dadd_rn((double)n.y, t1), A.kscale);
        kv[3 * p + 2] = __dmul_rn(__dadd_rn((double)n.z, t2), A.kscale);
    }
    __syncthreads();
    // eigenvalues (form_eigen): e = 0.5 |k_p|^2, then over the occupied q in order
    for (int p = threadIdx.x; p < A.nao; p += blockDim.x) {
        const double k0 = kv[3 * p], k1 = kv[3 * p + 1], k2 = kv[3 * p + 2];
        double e = __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)), __dmul_rn(k2, k2)));
        for (int q = 0; q < A.nocc; q++) {
            if (q != p) {
                const double q1 = __dsub_rn(k0, kv[3 * q]), q2 = __dsub_rn(k1, kv[3 * q + 1]),
                             q3 = __dsub_rn(k2, kv[3 * q + 2]);
                const double qq = __dadd_rn(__dadd_rn(__dmul_rn(q1, q1), __dmul_rn(q2, q2)), __dmul_rn(q3, q3));
                e = __dsub_rn(e, __dmul_rn(__dmul_rn(A.inv_omega, __ddiv_rn(kFourPi, qq)), A.xf));
            } else {
                e = __dsub_rn(__dadd_rn(e, A.madelung), A.gap);
            }
        }
        A.eigen[(int64_t)tw * A.nao + p] = e;
    }
    // E_HF (hf_energy): one thread, the host's summation order
    if (threadIdx.x == 0) {
        double ehf = 0.0;
        const double half_inv = __dmul_rn(0.5, A.inv_omega);
        for (int p = 0; p < A.nocc; p++) {
            const double k0 = kv[3 * p], k1 = kv[3 * p + 1], k2 = kv[3 * p + 2];
            ehf = __dadd_rn(ehf, __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(k0, k0), __dmul_rn(k1, k1)),
                                                          __dmul_rn(k2, k2))));
            for (int q = 0; q < A.nocc; q++) {
                if (q == p) continue;
                const double q1 = __dsub_rn(k0, kv[3 * q]), q2 = __dsub_rn(k1, kv[3 * q + 1]),
                             q3 = __dsub_rn(k2, kv[3 * q + 2]);
                const double qq = __dadd_rn(__dadd_rn(__dmul_rn(q1, q1), __dmul_rn(q2, q2)), __dmul_rn(q3, q3));
                ehf = __dsub_rn(ehf, __dmul_rn(half_inv, __ddiv_rn(kFourPi, qq)));
            }
        }
        A.ehf[tw] = __dadd_rn(__dmul_rn(ehf, 2.0), A.half_nel_madelung);
    }
}

#define CUH(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            rc = fail(UEGCCD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_));              \
            goto done;                                                                                 \
        }                                                                                              \
    } while (0)

}  // namespace

extern "C" int uegccd_heg_twists(const UegccdHeg *h, int32_t ntwist, const double *twists, int32_t *nvec,
                                 double *eigen, double *ehf)
{
    if (!h || ntwist <= 0 || !twists || !nvec || !eigen) return fail(UEGCCD_ERR_ARG, "bad argument");
    uegccd::HegTwistSetup S;
    int rc = uegccd::heg_twist_setup(h, &S);
    if (rc) return fail(rc, uegccd_host_last_error());
    const int ncand = (int)S.cand.size();
    if (ncand > kMaxCand)
        return fail(UEGCCD_ERR_UNSUPPORTED, "more than " + std::to_string(kMaxCand) +
                                                " plane-wave candidates for the device set-up (MaxKPoint too large)");
    if ((rc = uegccd::device_ok())) return rc;
    int npow2 = 1;
    while (npow2 < ncand) npow2 <<= 1;
    const int nao = S.nao, nocc = S.nel / 2;
    std::vector<int4> cand(ncand);
    for (int c = 0; c < ncand; c++) cand[c] = make_int4(S.cand[c][0], S.cand[c][1], S.cand[c][2], 0);
    const size_t nv_n = (size_t)ntwist * nao * 3;
    int4 *d_cand = nullptr;
    double *d_tw = nullptr, *d_eig = nullptr, *d_kv = nullptr, *d_ehf = nullptr;
    int32_t *d_nv = nullptr;
    cudaStream_t st = nullptr;
    TwistArgs A;
    std::vector<double> ehf_h(ntwist);
    CUH(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CUH(cudaMalloc(&d_cand, sizeof(int4) * ncand));
    CUH(cudaMalloc(&d_tw, sizeof(double) * 3 * ntwist));
    CUH(cudaMalloc(&d_nv, sizeof(int32_t) * nv_n));
    CUH(cudaMalloc(&d_eig, sizeof(double) * ntwist * (size_t)nao));
    CUH(cudaMalloc(&d_kv, sizeof(double) * nv_n));
    CUH(cudaMalloc(&d_ehf, sizeof(double) * ntwist));
    CUH(cudaMemcpyAsync(d_cand, cand.data(), sizeof(int4) * ncand, cudaMemcpyHostToDevice, st));
    CUH(cudaMemcpyAsync(d_tw, twists, sizeof(double) * 3 * ntwist, cudaMemcpyHostToDevice, st));
    A.cand = d_cand;
    A.ncand = ncand;
    A.npow2 = npow2;
    A.nao = nao;
    A.mcore = S.mcore;
    A.nocc = nocc;
    A.kscale = S.kscale;
    A.inv_omega = S.inv_omega;
    A.madelung = S.madelung;
    A.gap = S.gap;
    A.xf = S.exchangefactor;
    A.half_nel_madelung = S.madelung * 0.5 * S.nel;   // hf_energy: Madelung * 0.5 * N
    A.twists = d_tw;
    A.nvec = d_nv;
    A.eigen = d_eig;
    A.kvec = d_kv;
    A.ehf = d_ehf;
    k_twist_setup<<<ntwist, kThreads, 0, st>>>(A);
    CUH(cudaGetLastError());
    CUH(cudaMemcpyAsync(nvec, d_nv, sizeof(int32_t) * nv_n, cudaMemcpyDeviceToHost, st));
    CUH(cudaMemcpyAsync(eigen, d_eig, sizeof(double) * ntwist * (size_t)nao, cudaMemcpyDeviceToHost, st));
    CUH(cudaMemcpyAsync(ehf_h.data(), d_ehf, sizeof(double) * ntwist, cudaMemcpyDeviceToHost, st));
    CUH(cudaStreamSynchronize(st));
    if (ehf) std::memcpy(ehf, ehf_h.data(), sizeof(double) * ntwist);
done:
    for (void *p : {(void *)d_cand, (void *)d_tw, (void *)d_nv, (void *)d_eig, (void *)d_kv, (void *)d_ehf})
        if (p) cudaFree(p);
    if (st) cudaStreamDestroy(st);
    return rc;
}

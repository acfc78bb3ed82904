// mp2_static.cu -- E(2) of one system without any device allocation.
//
// uegccd_mp2_energy_static computes the same MP2 energy as uegccd_mp2 (the sum
// of k_mp2's per-amplitude terms), but every buffer it needs on the device --
// the staged eigenvalues and plane-wave vectors, a dense lattice lookup from
// n to orbital, the per-block partial sums and the result -- lives in one
// file-scope device array of fixed size, g_static_scratch.  Nothing is
// allocated or freed, by this code or by a library on its behalf.
//
// It serves callers that cannot allocate device memory at the point of the
// call: a host whose device memory is already handed out to its own pool
// allocator, or one that runs other streams concurrently and cannot accept the
// device-wide synchronisation cudaFree implies.
//
// Limits: NAO <= kStaticMaxOrb and every plane-wave component |n_d| <=
// kStaticMaxRadius; larger systems are refused with UEGCCD_ERR_ARG.
//
// Sharing: all calls on a device use the same array.  Two calls in flight at
// the same time on one device (different streams or host threads) race on it
// and give wrong results; serialise them.  No region has to start at zero:
// every call resets the lattice to "no orbital" itself, every block writes its
// own partial sum and the reduction overwrites the result.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (which may load the module into the context) and keeps it
// for the life of the process.  A cudaDeviceReset unloads the module, so the kept address
// is no longer valid afterwards: do not use this entry point across a reset.
//
// Every call copies E(2) back into host memory and synchronises `stream` before
// it returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/uegccd.h"

namespace uegccd {
int set_last_error(int code, const char *msg);
}

namespace {

constexpr int kStaticMaxOrb = 2048;                       // orbitals
constexpr int kStaticMaxRadius = 31;                      // |n_d| bound
constexpr int kStaticSide = 2 * kStaticMaxRadius + 1;     // 63
constexpr int kStaticLattice = kStaticSide * kStaticSide * kStaticSide;
constexpr int kStaticThreads = 256;
constexpr int kStaticMaxBlocks = 148 * 8;
constexpr int kStaticMaxDevices = 64;

// byte offsets inside the scratch array (each a multiple of 256)
constexpr size_t kOffEigen = 0;
constexpr size_t kOffNvec = kOffEigen + sizeof(double) * kStaticMaxOrb;
constexpr size_t kOffLattice = kOffNvec + ((sizeof(int32_t) * 3 * kStaticMaxOrb + 255) / 256) * 256;
constexpr size_t kOffPartial = kOffLattice + ((sizeof(int32_t) * (size_t)kStaticLattice + 255) / 256) * 256;
constexpr size_t kOffResult = kOffPartial + sizeof(double) * kStaticMaxBlocks;
constexpr size_t kStaticScratchBytes = kOffResult + 256;  // 1,050,880 bytes (1.05 MB)

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_setup_mu;
void *g_scratch_ptr[kStaticMaxDevices] = {};

constexpr double kPi = 3.1415926535897932384626433833;  // Constants.f90:7

int fail(int code, const std::string &m) { return uegccd::set_last_error(code, m.c_str()); }

#define CUS(call)                                                                                      \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(UEGCCD_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// Lattice reset: every cell "no orbital" (-1).
__global__ void k_static_lattice_clear(int32_t *lat, int n)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) lat[k] = -1;
}

// lat[(x + r) * side^2 + (y + r) * side + (z + r)] = p for orbital p with n_p = (x, y, z).
__global__ void k_static_lattice_fill(const int32_t *nvec, int M, int r, int32_t *lat)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const int side = 2 * r + 1;
    const int x = nvec[p], y = nvec[p + M], z = nvec[p + 2 * M];
    lat[((x + r) * side + (y + r)) * side + (z + r)] = p;
}

__device__ __forceinline__ double coulomb(double L, int q2) { return 1.0 / (L * kPi * (double)q2); }

// The MP2 sum over the dense (i, j, a) index space, grid-stride; b from the lattice.
// Per element: t = v(i-a) / (e_i + e_j - e_a - e_b), term = t (2 v(i-a) - v(i-b))
// (MP2.f90:56-74 after the a <-> b re-indexing; the per-element arithmetic of k_mp2).
// Block partial sums go to part[blockIdx.x].
__global__ void __launch_bounds__(kStaticThreads) k_mp2_static(const double *eigen, const int32_t *nvec,
                                                               const int32_t *lat, int O, int M, int r, double L,
                                                               double *part)
{
    const int V = M - O, side = 2 * r + 1;
    const int64_t total = (int64_t)O * O * V;
    double e = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int a = O + (int)(k % V);
        const int64_t ij = k / V;
        const int j = (int)(ij % O), i = (int)(ij / O);
        const int x = nvec[i] + nvec[j] - nvec[a];
        const int y = nvec[i + M] + nvec[j + M] - nvec[a + M];
        const int z = nvec[i + 2 * M] + nvec[j + 2 * M] - nvec[a + 2 * M];
        if (x < -r || x > r || y < -r || y > r || z < -r || z > r) continue;
        const int b = lat[((x + r) * side + (y + r)) * side + (z + r)];
        if (b < O) continue;  // not in the basis, or occupied
        int qa = 0, qb = 0;
        for (int d = 0; d < 3; d++) {
            const int da = nvec[i + d * M] - nvec[a + d * M], db = nvec[i + d * M] - nvec[b + d * M];
            qa += da * da;
            qb += db * db;
        }
        const double denom = eigen[i] + eigen[j] - eigen[a] - eigen[b];
        const double via = coulomb(L, qa), vib = coulomb(L, qb);
        const double t = via / denom;
        e += t * (2.0 * via - vib);
    }
    __shared__ double s[kStaticThreads / 32];
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        e = threadIdx.x < kStaticThreads / 32 ? s[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
        if (threadIdx.x == 0) part[blockIdx.x] = e;
    }
}

// Fixed-order sum of the block partials (one block): deterministic.
__global__ void __launch_bounds__(kStaticThreads) k_mp2_static_reduce(const double *part, int n, double *out)
{
    double e = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) e += part[k];
    __shared__ double s[kStaticThreads / 32];
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        e = threadIdx.x < kStaticThreads / 32 ? s[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
        if (threadIdx.x == 0) *out = e;
    }
}

// The device address of g_static_scratch on the current device, looked up once per device.
int scratch_for_current_device(unsigned char **out)
{
    int dev = -1;
    CUS(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) return fail(UEGCCD_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess || !p)
            return fail(UEGCCD_ERR_CUDA, std::string("cudaGetSymbolAddress(g_static_scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_ptr[dev]);
    return UEGCCD_OK;
}

}  // namespace

extern "C" int uegccd_mp2_energy_static(const UegccdSystem *sys, void *stream, double *e2)
{
    if (!sys || !e2 || !sys->eigen || !sys->nvec) return fail(UEGCCD_ERR_ARG, "null argument");
    const int O = sys->nocc, M = sys->nao;
    if (O <= 0 || M <= O) return fail(UEGCCD_ERR_ARG, "need 0 < nocc < nao");
    if (M > kStaticMaxOrb)
        return fail(UEGCCD_ERR_ARG, "nao " + std::to_string(M) + " exceeds the static scratch limit of " +
                                        std::to_string(kStaticMaxOrb) + " orbitals");
    if (!(sys->L > 0.0)) return fail(UEGCCD_ERR_ARG, "L must be positive");
    int r = 0;
    for (int p = 0; p < M; p++)
        for (int d = 0; d < 3; d++) {
            const int v = sys->nvec[p + (size_t)M * d];
            r = v < 0 ? (-v > r ? -v : r) : (v > r ? v : r);
        }
    if (r > kStaticMaxRadius)
        return fail(UEGCCD_ERR_ARG, "plane-wave component " + std::to_string(r) +
                                        " exceeds the static scratch limit of " + std::to_string(kStaticMaxRadius));
    const int side = 2 * r + 1;
    const int ncell = side * side * side;
    unsigned char *base = nullptr;
    if (int rc = scratch_for_current_device(&base)) return rc;
    double *d_eigen = reinterpret_cast<double *>(base + kOffEigen);
    int32_t *d_nvec = reinterpret_cast<int32_t *>(base + kOffNvec);
    int32_t *d_lat = reinterpret_cast<int32_t *>(base + kOffLattice);
    double *d_part = reinterpret_cast<double *>(base + kOffPartial);
    double *d_out = reinterpret_cast<double *>(base + kOffResult);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    const int64_t total = (int64_t)O * O * (M - O);
    int64_t want = (total + kStaticThreads - 1) / kStaticThreads;
    const int blocks = (int)(want < 1 ? 1 : (want > kStaticMaxBlocks ? kStaticMaxBlocks : want));

    CUS(cudaMemcpyAsync(d_eigen, sys->eigen, sizeof(double) * M, cudaMemcpyHostToDevice, st));
    CUS(cudaMemcpyAsync(d_nvec, sys->nvec, sizeof(int32_t) * 3 * M, cudaMemcpyHostToDevice, st));
    k_static_lattice_clear<<<(ncell + kStaticThreads - 1) / kStaticThreads, kStaticThreads, 0, st>>>(d_lat, ncell);
    k_static_lattice_fill<<<(M + kStaticThreads - 1) / kStaticThreads, kStaticThreads, 0, st>>>(d_nvec, M, r, d_lat);
    k_mp2_static<<<blocks, kStaticThreads, 0, st>>>(d_eigen, d_nvec, d_lat, O, M, r, sys->L, d_part);
    k_mp2_static_reduce<<<1, kStaticThreads, 0, st>>>(d_part, blocks, d_out);
    CUS(cudaGetLastError());
    double h = 0.0;
    CUS(cudaMemcpyAsync(&h, d_out, sizeof(double), cudaMemcpyDeviceToHost, st));
    CUS(cudaStreamSynchronize(st));
    *e2 = h;
    return UEGCCD_OK;
}

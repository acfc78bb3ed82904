// bench_peak.cu -- bench.py's measurement of the FP64 tensor-core peak of the current
// device: the roofline denominator of the FP64 DMMA kernels (the ladders and rings), which
// the measured-peaks record of the machine does not hold.  A register-only kernel issues
// independent mma.sync.m8n8k4.f64 chains (eight per warp, eight CTAs of four warps per SM)
// and is timed with CUDA events after one untimed launch.  Built into bench_peak.so beside
// bench.py; it is measurement tooling, not part of the library's ABI.
//
//   int bench_fp64_peak(double *tflops, char *msg, int msg_len);   0 ok, else a CUDA error
#include <cuda_runtime.h>

#include <cstdio>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(128) k_fp64_mma_probe(double *out, int iters)
{
    double d[kChains][2];
#pragma unroll
    for (int c = 0; c < kChains; c++) d[c][0] = d[c][1] = 0.0;
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 1.0 - 1e-9 * threadIdx.x;
    for (int it = 0; it < iters; it++)
#pragma unroll
        for (int c = 0; c < kChains; c++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(d[c][0]), "+d"(d[c][1])
                         : "d"(a), "d"(b));
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += d[c][0] + d[c][1];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // keeps the chains live
}

}  // namespace

extern "C" int bench_fp64_peak(double *tflops, char *msg, int msg_len)
{
    if (!tflops) return -1;
    int dev = 0, sms = 0, major = 0;
    cudaError_t e0q = cudaGetDevice(&dev);
    if (e0q == cudaSuccess) e0q = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e0q == cudaSuccess) e0q = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e0q != cudaSuccess || major != 10) {
        if (msg && msg_len > 0)
            std::snprintf(msg, (size_t)msg_len, "no sm_100 device: %s", cudaGetErrorString(e0q));
        return -2;
    }
    const int threads = 128, blocks = sms * 8, iters = 4096;
    double *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(double) * threads * blocks);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    float ms = 0.f;
    if (e == cudaSuccess) {
        k_fp64_mma_probe<<<blocks, threads>>>(out, iters);   // untimed
        cudaEventRecord(e0);
        k_fp64_mma_probe<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    if (e != cudaSuccess) {
        if (msg && msg_len > 0) std::snprintf(msg, (size_t)msg_len, "FP64 probe: %s", cudaGetErrorString(e));
        return -2;
    }
    const double flops = (double)blocks * (threads / 32) * iters * kChains * 512.0;  // 2*8*8*4 per mma
    *tflops = flops / (ms * 1e-3) / 1e12;
    return 0;
}

// FP32 FMA throughput probe: the measured denominator of the treecode roofline;
// and the double-precision reciprocal square root the FP64 traversals use,
// applied elementwise so that tests can compare it with CUDA's rsqrt(double).
#include <string>

#include "../../include/cagr.h"
#include "internal.h"

namespace {

constexpr int kChains = 8;  // independent FMA chains per thread (covers FMA latency)

__global__ void __launch_bounds__(256) k_fma_probe(int64_t iters, float b, float c, float* sink) {
    float a[kChains];
#pragma unroll
    for (int j = 0; j < kChains; j++) a[j] = float(threadIdx.x + j) * 1e-7f;
    for (int64_t it = 0; it < iters; it++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
#pragma unroll
            for (int j = 0; j < kChains; j++) a[j] = fmaf(a[j], b, c);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < kChains; j++) s += a[j];
    if (s == 1234.5f) sink[blockIdx.x] = s;  // keeps the chains alive; never true in practice
}

__global__ void k_rsqrt64(const double* __restrict__ in, double* __restrict__ out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = cagr::rsqrt_t(in[i]);
}

}  // namespace

extern "C" int cagr_probe_rsqrt64(const double* in_dev, double* out_dev, int64_t n,
                                  void* stream) {
    using cagr::set_error;
    if (n < 0 || (n > 0 && (!in_dev || !out_dev)))
        return set_error(CAGR_ERR_INVALID, "bad probe arguments");
    if (n == 0) return CAGR_OK;
    const int64_t blocks = (n + 255) / 256;
    if (blocks > 0x7fffffffLL) return set_error(CAGR_ERR_INVALID, "too many values");
    k_rsqrt64<<<(unsigned)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(in_dev,
                                                                                    out_dev, n);
    CAGR_CUDA(cudaGetLastError());
    return CAGR_OK;
}

extern "C" int cagr_probe_fp32_peak(int64_t iters, double* gflops, void* stream) {
    using cagr::set_error;
    if (!gflops || iters <= 0) return set_error(CAGR_ERR_INVALID, "bad probe arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    CAGR_CUDA(cudaGetDevice(&dev));
    CAGR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256;
    float* sink = nullptr;
    CAGR_CUDA(cudaMallocAsync(&sink, sizeof(float) * blocks, s));
    cudaEvent_t e0, e1;
    CAGR_CUDA(cudaEventCreate(&e0));
    CAGR_CUDA(cudaEventCreate(&e1));
    k_fma_probe<<<blocks, threads, 0, s>>>(iters / 8 + 1, 0.999999f, 1e-6f, sink);  // warm-up
    CAGR_CUDA(cudaEventRecord(e0, s));
    k_fma_probe<<<blocks, threads, 0, s>>>(iters, 0.999999f, 1e-6f, sink);
    CAGR_CUDA(cudaEventRecord(e1, s));
    CAGR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    CAGR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CAGR_CUDA(cudaFreeAsync(sink, s));
    CAGR_CUDA(cudaStreamSynchronize(s));
    const double flops = 2.0 * kChains * 16.0 * (double)iters * blocks * threads;
    *gflops = flops / (ms * 1e-3) / 1e9;
    return CAGR_OK;
}

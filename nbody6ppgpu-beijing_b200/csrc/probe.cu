// probe.cu -- measured FP32 FMA throughput of this GPU, the roofline
// denominator for the pairwise-gravity kernels (they are bound by the FP32
// pipe, not by HBM or tensor cores).  16 independent FFMA chains per thread,
// every SM filled; returns the best of three CUDA-event-timed runs in
// TFLOP/s (2 flops per FFMA).  No reference counterpart.
#include "nb6_common.cuh"

namespace {

constexpr int CHAINS = 16;

__global__ void __launch_bounds__(256) fma_probe(int iters, float a, float b, float *out) {
    float x[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) x[k] = (threadIdx.x + k) * 1.0e-3f;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < CHAINS; ++k) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < CHAINS; ++k) s += x[k];
    if (s == -1.2345f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" double nb6_fp32_peak_probe_(int *iters_in) {
    nb6_devinit_once(0);
    const int iters = (iters_in && *iters_in > 0) ? *iters_in : 20000;
    const int blocks = nb6_num_sms() * 8;
    const int threads = 256;
    float *out = nullptr;
    NB6_CUDA_CHECK(cudaMalloc(&out, sizeof(float) * blocks * threads));
    cudaEvent_t e0, e1;
    NB6_CUDA_CHECK(cudaEventCreate(&e0));
    NB6_CUDA_CHECK(cudaEventCreate(&e1));
    cudaStream_t st = nb6_stream();
    fma_probe<<<blocks, threads, 0, st>>>(iters / 10 + 1, 0.9999999f, 1.0e-7f, out);  // warm-up
    double best = 0.0;
    for (int r = 0; r < 3; ++r) {
        NB6_CUDA_CHECK(cudaEventRecord(e0, st));
        fma_probe<<<blocks, threads, 0, st>>>(iters, 0.9999999f, 1.0e-7f, out);
        NB6_CUDA_CHECK(cudaEventRecord(e1, st));
        NB6_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms = 0.f;
        NB6_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = 2.0 * CHAINS * (double)iters * blocks * threads;
        const double tf = flops / (ms * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    NB6_CUDA_CHECK(cudaEventDestroy(e0));
    NB6_CUDA_CHECK(cudaEventDestroy(e1));
    NB6_CUDA_CHECK(cudaFree(out));
    return best;
}

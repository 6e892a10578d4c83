// FP32 FMA throughput microbenchmark: the denominator of the FP32 roofline.
//
// Every thread runs eight independent fmaf chains (x = x*a + b) so that each
// SM sub-partition always has ready FMA instructions; a and b are kernel
// arguments (no constant folding) with |a| < 1, so the chains converge to
// b/(1-a) and never reach infinities or denormals.  The grid is a multiple of
// the SM count with several CTAs resident per SM.  FLOP = 2 per FMA lane.
//
// Built into its own library (libgpudemod_peak.so) so the product library's
// ABI stays the path's; only the benchmark loads it.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 8;

__global__ void __launch_bounds__(256) k_fma_peak(float* sink, int iters, float a, float b) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = 1e-3f * (float)(threadIdx.x + c);
    for (int i = 0; i < iters; i += kUnroll) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = fmaf(x[c], a, b);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    // never true for the arguments used; keeps the chains live
    if (s == -1.0f) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

// Measures the FP32 FMA rate of the current device.  `iters` FMAs per chain
// (a multiple of 8; 0 picks 8192), `ctas_per_sm` resident CTAs of 256 threads
// per SM (0 picks 8).  Writes TFLOP/s (2 flop per FMA) and the kernel time in
// ms of the best of `reps` launches (0 picks 5).  Returns 0 or a cudaError_t.
__attribute__((visibility("default"))) int gpud_peak_fp32_fma(int iters, int ctas_per_sm, int reps, double* tflops,
                                                              double* ms_out) {
    if (!tflops || !ms_out) return -1;
    if (iters <= 0) iters = 8192;
    iters = (iters + kUnroll - 1) / kUnroll * kUnroll;
    if (ctas_per_sm <= 0) ctas_per_sm = 8;
    if (reps <= 0) reps = 5;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return (int)e;
    const int threads = 256, blocks = sms * ctas_per_sm;
    float* sink = nullptr;
    e = cudaMalloc(&sink, (size_t)blocks * threads * sizeof(float));
    if (e != cudaSuccess) return (int)e;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_fma_peak<<<blocks, threads>>>(sink, iters, 0.999f, 1e-4f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < reps && (e = cudaGetLastError()) == cudaSuccess; ++r) {
        cudaEventRecord(e0);
        k_fma_peak<<<blocks, threads>>>(sink, iters, 0.999f, 1e-4f);
        cudaEventRecord(e1);
        e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return (int)e;
    const double flop = 2.0 * kChains * (double)iters * (double)blocks * threads;
    *ms_out = best;
    *tflops = flop / (best * 1e-3) / 1e12;
    return 0;
}

}  // extern "C"

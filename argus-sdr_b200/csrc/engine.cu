// engine.cu -- the front end of the reference's single-signal Engine on the
// device: Engine.ShiftFilterDecimate (internal/demod/gpudemod/gpudemod.go:325-350)
// and the shift / FIR / decimate stages of Engine.Demod (gpudemod.go:359-427).
//
// The reference runs these stages with its CPU dsp functions (ShiftFilterDecimate
// always; Demod whenever its GPU result fails the CPU comparison, which the
// shift and decimation stages do for any non-trivial input), so the device path
// reproduces the CPU semantics:
//   dsp.FreqShift (dsp/freqshift.go:6-23): the phase starts at 0 every call and
//     is incremented before use by float64 additions of inc = -2*pi*offset/fs;
//     the rotation is float64 cos/sin with the products rounded once to float32;
//   dsp.ApplyFIR (dsp/fir.go:31-50): zero history, float64 accumulation;
//   dsp.Decimate (dsp/fir.go:84-95): every decim-th sample from index 0,
//     ceil(n / decim) outputs.
// The FIR is evaluated only at the kept outputs.  The phase sequence is the
// reference's exact sequence of rounded additions (BinadeTable), not the exact
// product i*inc: over 2^20 samples the two differ by up to 5e-5 rad.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gpudemod.h"
#include "gpud_internal.cuh"

using namespace gpud;

namespace {

constexpr int kEngThreads = 256;
constexpr int kEngMaxTaps = 4096;

__global__ void __launch_bounds__(kEngThreads) ek_freq_shift_go(const float2 *__restrict__ in,
                                                                float2 *__restrict__ out, int n, BinadeTable tab,
                                                                double sign) {
    __shared__ BinadeTable st;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&tab);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&st);
        for (int w = threadIdx.x; w < (int)(sizeof(BinadeTable) / 4); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ph = sign * binade_value(st, (int64_t)i + 1);  // phase after i+1 additions
        double s, c;
        sincos(ph, &s, &c);
        const float2 v = __ldg(in + i);
        const double xr = v.x, xi = v.y;
        // Go: complex(float32(re*cos - im*sin), float32(re*sin + im*cos)), no fused multiply-add
        out[i] = make_float2((float)__dsub_rn(__dmul_rn(xr, c), __dmul_rn(xi, s)),
                             (float)__dadd_rn(__dmul_rn(xr, s), __dmul_rn(xi, c)));
    }
}

__global__ void __launch_bounds__(kEngThreads) ek_fir_decim_f64(const float2 *__restrict__ x, const double *__restrict__ taps,
                                                                int T, int decim, int n_out, float2 *__restrict__ out) {
    extern __shared__ double st[];
    for (int k = threadIdx.x; k < T; k += blockDim.x) st[k] = taps[k];
    __syncthreads();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_out; j += gridDim.x * blockDim.x) {
        const int i = j * decim;
        const int kmax = i < T - 1 ? i : T - 1;
        double ar = 0.0, ai = 0.0;
        for (int k = 0; k <= kmax; ++k) {
            const float2 v = __ldg(x + (i - k));
            ar = __dadd_rn(ar, __dmul_rn((double)v.x, st[k]));
            ai = __dadd_rn(ai, __dmul_rn((double)v.y, st[k]));
        }
        out[j] = make_float2((float)ar, (float)ai);
    }
}

int eng_grid(long long items) {
    long long g = (items + kEngThreads - 1) / kEngThreads;
    if (g > 148LL * 16) g = 148LL * 16;
    return (int)(g < 1 ? 1 : g);
}

}  // namespace

extern "C" GPUD_API int GPUD_CALL gpud_lowpass_fir(double cutoff_hz, int sample_rate, int taps, double *out,
                                                   int out_cap) {
    if (!out || sample_rate <= 0 || taps <= 0) return GPUD_E_ARG;
    const int len = taps | 1;
    if (out_cap < len) return GPUD_E_ARG;
    const std::vector<double> h = lowpass_fir(cutoff_hz, sample_rate, taps);
    for (int k = 0; k < len; ++k) out[k] = h[(size_t)k];
    return len;
}

extern "C" GPUD_API int GPUD_CALL gpud_shift_fir_decimate_cuda(const gpud_float2 *in, int n, int sample_rate,
                                                               double offset_hz, const double *taps, int num_taps,
                                                               int decim, gpud_float2 *shifted_tmp, gpud_float2 *out,
                                                               int out_cap, int *n_out, gpud_stream_handle stream) {
    if (!n_out) return GPUD_E_ARG;
    *n_out = 0;
    if (n <= 0) return 0;
    if (!in || !taps || !shifted_tmp || !out || num_taps <= 0 || num_taps > kEngMaxTaps || decim <= 0)
        return GPUD_E_ARG;
    const int count = (int)(((long long)n + decim - 1) / decim);
    if (out_cap < count) return GPUD_E_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (sample_rate <= 0 || offset_hz == 0.0) {
        // FreqShift returns its input unchanged (freqshift.go:7-11)
        if (cudaMemcpyAsync(shifted_tmp, in, (size_t)n * sizeof(gpud_float2), cudaMemcpyDeviceToDevice, st) !=
            cudaSuccess)
            return GPUD_E_CUDA;
    } else {
        const double inc = -2 * GPUD_PI * offset_hz / (double)sample_rate;
        BinadeTable tab;
        build_binade_table(std::fabs(inc), &tab);  // the sequence for -inc is the negated one
        ek_freq_shift_go<<<eng_grid(n), kEngThreads, 0, st>>>((const float2 *)in, (float2 *)shifted_tmp, n, tab,
                                                              inc < 0 ? -1.0 : 1.0);
        gpud_count_launch(1);
    }
    ek_fir_decim_f64<<<eng_grid(count), kEngThreads, (size_t)num_taps * sizeof(double), st>>>(
        (const float2 *)shifted_tmp, taps, num_taps, decim, count, (float2 *)out);
    gpud_count_launch(1);
    if (cudaGetLastError() != cudaSuccess) return GPUD_E_CUDA;
    *n_out = count;
    return 0;
}

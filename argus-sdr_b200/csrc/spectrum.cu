// spectrum.cu -- surveillance spectrum on the device (internal/fft/fft.go:
// 19-55 Spectrum, welch.go:15-66 WelchPSD; cmd/sdrd/pipeline_runtime.go:
// 294-341 calls them, or cuFFT, per frame).
//
// The reference transforms in complex128 (gonum) on the CPU, or in complex64
// through cuFFT.  Here one CTA transforms one segment entirely in shared
// memory in float64: the windowed samples are loaded in bit-reversed order,
// then log2(N) radix-2 butterfly stages with twiddles exp(-j 2 pi k / m) from
// sincospi of exact rational arguments.  Welch segments write |X|^2 / N^2 per
// bin; a second kernel adds them in segment order (deterministic) and writes
// the fftshifted dB spectrum.  Power-of-two sizes up to 8192 (128 KB of
// float64 pairs in shared memory).
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/gpudemod.h"
#include "gpud_internal.cuh"

extern "C" void gpud_count_launch(int n);

namespace {

constexpr int kSpecThreads = 512;
constexpr int kMaxFft = 8192;

__device__ __forceinline__ unsigned bitrev(unsigned x, int bits) { return __brev(x) >> (32 - bits); }

// One segment: x[start + i] * w[i] (Hann when hann != 0), i < N, into |X_k|.
// pow_out[k] = |X_k|^2 / N^2 (welch) or |X_k| / N (single).
__global__ void __launch_bounds__(kSpecThreads)
k_spectrum_seg(const float2 *__restrict__ iq, int N, int log2n, int step, int hann, int welch,
               double *__restrict__ pow_out) {
    extern __shared__ double2 sx[];
    const int seg = blockIdx.x;
    const int64_t start = (int64_t)seg * step;
    for (int i = threadIdx.x; i < N; i += kSpecThreads) {
        const float2 v = iq[start + i];
        double w = 1.0;
        // fftutil.Hann: 0.5 (1 - cos(2 pi i / (n-1)))
        if (hann && N > 1) w = 0.5 * (1.0 - cospi(2.0 * (double)i / (double)(N - 1)));
        sx[bitrev((unsigned)i, log2n)] = make_double2((double)v.x * w, (double)v.y * w);
    }
    __syncthreads();
    for (int s = 1; s <= log2n; ++s) {
        const int m = 1 << s, half = m >> 1;
        for (int b = threadIdx.x; b < N / 2; b += kSpecThreads) {
            const int grp = b / half, k = b - grp * half;
            const int i0 = grp * m + k, i1 = i0 + half;
            double sn, cs;
            sincospi(-2.0 * (double)k / (double)m, &sn, &cs);  // exp(-j 2 pi k / m)
            const double2 a = sx[i0], c = sx[i1];
            const double tr = c.x * cs - c.y * sn, ti = c.x * sn + c.y * cs;
            sx[i0] = make_double2(a.x + tr, a.y + ti);
            sx[i1] = make_double2(a.x - tr, a.y - ti);
        }
        __syncthreads();
    }
    const double invN = 1.0 / (double)N;
    for (int k = threadIdx.x; k < N; k += kSpecThreads) {
        const double mag = hypot(sx[k].x, sx[k].y) * invN;
        pow_out[(int64_t)seg * N + k] = welch ? mag * mag : mag;
    }
}

// dB and fftshift: Welch 10 log10(mean power + 1e-24) (welch.go:57-63),
// single 20 log10(|X|/N + 1e-12) (fft.go:42-50); output bin i is bin
// (i + N/2) mod N.
__global__ void __launch_bounds__(256)
k_spectrum_db(const double *__restrict__ pw, int N, int segs, int welch, double *__restrict__ out) {
    const int i = blockIdx.x * 256 + (int)threadIdx.x;
    if (i >= N) return;
    const int idx = (i + N / 2) % N;
    if (welch) {
        double acc = 0.0;
        for (int s = 0; s < segs; ++s) acc += pw[(int64_t)s * N + idx];
        out[i] = 10.0 * log10(acc / (double)segs + 1e-24);
    } else {
        out[i] = 20.0 * log10(pw[idx] + 1e-12);
    }
}

int ilog2_exact(int n) {
    if (n <= 0 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

}  // namespace

struct gpud_spectrum {
    int max_fft = 0, max_segments = 0;
    double *d_pow = nullptr;  // max_segments x max_fft
    double *d_db = nullptr;   // max_fft
};

extern "C" {

GPUD_API int GPUD_CALL gpud_spectrum_destroy(gpud_spectrum *s) {
    if (!s) return 0;
    cudaFree(s->d_pow);
    cudaFree(s->d_db);
    delete s;
    return 0;
}

GPUD_API int GPUD_CALL gpud_spectrum_create(int max_fft, int max_segments, gpud_spectrum **out) {
    if (!out || ilog2_exact(max_fft) < 0 || max_fft > kMaxFft || max_segments <= 0) return GPUD_E_ARG;
    auto *s = new gpud_spectrum();
    s->max_fft = max_fft;
    s->max_segments = max_segments;
    if (cudaMalloc((void **)&s->d_pow, sizeof(double) * (size_t)max_fft * (size_t)max_segments) != cudaSuccess ||
        cudaMalloc((void **)&s->d_db, sizeof(double) * (size_t)max_fft) != cudaSuccess) {
        gpud_spectrum_destroy(s);
        return GPUD_E_CUDA;
    }
    *out = s;
    return 0;
}

static int spectrum_launch(gpud_spectrum *s, const gpud_float2 *iq, int N, int segs, int step, int hann, int welch,
                           cudaStream_t st, double *out_db) {
    const int l2 = ilog2_exact(N);
    // the shared-memory opt-in is per device: made on the launching device
    static std::atomic<uint64_t> optin{0};
    if (gpud::smem_optin_once(optin, (const void *)k_spectrum_seg, kMaxFft * 16) != cudaSuccess) return GPUD_E_CUDA;
    k_spectrum_seg<<<segs, kSpecThreads, N * 16, st>>>(reinterpret_cast<const float2 *>(iq), N, l2, step, hann, welch,
                                                       s->d_pow);
    k_spectrum_db<<<(N + 255) / 256, 256, 0, st>>>(s->d_pow, N, segs, welch, s->d_db);
    if (cudaGetLastError() != cudaSuccess) return GPUD_E_CUDA;
    gpud_count_launch(2);
    if (cudaMemcpyAsync(out_db, s->d_db, sizeof(double) * (size_t)N, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return GPUD_E_CUDA;
    return 0;
}

GPUD_API int GPUD_CALL gpud_spectrum_single(gpud_spectrum *s, const gpud_float2 *iq, int n, int hann,
                                            gpud_stream_handle stream, double *out_db) {
    if (!s || !iq || !out_db || ilog2_exact(n) < 0 || n > s->max_fft) return GPUD_E_ARG;
    return spectrum_launch(s, iq, n, 1, 0, hann, 0, (cudaStream_t)stream, out_db);
}

GPUD_API int GPUD_CALL gpud_spectrum_welch(gpud_spectrum *s, const gpud_float2 *iq, int64_t n, int seg_size,
                                           double overlap, int hann, gpud_stream_handle stream, double *out_db,
                                           int *n_out) {
    if (!s || !iq || !out_db || !n_out || n < 0 || seg_size <= 0) return GPUD_E_ARG;
    *n_out = 0;
    if (overlap < 0) overlap = 0;
    if (overlap > 0.95) overlap = 0.95;
    int step = (int)((double)seg_size * (1 - overlap));
    if (step < 1) step = 1;
    const int64_t segs = n >= seg_size ? (n - seg_size) / step + 1 : 0;
    if (segs == 0) {
        // fewer samples than one segment: Spectrum of the whole vector, no window (welch.go:52-55)
        if (ilog2_exact((int)n) < 0 || n > s->max_fft) return GPUD_E_ARG;
        *n_out = (int)n;
        return spectrum_launch(s, iq, (int)n, 1, 0, 0, 0, (cudaStream_t)stream, out_db);
    }
    if (ilog2_exact(seg_size) < 0 || seg_size > s->max_fft || segs > s->max_segments) return GPUD_E_ARG;
    *n_out = seg_size;
    return spectrum_launch(s, iq, seg_size, (int)segs, step, hann, 1, (cudaStream_t)stream, out_db);
}

}  // extern "C"

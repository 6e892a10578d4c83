// legacy_exports.cu -- the sixteen entry points of the reference's
// gpudemod_kernels library (internal/demod/gpudemod/native/exports.cu), same
// signatures and return codes, written for sm_100a.
//
// Semantics kept from the reference: argument checks and codes, n<=0 no-ops,
// the process-global constant taps of gpud_launch_fir[_stream]_cuda, zero FIR
// history at block start, the AM envelope without mean removal, legacy default
// stream for the non-_stream launchers.  Changed where the reference's GPU
// path diverges from its CPU oracle (the streaming polyphase pair follows
// streaming_host_core.go: layout stride = polyphase_len/decim and only taps
// p + k*decim < num_taps are applied), and no device memory is allocated
// (the prepare path rotates samples inside the fused kernel instead of
// cudaMalloc'ing a temporary, exports.cu:388).
//
// Phases are carried as Q0.64 turn counts inside each launch (exact
// phase_start + i*phase_inc modulo one turn), so the float32 rotator is
// accurate for any block length.
#include <atomic>
#include <cstdio>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gpudemod.h"
#include "gpud_internal.cuh"

using namespace gpud;

static std::atomic<uint64_t> g_launches{0};
extern "C" void gpud_count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
extern "C" GPUD_API uint64_t GPUD_CALL gpud_kernel_launch_count(void) { return g_launches.load(); }

static inline int grid_for(int n, int per_block) {
    long long g = ((long long)n + per_block - 1) / per_block;
    if (g > 148 * 32) g = 148 * 32;  // grid-stride beyond 32 CTAs per SM
    return (int)(g < 1 ? 1 : g);
}

// ---------------------------------------------------------------------------
// frequency shift / SSB product  (exports.cu:37-85, 296-326)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) lk_freq_shift(const float2 *__restrict__ in, float2 *__restrict__ out, int n,
                                                     uint64_t u0, uint64_t inc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        out[i] = cmulf(__ldg(in + i), q64_phasor(u0 + (uint64_t)i * inc));
    }
}

__global__ void __launch_bounds__(256) lk_ssb_product(const float2 *__restrict__ in, float *__restrict__ out, int n,
                                                      uint64_t u0, uint64_t inc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float2 v = __ldg(in + i);
        float2 r = q64_phasor(u0 + (uint64_t)i * inc);
        out[i] = fmaf(v.x, r.x, -v.y * r.y);
    }
}

extern "C" GPUD_API int GPUD_CALL gpud_stream_create(gpud_stream_handle *out) {
    if (!out) return -1;
    cudaStream_t s;
    cudaError_t e = cudaStreamCreate(&s);
    if (e != cudaSuccess) return (int)e;
    *out = (gpud_stream_handle)s;
    return 0;
}

extern "C" GPUD_API int GPUD_CALL gpud_stream_destroy(gpud_stream_handle stream) {
    if (!stream) return 0;
    return (int)cudaStreamDestroy((cudaStream_t)stream);
}

extern "C" GPUD_API int GPUD_CALL gpud_stream_sync(gpud_stream_handle stream) {
    if (!stream) return (int)cudaDeviceSynchronize();
    return (int)cudaStreamSynchronize((cudaStream_t)stream);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_freq_shift_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n,
                                                                     double phase_inc, double phase_start,
                                                                     gpud_stream_handle stream) {
    if (n <= 0) return 0;
    lk_freq_shift<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        (const float2 *)in, (float2 *)out, n, rad_to_q64(phase_start), rad_to_q64(phase_inc));
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_freq_shift_cuda(const gpud_float2 *in, gpud_float2 *out, int n,
                                                              double phase_inc, double phase_start) {
    return gpud_launch_freq_shift_stream_cuda(in, out, n, phase_inc, phase_start, 0);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_ssb_product_cuda(const gpud_float2 *in, float *out, int n,
                                                               double phase_inc, double phase_start) {
    if (n <= 0) return 0;
    lk_ssb_product<<<grid_for(n, 256), 256>>>((const float2 *)in, out, n, rad_to_q64(phase_start),
                                              rad_to_q64(phase_inc));
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FM discriminator  (exports.cu:87-112).  Cross and dot products in float64
// and a float64 atan2, as the CPU path (fm.go:188-193).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) lk_fm_discrim(const float2 *__restrict__ in, float *__restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        float2 p = __ldg(in + i), c = __ldg(in + i + 1);
        double num = (double)p.x * (double)c.y - (double)p.y * (double)c.x;
        double den = (double)p.x * (double)c.x + (double)p.y * (double)c.y;
        out[i] = (float)atan2(num, den);
    }
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_fm_discrim_cuda(const gpud_float2 *in, float *out, int n) {
    if (n <= 1) return 0;
    lk_fm_discrim<<<grid_for(n, 256), 256>>>((const float2 *)in, out, n);
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FIR with zero history  (exports.cu:125-244).  A 1024-sample tile plus the
// (T-1)-sample halo is staged in shared memory once; each thread produces four
// outputs 256 apart (coalesced stores, conflict-free shared reads).
// ---------------------------------------------------------------------------
__constant__ float c_fir_taps[256];

constexpr int kLfTile = 1024;

template <bool kConstTaps>
__global__ void __launch_bounds__(256) lk_fir(const float2 *__restrict__ in, float2 *__restrict__ out, int n, int T,
                                              const float *__restrict__ taps_ptr) {
    extern __shared__ float2 sx[];
    __shared__ float st[256];
    const int i0 = blockIdx.x * kLfTile;
    const int halo = T - 1;
    for (int k = threadIdx.x; k < T; k += blockDim.x) st[k] = kConstTaps ? c_fir_taps[k] : taps_ptr[k];
    for (int l = threadIdx.x; l < kLfTile + halo; l += blockDim.x) {
        int g = i0 - halo + l;
        sx[l] = (g >= 0 && g < n) ? __ldg(in + g) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // thread t: outputs i0 + t + 256*r, r = 0..3 (coalesced stores)
    for (int r = 0; r < 4; ++r) {
        int o = threadIdx.x + 256 * r;
        int g = i0 + o;
        if (g >= n) break;
        float ar = 0.f, ai = 0.f;
        for (int k = 0; k < T; ++k) {
            float2 v = sx[o + halo - k];
            float h = st[k];
            ar = fmaf(v.x, h, ar);
            ai = fmaf(v.y, h, ai);
        }
        out[g] = make_float2(ar, ai);
    }
}

extern "C" GPUD_API int GPUD_CALL gpud_upload_fir_taps_cuda(const float *taps, int n) {
    if (!taps || n <= 0 || n > 256) return -1;
    return (int)cudaMemcpyToSymbol(c_fir_taps, taps, (size_t)n * sizeof(float));
}

static int launch_fir(const gpud_float2 *in, gpud_float2 *out, int n, int num_taps, const float *taps,
                      cudaStream_t s) {
    if (n <= 0 || num_taps <= 0 || num_taps > 256) return 0;
    int grid = (n + kLfTile - 1) / kLfTile;
    size_t smem = (size_t)(kLfTile + num_taps - 1) * sizeof(float2);
    if (taps)
        lk_fir<false><<<grid, 256, smem, s>>>((const float2 *)in, (float2 *)out, n, num_taps, taps);
    else
        lk_fir<true><<<grid, 256, smem, s>>>((const float2 *)in, (float2 *)out, n, num_taps, nullptr);
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_fir_cuda(const gpud_float2 *in, gpud_float2 *out, int n, int num_taps) {
    return launch_fir(in, out, n, num_taps, nullptr, 0);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_fir_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n,
                                                              int num_taps, gpud_stream_handle stream) {
    return launch_fir(in, out, n, num_taps, nullptr, (cudaStream_t)stream);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_fir_v2_stream_cuda(const gpud_float2 *in, gpud_float2 *out,
                                                                 const float *taps, int n, int num_taps,
                                                                 gpud_stream_handle stream) {
    if (n <= 0 || num_taps <= 0 || num_taps > 256) return 0;
    if (!taps) return (int)cudaErrorInvalidValue;
    return launch_fir(in, out, n, num_taps, taps, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// decimate / AM envelope  (exports.cu:114-123, 246-294)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) lk_decimate(const float2 *__restrict__ in, float2 *__restrict__ out, int n_out,
                                                   int factor) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_out; i += gridDim.x * blockDim.x)
        out[i] = __ldg(in + (size_t)i * factor);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_decimate_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n_out,
                                                                   int factor, gpud_stream_handle stream) {
    if (n_out <= 0 || factor <= 0) return 0;
    lk_decimate<<<grid_for(n_out, 256), 256, 0, (cudaStream_t)stream>>>((const float2 *)in, (float2 *)out, n_out,
                                                                        factor);
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_decimate_cuda(const gpud_float2 *in, gpud_float2 *out, int n_out,
                                                            int factor) {
    return gpud_launch_decimate_stream_cuda(in, out, n_out, factor, 0);
}

__global__ void __launch_bounds__(256) lk_am_envelope(const float2 *__restrict__ in, float *__restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float2 v = __ldg(in + i);
        out[i] = sqrtf(v.x * v.x + v.y * v.y);
    }
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_am_envelope_cuda(const gpud_float2 *in, float *out, int n) {
    if (n <= 0) return 0;
    lk_am_envelope<<<grid_for(n, 256), 256>>>((const float2 *)in, out, n);
    gpud_count_launch(1);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Streaming polyphase extractor, single signal  (exports.cu:356-631)
// ---------------------------------------------------------------------------
// Sample i of the concatenation (history[0..H) ++ new[0..n_new)).  New samples
// are either read pre-shifted (stateful path) or rotated in place (prepare).
struct PolyArgs {
    const float2 *hist;
    int H;
    const float2 *newv;
    int n_new;
    bool rotate;
    uint64_t u0, inc;
};

__device__ __forceinline__ float2 poly_sample(const PolyArgs &a, int idx) {
    if (idx < 0) return make_float2(0.f, 0.f);
    if (idx < a.H) return a.hist[idx];
    int k = idx - a.H;
    if (k >= a.n_new) return make_float2(0.f, 0.f);
    float2 v = a.newv[k];
    return a.rotate ? cmulf(v, q64_phasor(a.u0 + (uint64_t)k * a.inc)) : v;
}

// One thread per output: taps[p*L + k] applied to sample (newest - p - k*D)
// for p + k*D < num_taps (streaming_host_core.go:31-48; only taps that exist
// in the applied length, zero samples before the stream start).
__global__ void __launch_bounds__(256) lk_poly_accum(PolyArgs a, const float *__restrict__ taps, int D, int L,
                                                     int num_taps, int start_idx, int n_out, float2 *__restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_out) return;
    int newest = a.H + start_idx + j * D;
    float ar = 0.f, ai = 0.f;
    for (int p = 0; p < D; ++p) {
        for (int k = 0; k < L; ++k) {
            int back = p + k * D;
            if (back >= num_taps) break;
            float t = __ldg(taps + p * L + k);
            float2 v = poly_sample(a, newest - back);
            ar = fmaf(t, v.x, ar);
            ai = fmaf(t, v.y, ai);
        }
    }
    out[j] = make_float2(ar, ai);
}

__global__ void __launch_bounds__(256) lk_history_tail(PolyArgs a, int keep, float2 *__restrict__ dst) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= keep) return;
    dst[q] = poly_sample(a, a.H + a.n_new - keep + q);
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_prepare_cuda(
    const gpud_float2 *in_new, int n_new, const gpud_float2 *history_in, int history_len, const float *polyphase_taps,
    int polyphase_len, int decim, int num_taps, int phase_count_in, double phase_start, double phase_inc,
    gpud_float2 *out, int *n_out, int *phase_count_out, double *phase_end_out, gpud_float2 *history_out) {
    if (n_new < 0 || !polyphase_taps || polyphase_len <= 0 || decim <= 0 || num_taps <= 0) return -1;
    const int phase_len = (num_taps + decim - 1) / decim;
    if (polyphase_len < decim * phase_len) return -2;
    const int L = polyphase_len / decim;
    const int keep = num_taps > 1 ? num_taps - 1 : 0;
    int H = history_len < 0 ? 0 : (history_len > keep ? keep : history_len);
    if (H > 0 && !history_in) return -5;
    if (n_new > 0 && !in_new) return -3;
    int pc = phase_count_in < 0 ? 0 : phase_count_in;
    if (pc >= decim) pc %= decim;
    const int total = pc + n_new;
    const int out_count = total / decim;
    PolyArgs a{(const float2 *)history_in, H, (const float2 *)in_new, n_new, true, rad_to_q64(phase_start),
               rad_to_q64(phase_inc)};
    if (out_count > 0) {
        if (!out) return -4;
        lk_poly_accum<<<(out_count + 255) / 256, 256>>>(a, polyphase_taps, decim, L, num_taps, decim - pc - 1,
                                                       out_count, (float2 *)out);
        gpud_count_launch(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    if (history_out && keep > 0) {
        int nh = H + n_new < keep ? H + n_new : keep;
        if (nh > 0) {
            lk_history_tail<<<(nh + 255) / 256, 256>>>(a, nh, (float2 *)history_out);
            gpud_count_launch(1);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return (int)e;
        }
    }
    if (n_out) *n_out = out_count;
    if (phase_count_out) *phase_count_out = total % decim;
    if (phase_end_out)
        *phase_end_out = q64_to_rad(rad_to_q64(phase_start) + (uint64_t)n_new * rad_to_q64(phase_inc));
    return 0;
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_stateful_cuda(
    const gpud_float2 *in_new, int n_new, gpud_float2 *shifted_new_tmp, const float *polyphase_taps,
    int polyphase_len, int decim, int num_taps, gpud_float2 *history_state, gpud_float2 *history_scratch,
    int history_cap, int *history_len_io, int *phase_count_state, double *phase_state, double phase_inc,
    gpud_float2 *out, int out_cap, int *n_out) {
    if (!polyphase_taps || decim <= 0 || num_taps <= 0 || !history_len_io || !phase_count_state || !phase_state ||
        !n_out)
        return -10;
    if (n_new < 0 || out_cap < 0 || history_cap < 0) return -11;
    const int phase_len = (num_taps + decim - 1) / decim;
    if (polyphase_len < decim * phase_len) return -12;
    const int L = polyphase_len / decim;
    int H = *history_len_io;
    if (H < 0) H = 0;
    if (H > history_cap) H = history_cap;
    int pc = *phase_count_state;
    if (pc < 0) pc = 0;
    if (pc >= decim) pc %= decim;
    const double phase_start = *phase_state;
    const uint64_t u0 = rad_to_q64(phase_start), inc = rad_to_q64(phase_inc);
    if (n_new > 0) {
        if (!in_new || !shifted_new_tmp) return -13;
        lk_freq_shift<<<grid_for(n_new, 256), 256>>>((const float2 *)in_new, (float2 *)shifted_new_tmp, n_new, u0,
                                                     inc);
        gpud_count_launch(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    const int total = pc + n_new;
    const int out_count = total / decim;
    if (out_count > out_cap) return -14;
    PolyArgs a{(const float2 *)history_state, H, (const float2 *)shifted_new_tmp, n_new, false, 0, 0};
    if (out_count > 0) {
        if (!out) return -15;
        lk_poly_accum<<<(out_count + 255) / 256, 256>>>(a, polyphase_taps, decim, L, num_taps, decim - pc - 1,
                                                       out_count, (float2 *)out);
        gpud_count_launch(1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    int newH = H;
    if (history_cap > 0) {
        newH = H + n_new;
        if (newH > history_cap) newH = history_cap;
        if (newH > 0) {
            if (!history_state || !history_scratch) return -16;
            lk_history_tail<<<(newH + 255) / 256, 256>>>(a, newH, (float2 *)history_scratch);
            gpud_count_launch(1);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return (int)e;
            e = cudaMemcpy(history_state, history_scratch, (size_t)newH * sizeof(float2), cudaMemcpyDeviceToDevice);
            if (e != cudaSuccess) return (int)e;
        }
    } else {
        newH = 0;
    }
    *history_len_io = newH;
    *phase_count_state = total % decim;
    *phase_state = q64_to_rad(u0 + (uint64_t)n_new * inc);
    *n_out = out_count;
    return 0;
}

extern "C" GPUD_API uint64_t GPUD_CALL gpud_streaming_config_hash(int64_t signal_id, int out_rate, int num_taps,
                                                                  int sample_rate) {
    // FNV-1a 64 over "sig=%d|out=%d|taps=%d|sr=%d" (streaming_types.go:58-72)
    char buf[160];
    int len = snprintf(buf, sizeof buf, "sig=%lld|out=%d|taps=%d|sr=%d", (long long)signal_id, out_rate, num_taps,
                       sample_rate);
    uint64_t h = 14695981039346656037ULL;
    for (int i = 0; i < len; i++) {
        h ^= (uint8_t)buf[i];
        h *= 1099511628211ULL;
    }
    return h;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the stateful streaming extractor.
//
// Some callers cannot allocate device memory around this call: the real-time
// DSP loop of the reference must not stall on cudaMalloc/cudaFree (both can
// synchronize the whole device, holding up every other signal's work), its
// per-frame allocation churn was removed on purpose (allocation-free frames),
// and a host process whose device memory is committed to a fixed budget has no
// room to hand out per-call temporaries.  This entry point needs no caller
// scratch: the shifted samples and the history staging live in one file-scope
// device array, so the caller passes only inputs, state and outputs.
//
// Limits: n_new <= GPUD_NOALLOC_MAX_NEW and history_cap <= GPUD_NOALLOC_MAX_HISTORY
// (larger requests return GPUD_E_SCRATCH before anything is launched).  The
// array (GPUD_NOALLOC_MAX_NEW + GPUD_NOALLOC_MAX_HISTORY complex samples,
// about 2.1 MB) is held by every GPU that loads this library until the process
// exits.  Every call shares it and it keeps the last call's contents; nothing
// in it has to start at zero (each call writes every element it reads before
// reading it).  Calls that overlap on the GPU (other host threads, other
// streams) race on the array: serialize them.
// ---------------------------------------------------------------------------
static __device__ __align__(256) float2 g_noalloc_scratch[GPUD_NOALLOC_MAX_NEW + GPUD_NOALLOC_MAX_HISTORY];

// Device address of g_noalloc_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, never a device address: it is
// resolved with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on that device (make that first call before
// any stream capture).  The resolved address is kept for the life of the
// process: cudaDeviceReset tears down the context that holds the array, and
// the address kept for that device is then stale, so a process that resets a
// device must not call the allocation-free entry point on it afterwards.
static float2 *noalloc_scratch(cudaError_t *err) {
    static std::atomic<float2 *> cache[64];
    int dev = 0;
    *err = cudaGetDevice(&dev);
    if (*err != cudaSuccess) return nullptr;
    if (dev < 0 || dev >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    float2 *p = cache[dev].load(std::memory_order_acquire);
    if (p) return p;
    void *addr = nullptr;
    *err = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (*err != cudaSuccess) return nullptr;
    p = static_cast<float2 *>(addr);
    cache[dev].store(p, std::memory_order_release);
    return p;
}

extern "C" GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
    const gpud_float2 *in_new, int n_new, const float *polyphase_taps, int polyphase_len, int decim, int num_taps,
    gpud_float2 *history_state, int history_cap, int *history_len_io, int *phase_count_state, double *phase_state,
    double phase_inc, gpud_float2 *out, int out_cap, int *n_out) {
    // the base entry point's argument codes come first (-10 null state
    // pointers, -11 negative sizes), then the scratch limits
    if (!polyphase_taps || decim <= 0 || num_taps <= 0 || !history_len_io || !phase_count_state || !phase_state ||
        !n_out)
        return -10;
    if (n_new < 0 || out_cap < 0 || history_cap < 0) return -11;
    if (n_new > GPUD_NOALLOC_MAX_NEW || history_cap > GPUD_NOALLOC_MAX_HISTORY) return GPUD_E_SCRATCH;
    cudaError_t err = cudaSuccess;
    float2 *scratch = noalloc_scratch(&err);
    if (!scratch) return (int)err;
    return gpud_launch_streaming_polyphase_stateful_cuda(
        in_new, n_new, (gpud_float2 *)scratch, polyphase_taps, polyphase_len, decim, num_taps, history_state,
        (gpud_float2 *)(scratch + GPUD_NOALLOC_MAX_NEW), history_cap, history_len_io, phase_count_state, phase_state,
        phase_inc, out, out_cap, n_out);
}

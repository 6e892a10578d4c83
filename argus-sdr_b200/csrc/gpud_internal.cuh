// gpud_internal.cuh -- device-side data layout and helpers shared by the
// sm_100a kernels of libgpudemod_kernels.so.
//
// Layout in HBM (one runner):
//   ChanParams[max_ch]   per-slot constants (written by the host on admit/update)
//   ChanState [max_ch]   per-slot state carried across blocks (device-resident)
//   taps arena           per slot: extraction taps, phase-major p*L+u, zero-padded
//   history arena        per slot: 2 ping-pong buffers of HCAP shifted samples
//   WFM arenas           per slot: 100-sample delay lines of the composite,
//                        L-R and mono-audio filters, RDS shifted history
//   per-block buffers    extracted IQ, composite, pilot/bpf/lpr/lr work arrays
//   output arena         results table | audio | RDS | emitted IQ (one D2H)
#pragma once
#include <atomic>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#ifndef GPUD_PI
#define GPUD_PI 3.14159265358979323846
#endif

namespace gpud {

// Opt kernel `fn` in to `bytes` of dynamic shared memory on the current
// device.  cudaFuncSetAttribute acts on the current device only, so the
// opt-in is made once per device: bit d of `done` (one mask per kernel, owned
// by its launch helper) records device d.  Threads racing on the first launch
// may both set the attribute, which is harmless.  Returns the API's error.
inline cudaError_t smem_optin_once(std::atomic<uint64_t> &done, const void *fn, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev < 64 ? (uint64_t{1} << dev) : 0;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// ---------------------------------------------------------------------------
// NCO phase as an unsigned Q0.64 fraction of a turn.  Sample i of a block has
// phase u0 + i*inc (mod 2^64) exactly, so a block's per-sample phases are
// computed in parallel with no accumulated rounding, and the carried phase
// never drifts.  (The reference carries float64 radians and adds the
// increment sample by sample, streaming_host_core.go:56-61; the two agree to
// ~1e-10 rad per 2^20 samples, far below float32 resolution of the rotator.)
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t rad_to_q64(double rad) {
    double t = rad * (1.0 / (2.0 * GPUD_PI));
    t -= floor(t);  // [0, 1)
    double s = t * 4294967296.0;
    double hi = floor(s);
    double lo = (s - hi) * 4294967296.0;
    uint64_t h = (uint64_t)hi;
    uint64_t l = (uint64_t)lo;
    return (h << 32) + l;
}

// Phase in [-pi, pi) radians (float64) of a Q0.64 turn count.
__host__ __device__ inline double q64_to_rad(uint64_t q) {
    int64_t s = (int64_t)q;  // two's complement: [-2^63, 2^63) <-> [-0.5, 0.5) turn
    return (double)s * (2.0 * GPUD_PI / 18446744073709551616.0);
}

// Unit phasor exp(j*2*pi*q/2^64) in float32.  sincospif on the signed top 32
// bits: argument resolution 2^-31 half-turns, result within ~1 ulp.
__device__ __forceinline__ float2 q64_phasor(uint64_t q) {
    int32_t top = (int32_t)(q >> 32);
    float x = (float)top * 4.656612873077393e-10f;  // 2^-31 -> half-turns in [-1, 1)
    float s, c;
    sincospif(x, &s, &c);
    return make_float2(c, s);
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// ---------------------------------------------------------------------------
// Per-slot constants
// ---------------------------------------------------------------------------
struct ChanParams {
    uint64_t inc_q;   // NCO increment (Q0.64 turns per input sample)
    double inc_rad;   // -2*pi*offset/fs
    int32_t decim;    // D
    int32_t ntaps;    // T (taps applied)
    int32_t nphase;   // P = min(D, T): phases carrying taps
    int32_t plen;     // L = ceil(T / D)
    int32_t mode;     // GPUD_MODE_*
    int32_t flags;    // GPUD_CH_*
    int32_t out_rate;
    int32_t taps_off; // float offset into the taps arena (phase-major P*L)
    int32_t dtaps_off;// float offset of the direct-form taps h[0..T-1]
    int32_t hist_off; // float2 offset of the history pair (2 * hcap)
    int32_t hcap;     // history capacity (>= T-1)
    int32_t wfm_idx;  // index into WFM arenas (-1 when not WFM)
    int32_t rds_dr;   // RDS decimation floor(out_rate/19000)
    int32_t rs_bank;  // 48 kHz resampler bank id (GPUD_CH_AUDIO48K)
    double ssb_inc;   // 2*pi*(+-700)/out_rate for USB/LSB/CW
    double pll_alpha, pll_beta, pll_lpa;   // stereo PLL constants
    double pll_fmin, pll_fmax;             // freq clamp (rad/sample)
    double rds_inc;                        // 2*pi*57000/out_rate
    int32_t rds_tab;                       // binade table id for the RDS phase
    int32_t aud_ch;                        // audio channels (2 for WFM_STEREO, else 1)
    int32_t d1;                            // pre-demod decimation (1: none)
    int32_t precise_sum;                   // 1: extraction rows summed in float32, rows added in float64
    double deemph_a;                       // de-emphasis coefficient exp(-1/(48000 tau)), 0: none
};

// Per-slot state carried across blocks.
struct ChanState {
    uint64_t nco_q;      // NCO phase at the start of the next block
    float2 last_iq;      // discriminator bridge sample
    int32_t has_last;
    int32_t pll_path;    // last block: 1 parallel-in-time solver, 2 serial loop
    // stereo pilot PLL (recorder/streamer.go:1560-1619)
    double pll_phase, pll_freq, pll_i, pll_q, err_avg;
    int32_t on_count, off_count, enabled, locked;
    float coherence, pilot_hz, last_err_avg, pad1;
    // RDS baseband stream
    int64_t rds_count;   // composite samples consumed
    int32_t rds_hist_len;
    int32_t pll_iters;   // Newton iterations of the last parallel solve
    double comp_power;   // GPUD_CH_BATCH_STEREO: sum of the block's composite squared
};

// Channel flags the kernels test (values of GPUD_CH_* in gpudemod.h).
constexpr int kChPcmF32 = 32;
constexpr int kChBatchStereo = 64;
constexpr int kChFreeStereo = 128;

// Per-block per-slot descriptor (host-built; all integer bookkeeping is
// mirrored on the host, so output sizes are known before launch).
struct SlotBlock {
    int32_t slot;
    int32_t pc;        // phase count before the block
    int32_t n_out;     // extraction outputs this block
    int32_t hist_len;  // history length before the block
    int32_t hist_sel;  // ping-pong buffer holding the current history
    int32_t ext_off;   // float2 offset of this slot's extracted IQ
    int32_t n_disc;    // discriminator outputs
    int32_t bridge;    // 1: first output uses last_iq
    int32_t comp_off;  // float offset of composite/work arrays
    int32_t audio_off; // float offset into the audio output region
    int32_t n_audio;   // floats written to audio
    int32_t rds_off;   // float2 offset into the RDS output region
    int32_t n_rds;
    int32_t rds_first; // first composite index of this block that is kept (-1: none)
    int32_t comp_hist_len; // valid samples in the composite delay line (<= 100)
    int32_t res_idx;   // index into the results table
    // 48 kHz audio back end (GPUD_CH_AUDIO48K)
    int32_t rs_t0;     // resampler phase counter before the block (outTime)
    int32_t rs_nout;   // 48 kHz frames produced this block
    int32_t pcm_off;   // int16 offset into the PCM output region
    int32_t rs_frames; // demod-rate frames consumed this block
    // demodulator input: the extraction output, or with a pre-demod
    // decimation stage its output (streamer.go:1098-1146)
    int32_t dem_off;   // float2 offset of the demod input in the IQ region
    int32_t n_dem;     // demod input samples this block
    int32_t d1_phase;  // pre-demod decimator phase before the block
    // phase-grouped extraction: ng groups of pg phases (one CTA per tile adds them)
    int32_t ng;
    int32_t pg;
    int32_t pad_pg;
    int32_t wide_end;  // > 0: the warp-per-output kernel computes only outputs before it (the rest: a bank)
};

// Channel group extracted on the tensor cores (gemm_extract.cu): channels of
// one decimation D, tap count T and phase count pc share the input grid.
struct GemmGroup {
    int32_t nmem;    // channels (members[mem_off .. mem_off + nmem): SlotBlock rows)
    int32_t ncol;    // N = 2 * channels, padded to a multiple of 16
    int32_t D, L, T, pc;
    int32_t n_out;   // outputs of every member this block
    int32_t jt0;     // first output of the group tiles (earlier ones: dense kernel)
    int32_t b_off;   // byte offset of the packed taps in the frame's buffer
    int32_t mem_off;
    int32_t ns;      // taps stages in shared memory
    int32_t na;      // TMEM accumulators (arm u accumulates into u % na; summed in the epilogue)
};

// Short-arm channel bank (bank_extract.cu): channels of one decimation D, tap
// count T <= 4D and phase count pc share the input grid; every output from
// jt0 on is computed for all members from one staging of the input windows.
struct BankGroup {
    int32_t nmem;    // channels (members[mem_off .. mem_off + nmem): SlotBlock rows)
    int32_t cpad;    // channel columns of the packed taps (a multiple of 32)
    int32_t D, T, pc;
    int32_t n_out;   // outputs of every member this block
    int32_t jt0;     // first output of the bank tiles (earlier ones: the warp-per-output kernel)
    int32_t mem_off;
    int32_t g_off;   // float2 offset of the packed modulated taps (T x cpad) in the frame's buffer
    int32_t r;       // outputs per lane of a work item (1, 2 or 4): 8r outputs per item
};

// Rational polyphase resampler bank (dsp/resample.go:45-93) for one input rate.
constexpr int kRsTaps = 33;     // taps per arm at 32 taps per phase (odd prototype)
struct RsBank {
    int32_t L, M, K, pad;
    const double *arm;  // device array arm[p*K + t], L*K doubles
};

// Per-slot audio back-end state.
struct AudState {
    float dl[2][kRsTaps];  // resampler delay lines, [0] newest
    double y[2];           // de-emphasis states
};

// Results table row written by the device each block.
struct DevResult {
    double nco_phase;
    int32_t flags;
    float coherence, pilot_hz, err_avg;
    int32_t status;
    int32_t pll_iters;
    int32_t pad[2];
};

// ---------------------------------------------------------------------------
// Shared-memory pipeline primitives (sm_90+ PTX): mbarriers with bounded
// waits, bulk copies global -> shared counted on an mbarrier, and the fault
// word a kernel writes when a bounded wait gives up.
// ---------------------------------------------------------------------------
constexpr unsigned kWaitPolls = 1u << 22;  // polls (64 ns apart after the first 64) before a wait gives up

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity: false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
    for (unsigned i = 0; i < kWaitPolls; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i >= 64) __nanosleep(64);
    }
    return false;
}

// Bulk copy global -> this CTA's shared memory, completion counted on bar.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Record a fault code in the runner's page-locked fault word (read by the host
// once the block completes).
__device__ __forceinline__ void device_fault(unsigned *fault, unsigned code) {
    *(volatile unsigned *)fault = code;
    __threadfence_system();
}

// Exact sequential float64 accumulation x_k = fl(x_{k-1} + inc), x_0 = 0
// (dsp.FreqShift's `phase += inc`, dsp/freqshift.go:13-15), evaluated in
// closed form per binade: inside one binade every value is a multiple of the
// binade's ulp, so the rounded step is a constant multiple of that ulp and
// x_k = x_start + (k - k_start) * q exactly.  The host builds the table by
// walking binade boundaries with the same float64 additions.
struct BinadeEntry {
    int64_t k_start;  // first index covered by this entry
    double x_start;   // x_{k_start}
    double q;         // exact step inside the entry
};
constexpr int kMaxBinades = 96;
struct BinadeTable {
    int32_t count;
    int32_t pad;
    BinadeEntry e[kMaxBinades];
};

__device__ __forceinline__ double binade_value(const BinadeTable &t, int64_t k) {
    int lo = 0, hi = t.count - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (t.e[mid].k_start <= k) lo = mid; else hi = mid - 1;
    }
    const BinadeEntry &b = t.e[lo];
    return b.x_start + (double)(k - b.k_start) * b.q;
}

// Host helpers shared by the runner and the engine entry points (runner.cu).
// dsp.LowpassFIR (internal/dsp/fir.go:6-28): Hann-windowed sinc, odd length.
std::vector<double> lowpass_fir(double cutoff_hz, int sample_rate, int taps);
// Binade table of x_k = fl(x_{k-1} + inc), x_0 = 0, for inc > 0.
int build_binade_table(double inc, BinadeTable *t);

constexpr int kWfmTaps = 101;      // stereo / RDS filter length (streamer.go:1531-1545, fm.go:155)
constexpr int kWfmHist = 100;
constexpr int kD1Taps = 101;       // pre-demod decimating FIR (streamer.go:1124)

}  // namespace gpud

// Kernel launch accounting (host side).
extern "C" void gpud_count_launch(int n);

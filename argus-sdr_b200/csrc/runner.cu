// runner.cu -- host side of the batched / serving runner (C++17, CUDA runtime).
//
// Replaces the reference's per-signal Go loop (BatchRunner.StreamingExtractGPU
// -> buildStreamingGPUInvocations -> executeStreamingGPUNativePrepared ->
// applyStreamingGPUExecutionResults, streaming_gpu_*.go) and the CPU demod of
// recorder/streamer.go processSnippet with:
//   - a device-resident slot table (ChanParams / ChanState / taps / histories),
//   - host mirrors of every integer counter (phase count, history length,
//     bridge flag, RDS sample count) so each block's output sizes and packed
//     offsets are known before launch,
//   - one launch sequence per block for all channels, with per-kernel work
//     lists of (slot, tile) pairs for uneven taps / decimation,
//   - one H2D of the block, one H2D of the descriptors, one D2H of all outputs,
//   - up to three blocks in flight, each with its own frame of buffers: block
//     k+1's front half (extraction, demod, stereo FIR bank, RDS) overlaps
//     block k's back half (pilot PLL, stereo output), ordered by events, and
//     the copies of neighbouring blocks overlap compute.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <string>
#include <time.h>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpudemod.h"
#include "gpud_internal.cuh"

namespace gpud {

// kernels (runner_kernels.cu)
struct WfmTaps;
cudaError_t launch_extract_dense(int L, int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                 const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                 const float2 *hist, const float *taps, float2 *ext);
cudaError_t launch_extract_dense_any(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                     const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                     const float2 *hist, const float *taps, float2 *ext);
cudaError_t launch_extract_dense_pipe(int L, int ng, int ntiles, int grid, int pmax, cudaStream_t sm,
                                      const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                                      const ChanState *st, const float2 *x, int n, const float2 *hist,
                                      const float *taps, float2 *ext, unsigned *fault);
cudaError_t launch_gemm_pack(int ngroups, int max_l, cudaStream_t sm, const GemmGroup *groups, const int *members,
                             const SlotBlock *sbt, const ChanParams *prm, const float *taps, float *gb);
cudaError_t launch_extract_gemm(int grid, int smem, cudaStream_t sm, const int2 *work, const GemmGroup *groups,
                                const int *members, const SlotBlock *sbt, const ChanParams *prm, const ChanState *st,
                                const float2 *x, int n, const float *gb, float2 *ext, unsigned *fault);
int gemm_smem_bytes_host(int D, int L, int N, int ns);
int gemm_tile();
cudaError_t launch_bank_pack(int ngroups, int max_total, cudaStream_t sm, const BankGroup *groups,
                             const int *members, const SlotBlock *sbt, const ChanParams *prm, const float *taps,
                             float2 *gtab);
cudaError_t launch_extract_bank(int grid, cudaStream_t sm, const int2 *work, const BankGroup *groups,
                                const int *members, const SlotBlock *sbt, const ChanParams *prm, const ChanState *st,
                                const float2 *x, const float2 *gtab, float2 *ext);
int bank_lanes();
int bank_warps();
size_t gemm_pack_bytes_host(int D, int L, int N);
cudaError_t launch_extract_wide(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                const float2 *hist, const float *taps, float2 *ext);
cudaError_t launch_demod(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                         const ChanState *st, const float2 *ext, float *comp, float *audio);
cudaError_t launch_am(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const float2 *ext,
                      float *audio);
cudaError_t launch_wfm_fir(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const WfmTaps *taps, float *wk, int W, const float *comp_dl);
cudaError_t launch_free_stereo(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                               const ChanParams *prm, const BinadeTable *tabs38, float *wk, int W);
cudaError_t launch_seg_aa(cudaStream_t sm, const float *in, int C, const double *taps, int nt, int d2, int of,
                          float *out);
cudaError_t launch_comp_power(int count, cudaStream_t sm, const int *list, const SlotBlock *sbt,
                              const ChanParams *prm, ChanState *st, const float *wk);
cudaError_t launch_pll(int count, cudaStream_t sm, const int *list, const SlotBlock *sbt, const ChanParams *prm,
                       ChanState *st, float *wk, int W);
cudaError_t launch_pll_newton(int count, int cluster, cudaStream_t sm, const int *list, const SlotBlock *sbt,
                              const ChanParams *prm, ChanState *st, float *wk, int W, int max_iters);
int pll_newton_threads();
int pll_cluster_for(int max_n);
cudaError_t launch_wfm_out(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const ChanState *st, const WfmTaps *taps, const float *wk, int W, const float *lr_dl,
                           const float *audio_dl, float *audio);
cudaError_t launch_rds(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                       const ChanParams *prm, const ChanState *st, const WfmTaps *taps, const BinadeTable *tabs,
                       const float *wk, const float2 *rds_dl, float2 *rds_out);
cudaError_t launch_post_extract(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                                const float2 *x, int n, float2 *hist, DevResult *res);
cudaError_t launch_post_front(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                              const float2 *ext, const float *wk, float *comp_dl, float2 *rds_dl,
                              const BinadeTable *tabs, float2 *d1hist, DevResult *res);
cudaError_t launch_decim2(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                          const double *d1taps, const float2 *d1hist, float2 *ext);
int decim2_tile();
cudaError_t launch_post_back(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                             const float *wk, int W, float *lr_dl, float *audio_dl, DevResult *res);
cudaError_t launch_audio48(int grid_rs, int count, cudaStream_t sm, const int2 *work, const int *list,
                           const SlotBlock *sbt, const ChanParams *prm, const RsBank *banks, AudState *aud,
                           const float *audio, float *rs_buf, int16_t *pcm);
int audio48_tile();
int rds_smem_bytes(int dr);
int rds_tile();
int dense_smem_bytes_host(int P, int L);
int dense_pipe_groups_host(int P, int L, int cap);
int dense_tile();
int wide_smem_bytes_host(int T);
int group_smem_bytes_host(int Pc, int L);
int mod_smem_bytes_host(int Pc, int L);
cudaError_t launch_extract_group(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                 const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                 const float2 *hist, const float *taps, float2 *ext);
cudaError_t launch_extract_mod(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                               const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                               const float2 *hist, const float *taps, float2 *ext);

constexpr int kWfmTapsPadH = 104;
struct WfmTapsHost {
    float t[kWfmTapsPadH][4];
    double rds[kWfmTaps];
};
constexpr int kAudioDlStrideH = kWfmHist + 4;
constexpr int kMaxWfmClasses = 16;
constexpr int kDenseMaxL = 16;
constexpr int kDenseSmemLimit = 200 * 1024;
constexpr int kDensePipeSmemCap = 220 * 1024;  // what the pipelined dense kernel opts in to
#ifndef GPUD_GEMM_PAIR
#define GPUD_GEMM_PAIR 1  // 0: three taps stages, one group CTA per SM
#endif
#ifndef GPUD_GEMM_EXTRACT
#define GPUD_GEMM_EXTRACT 1  // 0: no tensor-core channel groups
#endif
constexpr int kGemmMinChannels = 4;           // smaller groups stay on the dense kernel
constexpr int kGemmSmemCap = 220 * 1024;
constexpr int kGemmFirstOutput = 256;         // outputs before it (history) stay on the dense kernel
#ifndef GPUD_BANK_EXTRACT
#define GPUD_BANK_EXTRACT 1  // 0: no short-arm channel banks
#endif
constexpr int kBankMinChannels = 4;           // smaller classes keep their own form
constexpr int kBankMaxL = 4;                  // arms of at most four taps (T <= 4D)
constexpr int kWideTile = 32;                 // outputs per work item of the warp-per-output kernel
#ifndef GPUD_DENSE_PIPE
#define GPUD_DENSE_PIPE 2  // most consumer groups of the pipelined dense kernel (0: one-tile-per-CTA kernel only)
#endif
constexpr int kGroupSmemTarget = 100 * 1024;  // two CTAs per SM
constexpr int kModSmemTarget = 72 * 1024;     // three CTAs per SM
constexpr int kModMaxL = 4;
constexpr int kPllMaxIters = 64;
#ifndef GPUD_FRAMES
#define GPUD_FRAMES 3
#endif
constexpr int kFrames = GPUD_FRAMES;  // blocks in flight
constexpr int kInRing = kFrames + 1;  // input ring slots: one more than frames, so a copy can start before a frame is free
constexpr int kMaxRsClasses = 16;  // 48 kHz resampler banks (one per demod rate)

// ---------------------------------------------------------------------------
// DSP design helpers (host) -- restated from the reference
// ---------------------------------------------------------------------------

// dsp.LowpassFIR (internal/dsp/fir.go:6-28): Hann-windowed sinc, odd length.
std::vector<double> lowpass_fir(double cutoff_hz, int sample_rate, int taps) {
    if (taps % 2 == 0) taps++;
    std::vector<double> out((size_t)taps, 0.0);
    double fc = cutoff_hz / (double)sample_rate;
    if (fc <= 0) return out;
    double m = (double)(taps - 1) / 2.0;
    for (int n = 0; n < taps; n++) {
        double x = (double)n - m;
        double sinc = (x == 0) ? 2 * fc : std::sin(2 * GPUD_PI * fc * x) / (GPUD_PI * x);
        double w = 0.5 * (1 - std::cos(2 * GPUD_PI * (double)n / (double)(taps - 1)));
        out[(size_t)n] = sinc * w;
    }
    return out;
}

// recorder/streamer.go:1496-1509 pllCoefficients
static void pll_coefficients(double loop_bw, double damping, int sample_rate, double *alpha, double *beta) {
    if (sample_rate <= 0 || loop_bw <= 0) {
        *alpha = *beta = 0;
        return;
    }
    double bl = loop_bw / (double)sample_rate;
    double theta = bl / (damping + 0.25 / damping);
    double d = 1 + 2 * damping * theta + theta * theta;
    *alpha = (4 * damping * theta) / d;
    *beta = (4 * theta * theta) / d;
}

// Binade table of x_k = fl(x_{k-1} + inc), x_0 = 0, inc > 0 (see BinadeTable).
int build_binade_table(double inc, BinadeTable *t) {
    std::memset(t, 0, sizeof *t);
    const int64_t kmax = (int64_t)1 << 42;
    int64_t k = 1;
    double x = inc;  // x_1 = fl(0 + inc) = inc
    int c = 0;
    while (k < kmax && c < kMaxBinades - 2) {
        int e;
        std::frexp(x, &e);            // x in [2^(e-1), 2^e)
        double top = std::ldexp(1.0, e);
        double u = std::ldexp(1.0, e - 53);  // ulp inside [2^(e-1), 2^e)
        double y = x + inc;           // same float64 addition as the reference
        if (y >= top) {               // leaves the binade after one step
            t->e[c++] = BinadeEntry{k, x, y - x};
            x = y;
            k += 1;
            continue;
        }
        double q = y - x;             // exact: both multiples of u
        double z = y + inc;
        if (z < top && z - y != q) {  // round-half-even tie: the step settles after one move
            t->e[c++] = BinadeEntry{k, x, q};
            x = y;
            k += 1;
            q = z - y;
        }
        // largest J with x + J*q < top (integers in units of u)
        double A = (top - x) / u;     // exact integer
        double m = q / u;
        int64_t J = (int64_t)((A - 1) / m);
        while (J > 0 && x + (double)J * q >= top) J--;
        t->e[c++] = BinadeEntry{k, x, q};
        double xl = x + (double)J * q;
        k += J;
        x = xl + inc;  // explicit boundary step
        k += 1;
    }
    t->count = c;
    return c;
}

// ---------------------------------------------------------------------------
// Runner
// ---------------------------------------------------------------------------
struct Slot {
    bool active = false;
    uint64_t pver = 0;  // version of the taps and NCO increment (the channel-group taps cache key)
    uint64_t reusable_after = 0;  // a retired slot is reused once this ticket completed
    gpud_channel_spec spec{};
    int D = 1, T = 1, P = 1, L = 1, hcap = 0;
    int ext_kind = 0;  // 0 dense (all D phases of a tile), 1 wide, 2 phase groups, 3 modulated short arms
    int pg = 0, ng = 1;  // phase groups: ng groups of at most pg phases
    int taps_off = 0, dtaps_off = 0, hist_off = 0, wfm_idx = -1, rate_class = -1;
    double cutoff = 0;
    // host mirrors of device integer state (as of the last submitted block)
    int pc = 0, hist_len = 0, hist_sel = 0, comp_hist_len = 0;
    bool has_last = false;
    int64_t rds_count = 0;
    int64_t rs_t = 0;  // 48 kHz resampler phase counter (outTime)
    int d1 = 1, d1_phase = 0;  // pre-demod decimation and its phase counter
    double deemph_us = -1.0;   // >= 0: de-emphasis time constant instead of the flags' choice
    int rs_class = -1, rs_L = 1, rs_M = 1, aud_ch = 1;
    uint64_t footprint = 0;
};

struct BlockPlan {
    int n = 0;
    std::vector<SlotBlock> sbs;
    // work lists
    std::vector<int2> w_dense[kDenseMaxL + 1];
    int dense_smem[kDenseMaxL + 1] = {};
    int dense_pmax[kDenseMaxL + 1] = {};  // most phases of a class's channels (pipelined form layout)
    // tensor-core channel groups (gemm_extract.cu)
    std::vector<GemmGroup> groups;
    std::vector<int> gmembers;            // SlotBlock rows of the groups' channels
    std::vector<int2> w_gemm;             // (group, 128-output tile from kGemmFirstOutput)
    int gemm_smem = 0, gemm_max_l = 0;
    size_t gemm_b_bytes = 0;              // packed taps of all groups
    // short-arm channel banks (bank_extract.cu)
    std::vector<BankGroup> banks;
    std::vector<int> bmembers;            // SlotBlock rows of the banks' channels
    std::vector<int2> w_bank;             // (bank, tile * chunks + chunk)
    int64_t bank_g = 0;                   // float2 entries of the packed modulated taps
    int bank_max_total = 0;               // largest T x cpad of a bank
    std::vector<int2> w_wide;
    int wide_smem = 0;
    std::vector<int2> w_group;  // (entry, 256-output tile): one CTA takes the tile's phase groups in turn
    int group_smem = 0;
    std::vector<int2> w_mod;    // (entry, 256-output tile) of the modulated short-arm form, likewise
    int mod_smem = 0;
    std::vector<int2> w_demod, w_am, w_fir, w_out, w_rds;
    int rds_smem = 0;
    std::vector<int> pll_list;
    std::vector<int2> w_free;   // (entry, 1024-sample tile) of free-running stereo channels
    bool batch_stereo = false;  // a GPUD_CH_BATCH_STEREO channel has composite this block
    std::vector<int> aud_list;  // entries with a 48 kHz back end and input this block
    std::vector<int2> w_aud;    // (entry, tile) of the 48 kHz resampler
    std::vector<int2> w_dec;    // (entry, tile) of the pre-demod decimator
    int64_t tot_ext = 0, tot_emit_ext = 0, tot_comp = 0, tot_audio = 0, tot_audio_host = 0, tot_rds = 0,
            tot_pcm = 0;
};

struct SlotAfter {
    int pc, hist_len;
};

// One stream-ordered host->device write, applied before the next block's front half.
struct PendingOp {
    int slot;
    void *dst;
    std::vector<char> data;
};

// Everything one block in flight owns.
struct Frame {
    cudaStream_t s = nullptr;
    cudaEvent_t ev_front = nullptr, ev_back = nullptr, ev_done = nullptr, ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t ev_ext = nullptr;  // the block's extraction state (history, NCO phase) is carried
    int ring = -1;                 // input ring slot the block reads (-1: device input or the frame's own buffer)
    cudaEvent_t ev_start = nullptr;  // where the block's latency starts (ev0, or its ring copy's start)
    cudaStream_t s2 = nullptr;  // side stream: dense classes beside the channel-group kernel
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    char *d_desc = nullptr, *h_desc = nullptr;
    size_t desc_cap = 0;
    char *d_out = nullptr, *h_out = nullptr;
    size_t out_cap = 0;
    char *h_stage = nullptr;
    size_t stage_cap = 0;
    float *d_wk = nullptr;
    int64_t wk_cap = 0;
    float2 *d_block = nullptr;
    float2 *h_in = nullptr;
    float *d_rs = nullptr;  // resampled 48 kHz audio before de-emphasis
    int64_t rs_cap = 0;
    float2 *d_bank = nullptr;   // packed modulated taps of the short-arm channel banks
    int64_t bank_cap = 0;
    float *d_gb = nullptr;      // packed taps of the tensor-core channel groups
    size_t gb_cap = 0;
    std::vector<uint64_t> gb_key;  // the groups and member versions d_gb was packed for
    std::vector<uint64_t> bank_key;  // the banks and member versions d_bank was packed for
    BlockPlan plan;
    std::vector<SlotAfter> after;
    std::vector<int> row_of_slot;
    size_t off_res = 0, off_pcm = 0, off_audio = 0, off_rds = 0, off_ext = 0, out_bytes = 0;
    bool host_outputs = true;
    uint64_t ticket = 0;
    bool inflight = false;
    uint64_t h2d = 0, d2h = 0;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<std::string> prof_names;
    int prof_n = 0;
};

}  // namespace gpud

using namespace gpud;

struct gpud_runner {
    int fs = 0, max_block = 0, max_ch = 0, max_taps = 0;
    uint64_t budget = 0, used = 0;
    int schedule = GPUD_SCHED_BATCHED;
    cudaStream_t stream = nullptr;  // joins every block: work recorded here follows all submitted blocks
    cudaStream_t admin = nullptr;   // admission copies into slots no block in flight uses
    // input ring: a block from pinned host memory is copied into the next
    // slot on its own stream as soon as it is submitted, before the submit
    // waits for a free frame; a slot is refilled once the block that read it
    // has carried its extraction state (every reader of the input is done)
    cudaStream_t in_s = nullptr;
    float2 *d_ring[kInRing] = {};
    cudaEvent_t ring_t0[kInRing] = {}, ring_copied[kInRing] = {}, ring_free[kInRing] = {};
    int ring_next = 0;
    double ring_ms = 0;       // device time of the ring copies since the last stats reset
    uint64_t ring_copies = 0;
    std::string err;
    std::recursive_mutex mu;

    std::vector<Slot> slots;
    int tapcap = 0;  // floats per slot in each taps region
    // persistent device arenas
    ChanParams *d_prm = nullptr;
    ChanState *d_st = nullptr;
    float *d_taps = nullptr;
    float2 *d_hist = nullptr;
    float *d_comp_dl = nullptr, *d_lr_dl = nullptr, *d_audio_dl = nullptr;
    float2 *d_rds_dl = nullptr;
    WfmTapsHost *d_wtaps = nullptr;
    BinadeTable *d_tabs = nullptr;
    std::vector<int> class_rate;  // rate of each WFM rate class
    std::vector<gpud_autotune_entry> tune;  // per (taps, decimation) extraction form overrides
    AudState *d_aud = nullptr;    // per slot
    double *d_d1taps = nullptr;   // per slot: pre-demod decimator taps
    float2 *d_d1hist = nullptr;   // per slot: its 100-sample history
    RsBank *d_banks = nullptr;
    std::vector<int> rs_rate;     // input rate of each resampler bank
    std::vector<int3> rs_lmk;     // (L, M, K) of each bank
    std::vector<double *> rs_arms;  // device arms of each bank
    bool pll_parallel = true;
    int pll_max_iters = kPllMaxIters;  // Newton iterations before the serial fallback
    int num_sms = 148;
    bool channel_groups = true;  // tensor-core channel groups (gpud_runner_set_channel_groups)
    // fault word the pipelined extraction kernel writes when a bounded wait
    // gives up (page-locked, mapped into the device)
    unsigned *h_fault = nullptr, *d_fault = nullptr;
    // frames
    Frame fr[kFrames];
    int nxt = 0;        // frame the next block uses
    int last = -1;      // frame of the last submitted block
    int done_frame = -1;  // frame whose results gpud_runner_result reads
    uint64_t submitted = 0, completed = 0;
    std::vector<PendingOp> pending;
    // stats
    uint64_t blocks = 0, launches = 0;
    uint64_t pver_seq = 0;  // source of Slot::pver
    int graph_rebuilds = 0;
    std::vector<float> lat_ms;
    size_t lat_pos = 0;
    double last_ms = 0;
    bool host_outputs = true;
    bool profiling = false;
    std::vector<gpud_stage_time> stage_times;
    // StreamingExtractGPU bookkeeping
    std::map<int64_t, int> by_signal;
};

static int set_err(gpud_runner *r, int code, const char *what, cudaError_t e = cudaSuccess) {
    char buf[256];
    if (e != cudaSuccess)
        std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    else
        std::snprintf(buf, sizeof buf, "%s", what);
    r->err = buf;
    return code;
}

#define CK(call)                                                          \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return set_err(r, GPUD_E_CUDA, #call, e_); \
    } while (0)

template <typename T>
static cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

static void prof_mark(gpud_runner *r, Frame &f, const char *name) {
    if (!r->profiling) return;
    if ((int)f.prof_ev.size() <= f.prof_n) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        f.prof_ev.push_back(e);
        f.prof_names.emplace_back();
    }
    cudaEventRecord(f.prof_ev[(size_t)f.prof_n], f.s);
    f.prof_names[(size_t)f.prof_n] = name;
    f.prof_n++;
}

// Per-kernel times of a completed frame.  Intervals that only cover a wait on
// the other frame ("wait_*" marks) are reported under their own names.
static void prof_collect(gpud_runner *r, Frame &f) {
    if (!r->profiling || f.prof_n < 2) return;
    r->stage_times.clear();
    for (int i = 0; i + 1 < f.prof_n; ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, f.prof_ev[(size_t)i], f.prof_ev[(size_t)i + 1]);
        gpud_stage_time t{};
        std::snprintf(t.name, sizeof t.name, "%s", f.prof_names[(size_t)i].c_str());
        t.ms = ms;
        r->stage_times.push_back(t);
    }
    if (f.ring >= 0) {  // the block's copy into the input ring, on the copy stream
        float ms = 0;
        cudaEventElapsedTime(&ms, r->ring_t0[f.ring], r->ring_copied[f.ring]);
        gpud_stage_time t{};
        std::snprintf(t.name, sizeof t.name, "%s", "h2d_ring");
        t.ms = ms;
        r->stage_times.push_back(t);
    }
}

// Bytes of per-block buffers one slot needs at max_block (both frames).
static uint64_t slot_block_bytes(const gpud_runner *r, int D, int mode, int flags) {
    uint64_t nout = (uint64_t)r->max_block / (uint64_t)D + 2;
    uint64_t b = nout * 8;  // extracted IQ (in the output arena)
    bool wfm = mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    if (wfm) b += 5 * (nout + 8) * 4;  // composite work arrays
    if (mode != GPUD_MODE_IQ) b += nout * 4 * (mode == GPUD_MODE_WFM_STEREO ? 2 : 1);
    if (wfm && (flags & GPUD_CH_RDS)) b += (nout / 16 + 4) * 8;
    if (flags & GPUD_CH_AUDIO48K) {
        // s16le at 48 kHz: at most nout * 48000 / out_rate + 2 frames
        uint64_t out_rate = (uint64_t)r->fs / (uint64_t)D;
        b += (nout * 48000 / out_rate + 4) * 2 * (mode == GPUD_MODE_WFM_STEREO ? 2 : 1);
    }
    return kFrames * b;
}

static uint64_t slot_state_bytes(const gpud_runner *r) {
    return sizeof(ChanParams) + sizeof(ChanState) + (uint64_t)r->tapcap * 2 * 4 + (uint64_t)2 * r->max_taps * 8 +
           (kWfmHist * 3 + kAudioDlStrideH) * 8 + sizeof(AudState) + kD1Taps * 8 + kWfmHist * 8;
}

// NewResampler (dsp/resample.go:45-93, 256-295): L/M from the gcd, odd
// prototype of L*32(+1) taps, windowed sinc fc = 0.90/max(L, M), Kaiser
// beta 6 (bessel0 series), gain L, split into L arms of K taps.
static double rs_bessel0(double x) {
    double sum = 1.0, term = 1.0;
    for (int k = 1; k < 30; k++) {
        term *= (x / (2 * (double)k)) * (x / (2 * (double)k));
        sum += term;
        if (term < 1e-12 * sum) break;
    }
    return sum;
}

static int rs_gcd(int a, int b) {
    while (b != 0) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a < 0 ? -a : a;
}

constexpr int kRsMaxArms = 1 << 17;  // any 48 kHz ratio from an integer rate up to 6 GS/s

static bool build_rs_bank(int in_rate, int out_rate, RsBank *bk, std::vector<double> &arms) {
    std::memset(bk, 0, sizeof *bk);
    const int g = rs_gcd(in_rate, out_rate);
    const int l = out_rate / g, m = in_rate / g;
    if (l > kRsMaxArms) return false;
    int plen = l * 32;
    if (plen % 2 == 0) plen++;
    const int k = (plen + l - 1) / l;
    if (k > kRsTaps) return false;
    arms.assign((size_t)l * k, 0.0);
    const double fc = 0.90 / (double)std::max(l, m);
    const double mid = (double)(plen - 1) / 2.0, b0 = rs_bessel0(6.0);
    for (int p = 0; p < l; ++p)
        for (int t = 0; t < k; ++t) {
            const int n = p + t * l;
            double v = 0.0;
            if (n < plen) {
                const double x = (double)n - mid;
                const double sn = std::fabs(x) < 1e-12 ? 2 * GPUD_PI * fc : std::sin(2 * GPUD_PI * fc * x) / x;
                const double xx = x / mid;
                v = sn * (rs_bessel0(6.0 * std::sqrt(1 - xx * xx)) / b0) * (double)l;
            }
            arms[(size_t)p * k + t] = v;
        }
    bk->L = l;
    bk->M = m;
    bk->K = k;
    return true;
}

static int rs_class_for(gpud_runner *r, int rate) {
    for (size_t i = 0; i < r->rs_rate.size(); ++i)
        if (r->rs_rate[i] == rate) return (int)i;
    if ((int)r->rs_rate.size() >= kMaxRsClasses) return -1;
    RsBank bk;
    std::vector<double> arms;
    if (!build_rs_bank(rate, 48000, &bk, arms)) return -1;
    const int id = (int)r->rs_rate.size();
    double *d_arm = nullptr;
    if (cudaMalloc((void **)&d_arm, arms.size() * sizeof(double)) != cudaSuccess) return -1;
    r->rs_arms.push_back(d_arm);
    bk.arm = d_arm;
    // a new bank id is not referenced by any block in flight
    if (cudaMemcpyAsync(d_arm, arms.data(), arms.size() * sizeof(double), cudaMemcpyHostToDevice, r->admin) !=
            cudaSuccess ||
        cudaMemcpyAsync(r->d_banks + id, &bk, sizeof(RsBank), cudaMemcpyHostToDevice, r->admin) != cudaSuccess)
        return -1;
    if (cudaStreamSynchronize(r->admin) != cudaSuccess) return -1;
    r->rs_rate.push_back(rate);
    r->rs_lmk.push_back(make_int3(bk.L, bk.M, bk.K));
    return id;
}

// Resampler.Process over n inputs from phase counter t0 (dsp/resample.go:
// 105-153): frames produced and the counter after, including the method's
// exit inside its consume loop (the counter is reduced by L for the sample it
// could not consume).  Output o is produced iff floor((t0+oM)/L) <= n and, for
// o >= 1, floor((t0+(o-1)M)/L) < n.
static void rs_advance(int64_t L, int64_t M, int64_t t0, int64_t n, int64_t *nout, int64_t *t1) {
    if (n <= 0) {
        *nout = 0;
        *t1 = t0;
        return;
    }
    if (L == M) {
        *nout = n;
        *t1 = t0;
        return;
    }
    auto cdiv = [](int64_t a, int64_t b) { return a >= 0 ? (a + b - 1) / b : -((-a) / b); };
    const int64_t A = cdiv((n + 1) * L - t0, M) - 1;
    int64_t last = -1;
    if (A >= 0) last = std::max<int64_t>(0, std::min(A, cdiv(n * L - t0, M)));
    const int64_t c_last = last >= 0 ? (t0 + last * M) / L : 0;
    *nout = last + 1;
    *t1 = t0 + (last + 1) * M - n * L - (c_last < n ? L : 0);
}

static int rate_class_for(gpud_runner *r, int rate) {
    for (size_t i = 0; i < r->class_rate.size(); ++i)
        if (r->class_rate[i] == rate) return (int)i;
    if ((int)r->class_rate.size() >= kMaxWfmClasses) return -1;
    int id = (int)r->class_rate.size();
    WfmTapsHost h{};
    auto t15 = lowpass_fir(15000, rate, 101), t53 = lowpass_fir(53000, rate, 101), t23 = lowpass_fir(23000, rate, 101),
         t21 = lowpass_fir(21000, rate, 101), t17 = lowpass_fir(17000, rate, 101), t75 = lowpass_fir(7500, rate, 101);
    for (int k = 0; k < kWfmTapsPadH; ++k) {
        if (k < kWfmTaps) {
            h.t[k][0] = (float)t15[(size_t)k];
            h.t[k][1] = (float)(t53[(size_t)k] - t23[(size_t)k]);
            h.t[k][2] = (float)(t21[(size_t)k] - t17[(size_t)k]);
            h.t[k][3] = 0.f;
            h.rds[k] = t75[(size_t)k];
        } else {
            h.t[k][0] = h.t[k][1] = h.t[k][2] = h.t[k][3] = 0.f;
        }
    }
    BinadeTable tab, tab38;
    build_binade_table(-2 * GPUD_PI * (-57000.0) / (double)rate, &tab);  // RDS FreqShift (fm.go:152)
    build_binade_table(2 * GPUD_PI * 38000.0 / (double)rate, &tab38);    // free-running stereo (fm.go:107)
    // a new class id is not referenced by any block in flight
    if (cudaMemcpyAsync(r->d_wtaps + id, &h, sizeof h, cudaMemcpyHostToDevice, r->admin) != cudaSuccess) return -1;
    if (cudaMemcpyAsync(r->d_tabs + id, &tab, sizeof tab, cudaMemcpyHostToDevice, r->admin) != cudaSuccess ||
        cudaMemcpyAsync(r->d_tabs + kMaxWfmClasses + id, &tab38, sizeof tab38, cudaMemcpyHostToDevice, r->admin) !=
            cudaSuccess)
        return -1;
    if (cudaStreamSynchronize(r->admin) != cudaSuccess) return -1;
    r->class_rate.push_back(rate);
    return id;
}

// Tap design of gpudemod/stream_state.go:57-77 (cutoff = max(BW/2, 200),
// LowpassFIR in float64, cast to float32, the first T taps applied), laid out
// phase-major (p*L + u -> h[p + u*D]) and direct.
static void design_taps(gpud_runner *r, const Slot &s, double bandwidth, std::vector<float> &pm,
                        std::vector<float> &h, double *cutoff_out) {
    double cutoff = bandwidth / 2;
    if (cutoff < 200) cutoff = 200;
    auto base = lowpass_fir(cutoff, r->fs, s.T);
    h.assign((size_t)s.T, 0.f);
    for (int k = 0; k < s.T; ++k) h[(size_t)k] = (float)base[(size_t)k];
    pm.assign((size_t)s.P * s.L, 0.f);
    for (int p = 0; p < s.P; ++p)
        for (int u = 0; u < s.L; ++u) {
            int k = p + u * s.D;
            pm[(size_t)p * s.L + u] = k < s.T ? h[(size_t)k] : 0.f;
        }
    *cutoff_out = cutoff;
}

// Rate of the demodulator and everything after it.
static int demod_rate(const Slot &s) { return s.spec.out_rate / std::max(1, s.d1); }

// FM discriminators on an oversampled channel (output rate well above the
// signal bandwidth) see consecutive samples that differ little, and magnify
// the white rounding error of each extraction output; such channels add the
// float32 sums of the polyphase rows in float64.
static bool precise_sum(const gpud_channel_spec &sp) {
    bool fm = sp.mode == GPUD_MODE_NFM || sp.mode == GPUD_MODE_WFM || sp.mode == GPUD_MODE_WFM_STEREO;
    return fm && (double)sp.out_rate >= 4.0 * std::max(sp.bandwidth, 400.0);
}

static void fill_params(gpud_runner *r, int slot, ChanParams *p) {
    Slot &s = r->slots[(size_t)slot];
    std::memset(p, 0, sizeof *p);
    double inc = -2.0 * GPUD_PI * s.spec.offset_hz / (double)r->fs;
    p->inc_q = rad_to_q64(inc);
    p->inc_rad = inc;
    p->decim = s.D;
    p->ntaps = s.T;
    p->nphase = s.P;
    p->plen = s.L;
    p->mode = s.spec.mode;
    p->flags = s.spec.flags;
    p->precise_sum = precise_sum(s.spec) ? 1 : 0;
    p->out_rate = demod_rate(s);
    p->taps_off = s.taps_off;
    p->dtaps_off = s.dtaps_off;
    p->hist_off = s.hist_off;
    p->hcap = s.hcap;
    p->wfm_idx = s.wfm_idx;
    int rate = demod_rate(s);
    p->rds_dr = std::max(1, rate / 19000);
    double bfo = s.spec.mode == GPUD_MODE_LSB ? -700.0 : 700.0;
    p->ssb_inc = 2 * GPUD_PI * bfo / (double)rate;
    pll_coefficients(50, 0.707, rate, &p->pll_alpha, &p->pll_beta);
    p->pll_lpa = 1 - std::exp(-2 * GPUD_PI * 200 / (double)rate);
    p->pll_fmin = 2 * GPUD_PI * 17000 / (double)rate;
    p->pll_fmax = 2 * GPUD_PI * 21000 / (double)rate;
    p->rds_inc = -2 * GPUD_PI * (-57000.0) / (double)rate;
    p->rds_tab = s.rate_class < 0 ? 0 : s.rate_class;
    p->rs_bank = s.rs_class < 0 ? 0 : s.rs_class;
    p->aud_ch = s.aud_ch;
    // de-emphasis tau (recorder/streamer.go:1443-1463): 50 us default, WFM only
    const bool wfm = s.spec.mode == GPUD_MODE_WFM || s.spec.mode == GPUD_MODE_WFM_STEREO;
    double tau_us = (s.spec.flags & GPUD_CH_DEEMPH75) ? 75.0 : 50.0;
    if (s.spec.flags & GPUD_CH_NO_DEEMPH) tau_us = 0.0;
    if (s.deemph_us >= 0.0) tau_us = s.deemph_us;
    p->deemph_a = (wfm && tau_us > 0) ? std::exp(-1.0 / (48000.0 * tau_us * 1e-6)) : 0.0;
    p->d1 = s.d1;
}

static void queue_write(gpud_runner *r, int slot, void *dst, const void *src, size_t bytes) {
    PendingOp op;
    op.slot = slot;
    op.dst = dst;
    op.data.assign((const char *)src, (const char *)src + bytes);
    r->pending.push_back(std::move(op));
}

static void drop_pending(gpud_runner *r, int slot) {
    r->pending.erase(std::remove_if(r->pending.begin(), r->pending.end(),
                                    [slot](const PendingOp &op) { return op.slot == slot; }),
                     r->pending.end());
}

static int validate_spec(gpud_runner *r, const gpud_channel_spec *spec, int *D, int *T) {
    if (!spec) return set_err(r, GPUD_E_ARG, "null channel spec");
    if (spec->mode < 0 || spec->mode > GPUD_MODE_CW) return set_err(r, GPUD_E_MODE, "unknown mode");
    if (r->fs <= 0 || spec->out_rate <= 0 || r->fs % spec->out_rate != 0)
        return set_err(r, GPUD_E_DECIM, "streaming polyphase extractor requires integer decimation");
    *D = r->fs / spec->out_rate;
    *T = spec->num_taps > 0 ? spec->num_taps : 101;
    if (*T > r->max_taps) return set_err(r, GPUD_E_TAPS, "num_taps above the runner's max_taps");
    int P = std::min(*D, *T), L = (*T + *D - 1) / *D;
    if ((int64_t)P * L > r->tapcap || *T > r->tapcap) return set_err(r, GPUD_E_TAPS, "tap layout too large");
    if (spec->demod_decim < 0 || spec->demod_decim > 64 ||
        (spec->demod_decim > 1 && spec->out_rate / spec->demod_decim < 1000))
        return set_err(r, GPUD_E_DECIM, "demod_decim out of range");
    return 0;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// ---------------------------------------------------------------------------
// block completion
// ---------------------------------------------------------------------------
static void record_latency(gpud_runner *r, Frame &f) {
    float ms = 0;
    cudaEventElapsedTime(&ms, f.ev_start ? f.ev_start : f.ev0, f.ev1);
    r->last_ms = ms;
    r->lat_ms[r->lat_pos % r->lat_ms.size()] = ms;
    r->lat_pos++;
}

static int finish_frame(gpud_runner *r, int fi, int timeout_ms) {
    Frame &f = r->fr[fi];
    if (!f.inflight) return 0;
    if (timeout_ms < 0) {
        CK(cudaEventSynchronize(f.ev_done));
    } else {
        double waited = 0;
        while (true) {
            cudaError_t q = cudaEventQuery(f.ev_done);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return set_err(r, GPUD_E_CUDA, "event query", q);
            if (waited >= timeout_ms) return set_err(r, GPUD_E_TIMEOUT, "wait timed out");
            struct timespec ts{0, 50000};
            nanosleep(&ts, nullptr);
            waited += 0.05;
        }
    }
    f.inflight = false;
    if (f.ticket > r->completed) r->completed = f.ticket;
    r->done_frame = fi;
    record_latency(r, f);
    if (f.ring >= 0) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r->ring_t0[f.ring], r->ring_copied[f.ring]) == cudaSuccess) {
            r->ring_ms += ms;
            r->ring_copies++;
        }
        cudaGetLastError();
    }
    prof_collect(r, f);
    if (r->h_fault && *(volatile unsigned *)r->h_fault != 0) {
        const unsigned code = *(volatile unsigned *)r->h_fault;
        *(volatile unsigned *)r->h_fault = 0;
        return set_err(r, GPUD_E_DEVICE_STATUS,
                       code == 1 ? "extraction: producer wait for a free staging buffer gave up"
                                 : "extraction: wait for a staged tile gave up");
    }
    return 0;
}

// Wait for every block in flight (oldest first).
static int oldest_inflight(const gpud_runner *r) {
    int a = -1;
    for (int k = 0; k < kFrames; ++k)
        if (r->fr[k].inflight && (a < 0 || r->fr[k].ticket < r->fr[a].ticket)) a = k;
    return a;
}

static int drain(gpud_runner *r) {
    for (int a = oldest_inflight(r); a >= 0; a = oldest_inflight(r)) {
        int rc = finish_frame(r, a, -1);
        if (rc) return rc;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// block planning
// ---------------------------------------------------------------------------

static void plan_slot(gpud_runner *r, BlockPlan &pl, int slot, int n) {
    Slot &s = r->slots[(size_t)slot];
    SlotBlock sb{};
    sb.slot = slot;
    sb.pc = s.pc;
    sb.n_out = (s.pc + n) / s.D;
    sb.hist_len = s.hist_len;
    sb.hist_sel = s.hist_sel;
    // demodulator input: the extraction output, or the samples the pre-demod
    // decimator emits (those with phase counter 0: d1_phase + j*d1)
    sb.d1_phase = s.d1_phase;
    sb.ng = s.ng;
    sb.pg = s.pg;
    sb.n_dem = sb.n_out;
    if (s.d1 > 1) sb.n_dem = sb.n_out > s.d1_phase ? (sb.n_out - 1 - s.d1_phase) / s.d1 + 1 : 0;
    int mode = s.spec.mode;
    bool fm = mode == GPUD_MODE_NFM || mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    bool wfm = mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    sb.n_disc = 0;
    sb.bridge = 0;
    if (fm && sb.n_dem > 0) {
        sb.bridge = s.has_last ? 1 : 0;
        sb.n_disc = s.has_last ? sb.n_dem : sb.n_dem - 1;
    }
    switch (mode) {
    case GPUD_MODE_NFM:
    case GPUD_MODE_WFM: sb.n_audio = sb.n_disc; break;
    case GPUD_MODE_WFM_STEREO: sb.n_audio = 2 * sb.n_disc; break;
    case GPUD_MODE_AM:
    case GPUD_MODE_USB:
    case GPUD_MODE_LSB:
    case GPUD_MODE_CW: sb.n_audio = sb.n_dem; break;
    default: sb.n_audio = 0;
    }
    sb.comp_hist_len = s.comp_hist_len;
    sb.n_rds = 0;
    sb.rds_first = -1;
    if (wfm && (s.spec.flags & GPUD_CH_RDS) && sb.n_disc > 0) {
        int dr = std::max(1, demod_rate(s) / 19000);
        int64_t c0 = s.rds_count;
        int qf = (int)((dr - c0 % dr) % dr);
        if (qf < sb.n_disc) {
            sb.rds_first = qf;
            sb.n_rds = (sb.n_disc - 1 - qf) / dr + 1;
        }
    }
    sb.rs_t0 = (int)s.rs_t;
    sb.rs_nout = sb.rs_frames = sb.pcm_off = 0;
    if ((s.spec.flags & GPUD_CH_AUDIO48K) && s.rs_class >= 0 && sb.n_audio > 0) {
        int64_t nout, t1;
        sb.rs_frames = sb.n_audio / s.aud_ch;
        rs_advance(s.rs_L, s.rs_M, s.rs_t, sb.rs_frames, &nout, &t1);
        sb.rs_nout = (int)nout;
    }
    sb.res_idx = (int)pl.sbs.size();
    pl.sbs.push_back(sb);
}

// Offsets (emitting slots' IQ first so one D2H covers it) and work lists.
// Tensor-core channel groups of a block: dense-form channels with the same
// decimation (a multiple of 4), tap count and phase count share the input
// grid; groups of at least kGemmMinChannels (split to fit shared memory) take
// every output from kGemmFirstOutput on in the group kernel.  Float64-summed
// channels stay on the dense kernel.  Returns the grouped flag of every row.
static std::vector<char> plan_gemm_groups(gpud_runner *r, BlockPlan &pl) {
    pl.groups.clear();
    pl.gmembers.clear();
    pl.w_gemm.clear();
    pl.gemm_smem = pl.gemm_max_l = 0;
    pl.gemm_b_bytes = 0;
    std::vector<char> grouped(pl.sbs.size(), 0);
    if (!GPUD_GEMM_EXTRACT || !r->channel_groups || !r->d_fault) return grouped;
    std::map<std::tuple<int, int, int>, std::vector<int>> by_key;
    for (int i = 0; i < (int)pl.sbs.size(); ++i) {
        const SlotBlock &sb = pl.sbs[(size_t)i];
        const Slot &s = r->slots[(size_t)sb.slot];
        if (s.ext_kind != 0 || s.D % 4 != 0 || precise_sum(s.spec) || sb.n_out <= kGemmFirstOutput) continue;
        by_key[std::make_tuple(s.D, s.T, sb.pc)].push_back(i);
    }
    for (auto &kv : by_key) {
        const std::vector<int> &rows = kv.second;
        if ((int)rows.size() < kGemmMinChannels) continue;
        const int D = std::get<0>(kv.first), T = std::get<1>(kv.first), pc = std::get<2>(kv.first);
        const int L = (T + D - 1) / D;
        int cmax = 0;  // most channels per group (a multiple of 8) with two taps stages in shared memory
        for (int c = 8; c <= 128; c += 8)
            if (gemm_smem_bytes_host(D, L, 2 * c, 2) <= kGemmSmemCap) cmax = c;
        if (cmax < kGemmMinChannels) continue;
        const int nchunk = ((int)rows.size() + cmax - 1) / cmax;
        const int per = ((int)rows.size() + nchunk - 1) / nchunk;
        for (int c0 = 0; c0 < (int)rows.size(); c0 += per) {
            const int C = std::min(per, (int)rows.size() - c0);
            if (C < kGemmMinChannels) break;
            GemmGroup g{};
            g.nmem = C;
            g.ncol = ((2 * C + 15) / 16) * 16;
            g.D = D;
            g.L = L;
            g.T = T;
            g.pc = pc;
            g.n_out = pl.sbs[(size_t)rows[(size_t)c0]].n_out;
            g.jt0 = kGemmFirstOutput;
            g.ns = gemm_smem_bytes_host(D, L, g.ncol, 3) <= kGemmSmemCap ? 3 : 2;
#if GPUD_GEMM_PAIR
            // one taps stage when two CTAs then fit on an SM: one CTA's MMAs
            // overlap the other's staging and epilogue
            if (2 * (gemm_smem_bytes_host(D, L, g.ncol, 1) + 1024) <= 228 * 1024) g.ns = 1;
#endif
            // accumulators: as many arms apart as fit in the TMEM share of one
            // of the CTAs that the shared memory lets reside on an SM
            {
                const int per_sm = std::max(1, (228 * 1024) / (gemm_smem_bytes_host(D, L, g.ncol, g.ns) + 1024));
                int p2 = 1;
                while (p2 < std::min(per_sm, 4)) p2 <<= 1;
                const int cols = 512 / p2;  // a power-of-two share: the allocations of resident CTAs never wait
                g.na = std::max(1, std::min(L, cols / g.ncol));
            }
            g.b_off = (int)pl.gemm_b_bytes;
            g.mem_off = (int)pl.gmembers.size();
            pl.gemm_b_bytes += align256(gemm_pack_bytes_host(D, L, g.ncol));
            pl.gemm_smem = std::max(pl.gemm_smem, gemm_smem_bytes_host(D, L, g.ncol, g.ns));
            pl.gemm_max_l = std::max(pl.gemm_max_l, L);
            const int gi = (int)pl.groups.size();
            for (int k = 0; k < C; ++k) {
                pl.gmembers.push_back(rows[(size_t)(c0 + k)]);
                grouped[(size_t)rows[(size_t)(c0 + k)]] = 1;
            }
            for (int t = 0; kGemmFirstOutput + t * gemm_tile() < g.n_out; ++t) pl.w_gemm.push_back(make_int2(gi, t));
            pl.groups.push_back(g);
        }
    }
    return grouped;
}

// Short-arm channel banks of a block: channels of the warp-per-output or the
// modulated short-arm form (T <= 4D), not float64-summed, that share the
// decimation, tap count and phase count, and are not in a tensor-core group,
// form a bank when there are at least kBankMinChannels of them.  A bank takes
// every output from jt0 on: the first output whose window lies inside the
// block; the warp-per-output kernel keeps the outputs before it (they reach
// into the carried history).  A bank's work items hold 8r outputs, r = 4
// unless the bank then gives fewer than two items per SM.  Returns the first
// banked output of every row (-1: not banked).
static std::vector<int> plan_bank_groups(gpud_runner *r, BlockPlan &pl, const std::vector<char> &grouped) {
    pl.banks.clear();
    pl.bmembers.clear();
    pl.w_bank.clear();
    pl.bank_g = 0;
    pl.bank_max_total = 0;
    std::vector<int> first(pl.sbs.size(), -1);
    if (!GPUD_BANK_EXTRACT || !r->channel_groups) return first;
    std::map<std::tuple<int, int, int>, std::vector<int>> by_key;
    for (int i = 0; i < (int)pl.sbs.size(); ++i) {
        const SlotBlock &sb = pl.sbs[(size_t)i];
        const Slot &s = r->slots[(size_t)sb.slot];
        if (grouped[(size_t)i] || (s.ext_kind != 1 && s.ext_kind != 3) || precise_sum(s.spec) || s.L > kBankMaxL)
            continue;
        by_key[std::make_tuple(s.D, s.T, sb.pc)].push_back(i);
    }
    for (auto &kv : by_key) {
        const std::vector<int> &rows = kv.second;
        if ((int)rows.size() < kBankMinChannels) continue;
        const int D = std::get<0>(kv.first), T = std::get<1>(kv.first), pc = std::get<2>(kv.first);
        const int s0 = D - pc - 1;
        // first output j with s0 + j*D - (T-1) >= 0, rounded up to a wide tile
        const int jb = T - 1 > s0 ? (T - 1 - s0 + D - 1) / D : 0;
        const int n_out = pl.sbs[(size_t)rows[0]].n_out;
        if (n_out <= jb) continue;
        BankGroup b{};
        b.nmem = (int)rows.size();
        b.cpad = (b.nmem + bank_lanes() - 1) / bank_lanes() * bank_lanes();
        b.D = D;
        b.T = T;
        b.pc = pc;
        b.n_out = n_out;
        b.jt0 = jb;
        b.mem_off = (int)pl.bmembers.size();
        b.g_off = (int)pl.bank_g;
        const int nch = b.cpad / bank_lanes();
        b.r = 4;
        while (b.r > 1 && (int64_t)(n_out - jb + 8 * b.r - 1) / (8 * b.r) * nch < 2 * r->num_sms) b.r >>= 1;
        pl.bank_g += ((int64_t)T * b.cpad + 63) & ~63;
        pl.bank_max_total = std::max(pl.bank_max_total, T * b.cpad);
        const int bi = (int)pl.banks.size();
        for (int row : rows) {
            pl.bmembers.push_back(row);
            first[(size_t)row] = jb;
        }
        const int tile = bank_warps() * b.r;
        for (int t = 0; jb + t * tile < n_out; ++t)
            for (int c = 0; c < nch; ++c) pl.w_bank.push_back(make_int2(bi, t * nch + c));
        pl.banks.push_back(b);
    }
    return first;
}

static void finish_plan(gpud_runner *r, BlockPlan &pl) {
    int64_t ext = 0;
    pl.tot_emit_ext = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (auto &sb : pl.sbs) {
            bool emit = (r->slots[(size_t)sb.slot].spec.flags & GPUD_CH_EMIT_IQ) != 0;
            if (emit != (pass == 0)) continue;
            sb.ext_off = (int)ext;
            ext += (sb.n_out + 3) & ~3;
            if (pass == 0) pl.tot_emit_ext = ext;
        }
    // pre-demod decimator outputs after every extraction output
    for (auto &sb : pl.sbs) {
        if (r->slots[(size_t)sb.slot].d1 > 1) {
            sb.dem_off = (int)ext;
            ext += (sb.n_dem + 3) & ~3;
        } else {
            sb.dem_off = sb.ext_off;
        }
    }
    pl.tot_ext = ext;
    int64_t comp = 0, audio = 0, rds = 0, pcm = 0;
    // demod-rate audio: channels that return it to the host first, then those
    // whose audio only feeds the 48 kHz back end on the device
    pl.tot_audio_host = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (auto &sb : pl.sbs) {
            const bool dev = (r->slots[(size_t)sb.slot].spec.flags & GPUD_CH_AUDIO48K) != 0;
            if (dev != (pass == 1)) continue;
            sb.audio_off = (int)audio;
            audio += (sb.n_audio + 3) & ~3;
            if (pass == 0) pl.tot_audio_host = audio;
        }
    pl.aud_list.clear();
    pl.w_aud.clear();
    pl.w_dec.clear();
    for (int i = 0; i < (int)pl.sbs.size(); ++i) {
        SlotBlock &sb = pl.sbs[(size_t)i];
        Slot &s = r->slots[(size_t)sb.slot];
        sb.comp_off = (int)comp;
        if (s.wfm_idx >= 0) comp += (sb.n_disc + 8 + 7) & ~7;
        sb.rds_off = (int)rds;
        rds += (sb.n_rds + 1) & ~1;
        sb.pcm_off = (int)pcm;
        // int16 slots; float32 PCM takes two per sample
        pcm += ((int64_t)sb.rs_nout * s.aud_ch * ((s.spec.flags & GPUD_CH_PCM_F32) ? 2 : 1) + 7) & ~7;
        if (sb.rs_frames > 0) {
            pl.aud_list.push_back(i);
            for (int t = 0; t * audio48_tile() < sb.rs_nout; ++t) pl.w_aud.push_back(make_int2(i, t));
        }
    }
    pl.tot_comp = comp;
    pl.tot_audio = audio;
    pl.tot_rds = rds;
    pl.tot_pcm = pcm;
    for (int L = 0; L <= kDenseMaxL; ++L) {
        pl.w_dense[L].clear();
        pl.dense_smem[L] = 0;
        pl.dense_pmax[L] = 0;
    }
    pl.w_wide.clear();
    pl.wide_smem = 0;
    pl.w_group.clear();
    pl.group_smem = 0;
    pl.w_mod.clear();
    pl.mod_smem = 0;
    pl.w_demod.clear();
    pl.w_am.clear();
    pl.w_fir.clear();
    pl.w_out.clear();
    pl.w_rds.clear();
    pl.pll_list.clear();
    pl.w_free.clear();
    pl.batch_stereo = false;
    pl.rds_smem = 0;
    std::vector<char> grouped = plan_gemm_groups(r, pl);
    const std::vector<int> banked = plan_bank_groups(r, pl, grouped);
    for (int i = 0; i < (int)pl.sbs.size(); ++i) {
        const SlotBlock &sb = pl.sbs[(size_t)i];
        Slot &s = r->slots[(size_t)sb.slot];
        if (sb.n_out > 0 && banked[(size_t)i] >= 0) {
            // a banked channel keeps only the outputs before its bank's first one here
            pl.sbs[(size_t)i].wide_end = std::max(1, banked[(size_t)i]);
            if (banked[(size_t)i] > 0) {
                for (int t = 0; t * kWideTile < banked[(size_t)i]; ++t) pl.w_wide.push_back(make_int2(i, t));
                pl.wide_smem = std::max(pl.wide_smem, wide_smem_bytes_host(s.T));
            }
        } else if (sb.n_out > 0) {
            if (s.ext_kind == 0) {
                // a grouped channel keeps only the outputs before kGemmFirstOutput here
                const int n_dense = grouped[(size_t)i] ? kGemmFirstOutput : sb.n_out;
                for (int t = 0; t * dense_tile() < n_dense; ++t) pl.w_dense[s.L].push_back(make_int2(i, t));
                pl.dense_smem[s.L] = std::max(pl.dense_smem[s.L], dense_smem_bytes_host(s.P, s.L));
                pl.dense_pmax[s.L] = std::max(pl.dense_pmax[s.L], s.P);
            } else if (s.ext_kind == 2 || s.ext_kind == 3) {
                auto &wl = s.ext_kind == 2 ? pl.w_group : pl.w_mod;
                for (int t = 0; t * dense_tile() < sb.n_out; ++t) wl.push_back(make_int2(i, t));
                if (s.ext_kind == 2)
                    pl.group_smem = std::max(pl.group_smem, group_smem_bytes_host(s.pg, s.L));
                else
                    pl.mod_smem = std::max(pl.mod_smem, mod_smem_bytes_host(s.pg, s.L));
            } else {
                for (int t = 0; t * kWideTile < sb.n_out; ++t) pl.w_wide.push_back(make_int2(i, t));
                pl.wide_smem = std::max(pl.wide_smem, wide_smem_bytes_host(s.T));
            }
        }
        int mode = s.spec.mode;
        int nd = (mode == GPUD_MODE_USB || mode == GPUD_MODE_LSB || mode == GPUD_MODE_CW) ? sb.n_dem : sb.n_disc;
        if ((mode >= GPUD_MODE_NFM && mode <= GPUD_MODE_WFM_STEREO) || mode >= GPUD_MODE_USB)
            for (int t = 0; t * 1024 < nd; ++t) pl.w_demod.push_back(make_int2(i, t));
        if (mode == GPUD_MODE_AM && sb.n_dem > 0) pl.w_am.push_back(make_int2(i, 0));
        if (s.d1 > 1)
            for (int t = 0; t * decim2_tile() < sb.n_dem; ++t) pl.w_dec.push_back(make_int2(i, t));
        if (mode == GPUD_MODE_WFM_STEREO && sb.n_disc > 0) {
            for (int t = 0; t * 1024 < sb.n_disc; ++t) pl.w_fir.push_back(make_int2(i, t));
            if (s.spec.flags & GPUD_CH_FREE_STEREO) {
                for (int t = 0; t * 1024 < sb.n_disc; ++t) pl.w_free.push_back(make_int2(i, t));
            } else {
                pl.pll_list.push_back(i);
                if (s.spec.flags & GPUD_CH_BATCH_STEREO) pl.batch_stereo = true;
            }
        }
        if ((mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO) && sb.n_disc > 0)
            for (int t = 0; t * 1024 < sb.n_disc; ++t) pl.w_out.push_back(make_int2(i, t));
        if (sb.n_rds > 0) {
            for (int t = 0; t * rds_tile() < sb.n_rds; ++t) pl.w_rds.push_back(make_int2(i, t));
            pl.rds_smem = std::max(pl.rds_smem, rds_smem_bytes(std::max(1, demod_rate(s) / 19000)));
        }
    }
    // a phase-grouped tile costs its channel's phases x arm length: the
    // longest go first, so that the short ones fill in behind them
    auto longest_first = [&](std::vector<int2> &wl) {
        std::stable_sort(wl.begin(), wl.end(), [&](int2 a, int2 b) {
            const Slot &sa = r->slots[(size_t)pl.sbs[(size_t)a.x].slot], &sb = r->slots[(size_t)pl.sbs[(size_t)b.x].slot];
            return (int64_t)sa.P * sa.L > (int64_t)sb.P * sb.L;
        });
    };
    longest_first(pl.w_group);
    longest_first(pl.w_mod);
}

static int ensure_frame(gpud_runner *r, Frame &f, const BlockPlan &pl) {
    int64_t W = std::max<int64_t>(pl.tot_comp, 8);
    if (W > f.wk_cap) {
        cudaFree(f.d_wk);
        f.d_wk = nullptr;
        int64_t cap = std::max<int64_t>(W * 5 / 4, 1 << 16);
        CK(dalloc(&f.d_wk, (size_t)cap * 5));
        f.wk_cap = cap;
        r->graph_rebuilds++;
    }
    if (pl.tot_pcm > f.rs_cap) {
        cudaFree(f.d_rs);
        f.d_rs = nullptr;
        int64_t cap = std::max<int64_t>(pl.tot_pcm * 5 / 4, 1 << 14);
        CK(dalloc(&f.d_rs, (size_t)cap));
        f.rs_cap = cap;
    }
    size_t res = align256(pl.sbs.size() * sizeof(DevResult));
    size_t need = res + align256((size_t)pl.tot_pcm * 2) + align256((size_t)pl.tot_audio * 4) +
                  align256((size_t)pl.tot_rds * 8) + align256((size_t)pl.tot_ext * 8);
    if (need > f.out_cap) {
        cudaFree(f.d_out);
        if (f.h_out) cudaFreeHost(f.h_out);
        f.d_out = nullptr;
        f.h_out = nullptr;
        size_t cap = need * 5 / 4 + 4096;
        CK(cudaMalloc((void **)&f.d_out, cap));
        CK(cudaMallocHost((void **)&f.h_out, cap));
        f.out_cap = cap;
        r->graph_rebuilds++;
    }
    size_t nw = 0;
    for (int L = 0; L <= kDenseMaxL; ++L) nw += pl.w_dense[L].size();
    nw += pl.w_wide.size() + pl.w_demod.size() + pl.w_am.size() + pl.w_fir.size() + pl.w_out.size() +
          pl.w_rds.size() + pl.w_aud.size() + pl.w_dec.size() + pl.w_group.size() +
          pl.w_mod.size() + pl.w_free.size() + pl.w_gemm.size() + pl.w_bank.size();
    size_t dneed = align256(pl.sbs.size() * sizeof(SlotBlock)) + align256(nw * sizeof(int2)) +
                   align256(pl.pll_list.size() * 4) + align256(pl.aud_list.size() * 4) +
                   align256(pl.groups.size() * sizeof(GemmGroup)) + align256(pl.gmembers.size() * 4) +
                   align256(pl.banks.size() * sizeof(BankGroup)) + align256(pl.bmembers.size() * 4) + 4096;
    if (pl.bank_g > f.bank_cap) {
        cudaFree(f.d_bank);
        f.d_bank = nullptr;
        int64_t cap = pl.bank_g * 5 / 4 + 1024;
        CK(dalloc(&f.d_bank, (size_t)cap));
        f.bank_cap = cap;
        f.bank_key.clear();  // a new buffer holds no packed taps
    }
    if (pl.gemm_b_bytes > f.gb_cap) {
        cudaFree(f.d_gb);
        f.d_gb = nullptr;
        size_t cap = pl.gemm_b_bytes * 5 / 4 + 4096;
        CK(cudaMalloc((void **)&f.d_gb, cap));
        f.gb_cap = cap;
        f.gb_key.clear();  // a new buffer holds no packed taps
    }
    if (dneed > f.desc_cap) {
        cudaFree(f.d_desc);
        if (f.h_desc) cudaFreeHost(f.h_desc);
        f.d_desc = nullptr;
        f.h_desc = nullptr;
        size_t cap = dneed * 5 / 4 + 4096;
        CK(cudaMalloc((void **)&f.d_desc, cap));
        CK(cudaMallocHost((void **)&f.h_desc, cap));
        f.desc_cap = cap;
    }
    size_t sneed = 0;
    for (auto &op : r->pending) sneed += align256(op.data.size());
    if (sneed > f.stage_cap) {
        if (f.h_stage) cudaFreeHost(f.h_stage);
        f.h_stage = nullptr;
        size_t cap = sneed * 5 / 4 + 4096;
        CK(cudaMallocHost((void **)&f.h_stage, cap));
        f.stage_cap = cap;
    }
    return 0;
}

// Host mirrors advance exactly as the device state does.
static void advance_mirrors(gpud_runner *r, const BlockPlan &pl, int n, std::vector<SlotAfter> *after) {
    if (after) after->clear();
    for (const SlotBlock &sb : pl.sbs) {
        Slot &s = r->slots[(size_t)sb.slot];
        s.pc = (s.pc + n) % s.D;
        s.hist_len = std::min(s.T - 1, s.hist_len + n);
        s.hist_sel = 1 - s.hist_sel;
        if (sb.n_dem > 0) s.has_last = true;
        if (s.d1 > 1) s.d1_phase = ((s.d1_phase - sb.n_out) % s.d1 + s.d1) % s.d1;
        if (s.wfm_idx >= 0) {
            s.comp_hist_len = std::min(kWfmHist, s.comp_hist_len + sb.n_disc);
            s.rds_count += sb.n_disc;
        }
        if (sb.rs_frames > 0) {
            int64_t nout, t1;
            rs_advance(s.rs_L, s.rs_M, s.rs_t, sb.rs_frames, &nout, &t1);
            s.rs_t = t1;
        }
        if (after) after->push_back(SlotAfter{s.pc, s.hist_len});
    }
}

static int stage_input(gpud_runner *r, Frame &f, const gpud_float2 *iq, int n, int on_device,
                       const float2 **x_dev) {
    if (n == 0) {
        *x_dev = f.d_block;
        return 0;
    }
    if (!iq) return set_err(r, GPUD_E_ARG, "null IQ block");
    if (on_device) {
        *x_dev = (const float2 *)iq;
        return 0;
    }
    cudaPointerAttributes at{};
    bool pinned = cudaPointerGetAttributes(&at, iq) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    const void *src = iq;
    if (!pinned) {
        std::memcpy(f.h_in, iq, (size_t)n * sizeof(float2));
        src = f.h_in;
    }
    CK(cudaMemcpyAsync(f.d_block, src, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice, f.s));
    f.h2d += (uint64_t)n * sizeof(float2);
    *x_dev = f.d_block;
    return 0;
}

// Enqueue one block on frame f: descriptors, front half, [wait prev back],
// back half, output D2H.  `prev` is the frame of the block before, or null.
static int enqueue_block(gpud_runner *r, Frame &f, const Frame *prev, BlockPlan &pl, const float2 *x_dev, int n) {
    // descriptor staging
    char *hd = f.h_desc;
    size_t o_sb = 0, o_w = align256(pl.sbs.size() * sizeof(SlotBlock));
    std::memcpy(hd + o_sb, pl.sbs.data(), pl.sbs.size() * sizeof(SlotBlock));
    int2 *hw = (int2 *)(hd + o_w);
    size_t cnt = 0;
    // Dense classes: the persistent kernel pays off with at least two tiles
    // per SM; smaller classes (e.g. the history tiles of grouped channels)
    // run one tile per CTA.  Such classes whose shared memory is within 2x of
    // each other go out as one launch (their tiles laid out contiguously,
    // largest footprint first), so that a dozen small classes fill the GPU
    // together instead of one after another.
    bool dense_pipe[kDenseMaxL + 1] = {};
    int dense_ng[kDenseMaxL + 1] = {};
    std::vector<int> tile_classes;
    for (int L = 0; L <= kDenseMaxL; ++L) {
        if (pl.w_dense[L].empty()) continue;
        const int ntiles = (int)pl.w_dense[L].size();
        dense_ng[L] = std::min(GPUD_DENSE_PIPE, dense_pipe_groups_host(pl.dense_pmax[L], L, kDensePipeSmemCap));
        dense_pipe[L] = dense_ng[L] > 0 && ntiles >= 2 * r->num_sms && r->d_fault && ((uintptr_t)x_dev & 15) == 0;
        if (!dense_pipe[L]) tile_classes.push_back(L);
    }
    std::stable_sort(tile_classes.begin(), tile_classes.end(),
                     [&](int a, int b) { return pl.dense_smem[a] > pl.dense_smem[b]; });
    struct DenseBatch {
        size_t off = 0, items = 0;
        int smem = 0, classes = 0, L = 0;
    };
    std::vector<DenseBatch> batches;
    size_t w_dense_off[kDenseMaxL + 1] = {};
    for (int L : tile_classes) {
        if (batches.empty() || 2 * pl.dense_smem[L] < batches.back().smem) {
            batches.emplace_back();
            batches.back().off = cnt;
            batches.back().smem = pl.dense_smem[L];
            batches.back().L = L;
        }
        DenseBatch &bt = batches.back();
        w_dense_off[L] = cnt;
        std::memcpy(hw + cnt, pl.w_dense[L].data(), pl.w_dense[L].size() * sizeof(int2));
        cnt += pl.w_dense[L].size();
        bt.items += pl.w_dense[L].size();
        bt.classes++;
    }
    for (int L = 0; L <= kDenseMaxL; ++L) {
        if (pl.w_dense[L].empty() || !dense_pipe[L]) continue;
        w_dense_off[L] = cnt;
        std::memcpy(hw + cnt, pl.w_dense[L].data(), pl.w_dense[L].size() * sizeof(int2));
        cnt += pl.w_dense[L].size();
    }
    auto put = [&](const std::vector<int2> &v) {
        size_t at = cnt;
        std::memcpy(hw + cnt, v.data(), v.size() * sizeof(int2));
        cnt += v.size();
        return at;
    };
    size_t o_wide = put(pl.w_wide), o_dem = put(pl.w_demod), o_am = put(pl.w_am), o_fir = put(pl.w_fir),
           o_out = put(pl.w_out), o_rds = put(pl.w_rds), o_waud = put(pl.w_aud), o_wdec = put(pl.w_dec),
           o_grp = put(pl.w_group), o_mod = put(pl.w_mod), o_free = put(pl.w_free),
           o_gemm = put(pl.w_gemm), o_bank = put(pl.w_bank);
    size_t o_pll = o_w + align256(cnt * sizeof(int2));
    std::memcpy(hd + o_pll, pl.pll_list.data(), pl.pll_list.size() * 4);
    size_t o_aud = o_pll + align256(pl.pll_list.size() * 4);
    std::memcpy(hd + o_aud, pl.aud_list.data(), pl.aud_list.size() * 4);
    size_t o_ggr = o_aud + align256(pl.aud_list.size() * 4);
    std::memcpy(hd + o_ggr, pl.groups.data(), pl.groups.size() * sizeof(GemmGroup));
    size_t o_gmem = o_ggr + align256(pl.groups.size() * sizeof(GemmGroup));
    std::memcpy(hd + o_gmem, pl.gmembers.data(), pl.gmembers.size() * 4);
    size_t o_bgr = o_gmem + align256(pl.gmembers.size() * 4);
    std::memcpy(hd + o_bgr, pl.banks.data(), pl.banks.size() * sizeof(BankGroup));
    size_t o_bmem = o_bgr + align256(pl.banks.size() * sizeof(BankGroup));
    std::memcpy(hd + o_bmem, pl.bmembers.data(), pl.bmembers.size() * 4);
    size_t dbytes = o_bmem + pl.bmembers.size() * 4;
    CK(cudaMemcpyAsync(f.d_desc, hd, dbytes, cudaMemcpyHostToDevice, f.s));
    f.h2d += dbytes;
    const SlotBlock *d_sb = (const SlotBlock *)(f.d_desc + o_sb);
    const int2 *d_w = (const int2 *)(f.d_desc + o_w);
    const int *d_pll = (const int *)(f.d_desc + o_pll);
    const int *d_aud_list = (const int *)(f.d_desc + o_aud);
    const GemmGroup *d_groups = (const GemmGroup *)(f.d_desc + o_ggr);
    const int *d_gmem = (const int *)(f.d_desc + o_gmem);
    const BankGroup *d_banks = (const BankGroup *)(f.d_desc + o_bgr);
    const int *d_bmem = (const int *)(f.d_desc + o_bmem);

    // output arena: results | PCM | RDS | audio (host part, then device part) | IQ (emitted part first)
    f.off_res = 0;
    f.off_pcm = align256(pl.sbs.size() * sizeof(DevResult));
    f.off_rds = f.off_pcm + align256((size_t)pl.tot_pcm * 2);
    f.off_audio = f.off_rds + align256((size_t)pl.tot_rds * 8);
    f.off_ext = f.off_audio + align256((size_t)pl.tot_audio * 4);
    DevResult *d_res = (DevResult *)(f.d_out + f.off_res);
    int16_t *d_pcm = (int16_t *)(f.d_out + f.off_pcm);
    float *d_audio = (float *)(f.d_out + f.off_audio);
    float2 *d_rds = (float2 *)(f.d_out + f.off_rds);
    float2 *d_ext = (float2 *)(f.d_out + f.off_ext);
    const int W = (int)f.wk_cap;
    const WfmTaps *wt = (const WfmTaps *)r->d_wtaps;
    int nl = 0;
    // ---- front half ----
    // With channel groups the dense classes (the groups' history tiles among
    // them) run on the frame's side stream beside the group kernel, whose
    // CTAs leave SMs free; the frame stream joins it before the first reader
    // of the extracted IQ.  Their stage times are then not recorded.
    const bool side = !pl.w_gemm.empty() && f.s2;
    cudaStream_t ds = side ? f.s2 : f.s;
    if (side) {
        CK(cudaEventRecord(f.ev_fork, f.s));
        CK(cudaStreamWaitEvent(f.s2, f.ev_fork, 0));
    }
    auto dense_name = [](int L) {
        return L < 10 ? std::string("extract_dense_L") + char('0' + L)
                      : std::string("extract_dense_L1") + char('0' + L - 10);
    };
    for (const DenseBatch &bt : batches) {
        // one tile per CTA; the smaller CTAs share SMs with the other blocks in flight
        if (!side) prof_mark(r, f, bt.classes > 1 ? "extract_dense" : dense_name(bt.L).c_str());
        if (bt.classes > 1)
            CK(launch_extract_dense_any((int)bt.items, bt.smem, ds, d_w + bt.off, d_sb, r->d_prm, r->d_st, x_dev, n,
                                        r->d_hist, r->d_taps, d_ext));
        else
            CK(launch_extract_dense(bt.L, (int)bt.items, bt.smem, ds, d_w + bt.off, d_sb, r->d_prm, r->d_st, x_dev,
                                    n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    for (int L = 0; L <= kDenseMaxL; ++L) {
        if (pl.w_dense[L].empty() || !dense_pipe[L]) continue;
        if (!side) prof_mark(r, f, dense_name(L).c_str());
        // persistent: one CTA per SM over contiguous runs of tiles
        CK(launch_extract_dense_pipe(L, dense_ng[L], (int)pl.w_dense[L].size(),
                                     std::min((int)pl.w_dense[L].size(), r->num_sms), pl.dense_pmax[L], ds,
                                     d_w + w_dense_off[L], d_sb, r->d_prm, r->d_st, x_dev, n, r->d_hist, r->d_taps,
                                     d_ext, r->d_fault));
        nl++;
    }
    if (!pl.w_gemm.empty()) {
        // the packed taps depend on the group layout and on each member's taps
        // and NCO increment: repack only when one of them changed since this
        // frame's buffer was packed
        std::vector<uint64_t> key;
        key.reserve(pl.groups.size() * 4 + pl.gmembers.size());
        for (const GemmGroup &g : pl.groups) {
            key.push_back(((uint64_t)(uint32_t)g.nmem << 32) | (uint32_t)g.ncol);
            key.push_back(((uint64_t)(uint32_t)g.D << 32) | (uint32_t)g.T);
            key.push_back((uint64_t)(uint32_t)g.b_off);
        }
        for (int row : pl.gmembers) {
            const int slot = pl.sbs[(size_t)row].slot;
            key.push_back(((uint64_t)(uint32_t)slot << 40) ^ r->slots[(size_t)slot].pver);
        }
        if (key != f.gb_key) {
            prof_mark(r, f, "gemm_pack");
            CK(launch_gemm_pack((int)pl.groups.size(), pl.gemm_max_l, f.s, d_groups, d_gmem, d_sb, r->d_prm,
                                r->d_taps, f.d_gb));
            f.gb_key = std::move(key);
            nl++;
        }
        prof_mark(r, f, "extract_gemm");
        CK(launch_extract_gemm((int)pl.w_gemm.size(), pl.gemm_smem, f.s, d_w + o_gemm, d_groups, d_gmem, d_sb,
                               r->d_prm, r->d_st, x_dev, n, f.d_gb, d_ext, r->d_fault));
        nl++;
    }
    if (!pl.w_bank.empty()) {
        // the packed modulated taps depend on the bank layout and on each
        // member's taps and NCO increment: repack only when one changed
        std::vector<uint64_t> key;
        key.reserve(pl.banks.size() * 3 + pl.bmembers.size());
        for (const BankGroup &b : pl.banks) {
            key.push_back(((uint64_t)(uint32_t)b.nmem << 32) | (uint32_t)b.cpad);
            key.push_back(((uint64_t)(uint32_t)b.T << 32) | (uint32_t)b.g_off);
        }
        for (int row : pl.bmembers) {
            const int slot = pl.sbs[(size_t)row].slot;
            key.push_back(((uint64_t)(uint32_t)slot << 40) ^ r->slots[(size_t)slot].pver);
        }
        if (key != f.bank_key) {
            prof_mark(r, f, "bank_pack");
            CK(launch_bank_pack((int)pl.banks.size(), pl.bank_max_total, f.s, d_banks, d_bmem, d_sb, r->d_prm,
                                r->d_taps, f.d_bank));
            f.bank_key = std::move(key);
            nl++;
        }
        prof_mark(r, f, "extract_bank");
        CK(launch_extract_bank((int)pl.w_bank.size(), f.s, d_w + o_bank, d_banks, d_bmem, d_sb, r->d_prm, r->d_st,
                               x_dev, f.d_bank, d_ext));
        nl++;
    }
    if (!pl.w_group.empty()) {
        prof_mark(r, f, "extract_group");
        CK(launch_extract_group((int)pl.w_group.size(), pl.group_smem, f.s, d_w + o_grp, d_sb, r->d_prm, r->d_st,
                                x_dev, n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    if (!pl.w_mod.empty()) {
        prof_mark(r, f, "extract_mod");
        CK(launch_extract_mod((int)pl.w_mod.size(), pl.mod_smem, f.s, d_w + o_mod, d_sb, r->d_prm, r->d_st, x_dev,
                              n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    if (!pl.w_wide.empty()) {
        prof_mark(r, f, "extract_wide");
        CK(launch_extract_wide((int)pl.w_wide.size(), pl.wide_smem, f.s, d_w + o_wide, d_sb, r->d_prm, r->d_st, x_dev,
                               n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    if (side) {
        prof_mark(r, f, "wait_side");  // ends the group kernel's interval; the join wait is its own
        CK(cudaEventRecord(f.ev_join, f.s2));
        CK(cudaStreamWaitEvent(f.s, f.ev_join, 0));
    }
    // the extraction state is carried at once, so the next block's extraction
    // overlaps this block's later front-half stages
    prof_mark(r, f, "post_extract");
    CK(launch_post_extract((int)pl.sbs.size(), f.s, d_sb, r->d_prm, r->d_st, x_dev, n, r->d_hist, d_res));
    nl++;
    CK(cudaEventRecord(f.ev_ext, f.s));
    if (f.ring >= 0) CK(cudaEventRecord(r->ring_free[f.ring], f.s));  // the input ring slot may be refilled
    // the later front-half stages carry state across blocks too (bridge
    // sample, decimator, composite and RDS delay lines): after the previous
    // block's front half
    if (prev) {
        prof_mark(r, f, "wait_prev_front");
        CK(cudaStreamWaitEvent(f.s, prev->ev_front, 0));
    }
    if (!pl.w_dec.empty()) {
        prof_mark(r, f, "decim2");
        CK(launch_decim2((int)pl.w_dec.size(), f.s, d_w + o_wdec, d_sb, r->d_prm, r->d_d1taps, r->d_d1hist, d_ext));
        nl++;
    }
    if (!pl.w_demod.empty()) {
        prof_mark(r, f, "demod");
        CK(launch_demod((int)pl.w_demod.size(), f.s, d_w + o_dem, d_sb, r->d_prm, r->d_st, d_ext, f.d_wk, d_audio));
        nl++;
    }
    if (!pl.w_am.empty()) {
        prof_mark(r, f, "am");
        CK(launch_am((int)pl.w_am.size(), f.s, d_w + o_am, d_sb, d_ext, d_audio));
        nl++;
    }
    if (!pl.w_fir.empty()) {
        prof_mark(r, f, "wfm_fir");
        CK(launch_wfm_fir((int)pl.w_fir.size(), f.s, d_w + o_fir, d_sb, r->d_prm, wt, f.d_wk, W, r->d_comp_dl));
        nl++;
    }
    if (!pl.w_rds.empty()) {
        prof_mark(r, f, "rds");
        CK(launch_rds((int)pl.w_rds.size(), pl.rds_smem, f.s, d_w + o_rds, d_sb, r->d_prm, r->d_st, wt, r->d_tabs,
                      f.d_wk, r->d_rds_dl, d_rds));
        nl++;
    }
    if (!pl.sbs.empty()) {
        prof_mark(r, f, "post_front");
        CK(launch_post_front((int)pl.sbs.size(), f.s, d_sb, r->d_prm, r->d_st, d_ext, f.d_wk, r->d_comp_dl,
                             r->d_rds_dl, r->d_tabs, r->d_d1hist, d_res));
        nl++;
    }
    CK(cudaEventRecord(f.ev_front, f.s));
    // ---- back half: after the previous block's back half ----
    if (prev) {
        prof_mark(r, f, "wait_prev_back");
        CK(cudaStreamWaitEvent(f.s, prev->ev_back, 0));
    }
    if (!pl.w_free.empty()) {
        prof_mark(r, f, "free_stereo");
        CK(launch_free_stereo((int)pl.w_free.size(), f.s, d_w + o_free, d_sb, r->d_prm, r->d_tabs + kMaxWfmClasses,
                              f.d_wk, W));
        nl++;
    }
    if (pl.batch_stereo) {
        prof_mark(r, f, "comp_power");
        CK(launch_comp_power((int)pl.pll_list.size(), f.s, d_pll, d_sb, r->d_prm, r->d_st, f.d_wk));
        nl++;
    }
    if (!pl.pll_list.empty()) {
        if (r->pll_parallel) {
            // cluster size: one thread per segment of the longest block
            int nch = (int)pl.pll_list.size();
            int max_n = 0;
            for (int i : pl.pll_list) max_n = std::max(max_n, pl.sbs[(size_t)i].n_disc);
            const int cluster = pll_cluster_for(max_n);
            prof_mark(r, f, "pll_newton");
            CK(launch_pll_newton(nch, cluster, f.s, d_pll, d_sb, r->d_prm, r->d_st, f.d_wk, W, r->pll_max_iters));
        } else {
            prof_mark(r, f, "pll_serial");
            CK(launch_pll((int)pl.pll_list.size(), f.s, d_pll, d_sb, r->d_prm, r->d_st, f.d_wk, W));
        }
        nl++;
    }
    if (!pl.w_out.empty()) {
        prof_mark(r, f, "wfm_out");
        CK(launch_wfm_out((int)pl.w_out.size(), f.s, d_w + o_out, d_sb, r->d_prm, r->d_st, wt, f.d_wk, W, r->d_lr_dl,
                          r->d_audio_dl, d_audio));
        nl++;
    }
    if (!pl.aud_list.empty()) {
        prof_mark(r, f, "audio48k");
        CK(launch_audio48((int)pl.w_aud.size(), (int)pl.aud_list.size(), f.s, d_w + o_waud, d_aud_list, d_sb,
                          r->d_prm, r->d_banks, r->d_aud, d_audio, f.d_rs, d_pcm));
        nl += pl.w_aud.empty() ? 1 : 2;
    }
    if (!pl.sbs.empty()) {
        prof_mark(r, f, "post_back");
        CK(launch_post_back((int)pl.sbs.size(), f.s, d_sb, r->d_prm, r->d_st, f.d_wk, W, r->d_lr_dl, r->d_audio_dl,
                            d_res));
        nl++;
    }
    CK(cudaEventRecord(f.ev_back, f.s));
    prof_mark(r, f, "d2h");
    r->launches += (uint64_t)nl;
    gpud_count_launch(nl);
    f.out_bytes = f.off_ext + (size_t)pl.tot_emit_ext * 8;
    f.host_outputs = r->host_outputs;
    if (f.host_outputs) {
        // results, PCM, RDS and the audio of channels without a 48 kHz back
        // end; then the IQ of channels that emit it
        const size_t head = f.off_audio + (size_t)pl.tot_audio_host * 4;
        CK(cudaMemcpyAsync(f.h_out, f.d_out, head, cudaMemcpyDeviceToHost, f.s));
        f.d2h += head;
        if (pl.tot_emit_ext > 0) {
            CK(cudaMemcpyAsync(f.h_out + f.off_ext, f.d_out + f.off_ext, (size_t)pl.tot_emit_ext * 8,
                               cudaMemcpyDeviceToHost, f.s));
            f.d2h += (size_t)pl.tot_emit_ext * 8;
        }
    } else {
        // the results table comes back; the payload stays on the device
        CK(cudaMemcpyAsync(f.h_out, f.d_out, f.off_pcm, cudaMemcpyDeviceToHost, f.s));
        f.d2h += f.off_pcm;
    }
    prof_mark(r, f, "end");
    return 0;
}

static int apply_pending(gpud_runner *r, Frame &f) {
    size_t off = 0;
    for (auto &op : r->pending) {
        std::memcpy(f.h_stage + off, op.data.data(), op.data.size());
        CK(cudaMemcpyAsync(op.dst, f.h_stage + off, op.data.size(), cudaMemcpyHostToDevice, f.s));
        f.h2d += op.data.size();
        off += align256(op.data.size());
    }
    r->pending.clear();
    return 0;
}

static void build_rows(gpud_runner *r, Frame &f) {
    f.row_of_slot.assign((size_t)r->max_ch, -1);
    for (size_t i = 0; i < f.plan.sbs.size(); ++i) f.row_of_slot[(size_t)f.plan.sbs[i].slot] = (int)i;
}

static bool host_pinned(const void *p) {
    cudaPointerAttributes at{};
    const bool pinned = cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return pinned;
}

static int submit_batched(gpud_runner *r, const gpud_float2 *iq, int n, int on_device) {
    // a block in pinned host memory starts its copy into the input ring now,
    // before this submit waits for a free frame
    int ring = -1;
    if (!on_device && n > 0 && iq && host_pinned(iq)) {
        ring = r->ring_next;
        r->ring_next = (ring + 1) % kInRing;
        CK(cudaStreamWaitEvent(r->in_s, r->ring_free[ring], 0));  // its previous block's readers are done
        CK(cudaEventRecord(r->ring_t0[ring], r->in_s));
        CK(cudaMemcpyAsync(r->d_ring[ring], iq, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice, r->in_s));
        CK(cudaEventRecord(r->ring_copied[ring], r->in_s));
    }
    const int fi = r->nxt;
    Frame &f = r->fr[fi];
    if (f.inflight) {
        int rc = finish_frame(r, fi, -1);
        if (rc) return rc;
    }
    if (r->done_frame == fi) r->done_frame = -1;  // its results are about to be overwritten
    Frame *prev = (r->last >= 0 && r->fr[r->last].inflight) ? &r->fr[r->last] : nullptr;
    BlockPlan &pl = f.plan;
    pl.sbs.clear();
    pl.n = n;
    for (int i = 0; i < r->max_ch; ++i)
        if (r->slots[(size_t)i].active) plan_slot(r, pl, i, n);
    finish_plan(r, pl);
    int rc = ensure_frame(r, f, pl);
    if (rc) return rc;
    f.h2d = f.d2h = 0;
    f.prof_n = 0;
    CK(cudaEventRecord(f.ev0, f.s));
    prof_mark(r, f, "h2d");
    const float2 *x = nullptr;
    f.ring = ring;
    f.ev_start = ring >= 0 ? r->ring_t0[ring] : f.ev0;
    if (ring >= 0) {
        CK(cudaStreamWaitEvent(f.s, r->ring_copied[ring], 0));
        f.h2d += (uint64_t)n * sizeof(float2);
        x = r->d_ring[ring];
    } else {
        rc = stage_input(r, f, iq, n, on_device, &x);
        if (rc) return rc;
    }
    // parameter updates and the extraction wait for the previous block's
    // extraction state (the later stages wait inside enqueue_block)
    if (prev) {
        prof_mark(r, f, "wait_prev_ext");
        CK(cudaStreamWaitEvent(f.s, prev->ev_ext, 0));
    }
    rc = apply_pending(r, f);
    if (rc) return rc;
    if (!pl.sbs.empty()) {
        rc = enqueue_block(r, f, prev, pl, x, n);
        if (rc) return rc;
    } else {
        // no channels: the chains of the block before pass through unchanged
        if (prev) {
            CK(cudaStreamWaitEvent(f.s, prev->ev_front, 0));
            CK(cudaStreamWaitEvent(f.s, prev->ev_back, 0));
        }
        CK(cudaEventRecord(f.ev_ext, f.s));
        if (f.ring >= 0) CK(cudaEventRecord(r->ring_free[f.ring], f.s));
        CK(cudaEventRecord(f.ev_front, f.s));
        CK(cudaEventRecord(f.ev_back, f.s));
        f.off_res = f.off_audio = f.off_rds = f.off_ext = f.out_bytes = 0;
    }
    CK(cudaEventRecord(f.ev1, f.s));
    CK(cudaEventRecord(f.ev_done, f.s));
    CK(cudaStreamWaitEvent(r->stream, f.ev_done, 0));  // join stream tracks every block
    advance_mirrors(r, pl, n, &f.after);
    build_rows(r, f);
    f.inflight = true;
    f.ticket = ++r->submitted;
    r->last = fi;
    r->nxt = (fi + 1) % kFrames;
    r->blocks++;
    return 0;
}

// Plain per-signal schedule (mirrors executeStreamingGPUNativePrepared,
// streaming_gpu_native_prepare.go:25-106): each channel alone -- block H2D,
// its own descriptors and launches, D2H, synchronised -- before the next.
static int run_plain(gpud_runner *r, const gpud_float2 *iq, int n, int on_device) {
    int rc = drain(r);
    if (rc) return rc;
    Frame &f = r->fr[0];
    r->done_frame = -1;
    BlockPlan full;
    full.n = n;
    for (int i = 0; i < r->max_ch; ++i)
        if (r->slots[(size_t)i].active) plan_slot(r, full, i, n);
    finish_plan(r, full);
    rc = ensure_frame(r, f, full);
    if (rc) return rc;
    f.h2d = f.d2h = 0;
    f.prof_n = 0;
    f.ring = -1;  // the plain schedule copies the block per signal, not through the input ring
    f.ev_start = f.ev0;
    std::vector<char> gathered;
    // the batched arena layout: results | PCM | RDS | audio | IQ
    size_t res_b = align256(full.sbs.size() * sizeof(DevResult));
    size_t p_off = res_b, r_off = p_off + align256((size_t)full.tot_pcm * 2),
           a_off = r_off + align256((size_t)full.tot_rds * 8), e_off = a_off + align256((size_t)full.tot_audio * 4);
    gathered.assign(e_off + align256((size_t)full.tot_ext * 8), 0);
    CK(cudaEventRecord(f.ev0, f.s));
    rc = apply_pending(r, f);
    if (rc) return rc;
    std::vector<SlotAfter> after;
    for (size_t k = 0; k < full.sbs.size(); ++k) {
        BlockPlan one;
        one.n = n;
        int slot = full.sbs[k].slot;
        Slot &s = r->slots[(size_t)slot];
        plan_slot(r, one, slot, n);
        finish_plan(r, one);
        // a channel alone can need buffers the whole set does not (it takes
        // no bank, so e.g. its phase-group partial sums): size the frame for
        // this plan too (the previous channel's work has completed)
        rc = ensure_frame(r, f, one);
        if (rc) return rc;
        const float2 *x = nullptr;
        rc = stage_input(r, f, iq, n, on_device, &x);  // the reference copies the whole block per signal
        if (rc) return rc;
        rc = enqueue_block(r, f, nullptr, one, x, n);
        if (rc) return rc;
        CK(cudaStreamSynchronize(f.s));
        const SlotBlock &o = one.sbs[0];
        const SlotBlock &fb = full.sbs[k];
        std::memcpy(gathered.data() + k * sizeof(DevResult), f.h_out + f.off_res, sizeof(DevResult));
        if (!(s.spec.flags & GPUD_CH_AUDIO48K))
            std::memcpy(gathered.data() + a_off + (size_t)fb.audio_off * 4,
                        f.h_out + f.off_audio + (size_t)o.audio_off * 4, (size_t)o.n_audio * 4);
        std::memcpy(gathered.data() + p_off + (size_t)fb.pcm_off * 2, f.h_out + f.off_pcm + (size_t)o.pcm_off * 2,
                    (size_t)o.rs_nout * (size_t)s.aud_ch * ((s.spec.flags & GPUD_CH_PCM_F32) ? 4 : 2));
        std::memcpy(gathered.data() + r_off + (size_t)fb.rds_off * 8, f.h_out + f.off_rds + (size_t)o.rds_off * 8,
                    (size_t)o.n_rds * 8);
        if (s.spec.flags & GPUD_CH_EMIT_IQ)
            std::memcpy(gathered.data() + e_off + (size_t)fb.ext_off * 8, f.h_out + f.off_ext + (size_t)o.ext_off * 8,
                        (size_t)o.n_out * 8);
        std::vector<SlotAfter> a1;
        advance_mirrors(r, one, n, &a1);
        after.push_back(a1[0]);
    }
    if (gathered.size() > f.out_cap) return set_err(r, GPUD_E_CUDA, "plain gather overflow");
    std::memcpy(f.h_out, gathered.data(), gathered.size());
    f.off_res = 0;
    f.off_pcm = p_off;
    f.off_audio = a_off;
    f.off_rds = r_off;
    f.off_ext = e_off;
    f.host_outputs = true;
    f.plan = full;
    f.after = after;
    build_rows(r, f);
    CK(cudaEventRecord(f.ev1, f.s));
    CK(cudaEventRecord(f.ev_done, f.s));
    f.inflight = true;
    f.ticket = ++r->submitted;
    r->last = 0;
    r->nxt = 1;
    r->blocks++;
    return finish_frame(r, 0, -1);
}

static int run_block(gpud_runner *r, const gpud_float2 *iq, int n, int on_device, bool wait, uint64_t *ticket) {
    if (n < 0 || n > r->max_block) return set_err(r, GPUD_E_BLOCK, "block larger than max_block");
    int rc;
    if (r->schedule == GPUD_SCHED_PLAIN) {
        rc = run_plain(r, iq, n, on_device);
    } else {
        rc = submit_batched(r, iq, n, on_device);
        if (!rc && wait) rc = drain(r);  // oldest first: the results are this block's
    }
    if (ticket) *ticket = r->submitted;
    return rc;
}

extern "C" {

GPUD_API int GPUD_CALL gpud_runner_create(int sample_rate, int max_block, int max_channels, int max_taps,
                                          uint64_t device_mem_budget, gpud_runner **out) {
    if (!out || sample_rate <= 0 || max_block <= 0 || max_channels <= 0 || max_channels > 4096 || max_taps <= 0 ||
        max_taps > 4096)
        return GPUD_E_ARG;
    auto *r = new gpud_runner();
    r->fs = sample_rate;
    r->max_block = max_block;
    r->max_ch = max_channels;
    r->max_taps = max_taps;
    r->budget = device_mem_budget;
    r->tapcap = 2 * max_taps + 64;
    r->slots.resize((size_t)max_channels);
    r->lat_ms.assign(4096, 0.f);
#define CKC(call)                    \
    do {                             \
        if ((call) != cudaSuccess) { \
            gpud_runner_destroy(r);  \
            return GPUD_E_CUDA;      \
        }                            \
    } while (0)
    CKC(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    CKC(cudaStreamCreateWithFlags(&r->admin, cudaStreamNonBlocking));
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
            r->num_sms = sms;
    }
    CKC(cudaHostAlloc((void **)&r->h_fault, 64, cudaHostAllocMapped));
    *(volatile unsigned *)r->h_fault = 0;
    CKC(cudaHostGetDevicePointer((void **)&r->d_fault, r->h_fault, 0));
    for (auto &f : r->fr) {
        CKC(cudaStreamCreateWithFlags(&f.s, cudaStreamNonBlocking));
        CKC(cudaEventCreateWithFlags(&f.ev_front, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&f.ev_ext, cudaEventDisableTiming));
        CKC(cudaStreamCreateWithFlags(&f.s2, cudaStreamNonBlocking));
        CKC(cudaEventCreateWithFlags(&f.ev_fork, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&f.ev_join, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&f.ev_back, cudaEventDisableTiming));
        CKC(cudaEventCreateWithFlags(&f.ev_done, cudaEventDisableTiming));
        CKC(cudaEventCreate(&f.ev0));
        CKC(cudaEventCreate(&f.ev1));
        CKC(dalloc(&f.d_block, (size_t)max_block));
        CKC(cudaMallocHost((void **)&f.h_in, (size_t)max_block * sizeof(float2)));
    }
    CKC(cudaStreamCreateWithFlags(&r->in_s, cudaStreamNonBlocking));
    for (int i = 0; i < kInRing; ++i) {
        CKC(dalloc(&r->d_ring[i], (size_t)max_block));
        CKC(cudaEventCreate(&r->ring_t0[i]));
        CKC(cudaEventCreate(&r->ring_copied[i]));
        CKC(cudaEventCreateWithFlags(&r->ring_free[i], cudaEventDisableTiming));
    }
    size_t M = (size_t)max_channels;
    CKC(dalloc(&r->d_prm, M));
    CKC(dalloc(&r->d_st, M));
    CKC(dalloc(&r->d_taps, M * 2 * (size_t)r->tapcap));
    CKC(dalloc(&r->d_hist, M * 2 * (size_t)max_taps));
    CKC(dalloc(&r->d_comp_dl, M * kWfmHist));
    CKC(dalloc(&r->d_lr_dl, M * kWfmHist));
    CKC(dalloc(&r->d_audio_dl, M * kAudioDlStrideH));
    CKC(dalloc(&r->d_rds_dl, M * kWfmHist));
    CKC(dalloc(&r->d_wtaps, (size_t)kMaxWfmClasses));
    CKC(dalloc(&r->d_tabs, (size_t)kMaxWfmClasses * 2));  // RDS 57 kHz tables, then 38 kHz tables
    CKC(dalloc(&r->d_aud, M));
    CKC(dalloc(&r->d_d1taps, M * kD1Taps));
    CKC(dalloc(&r->d_d1hist, M * kWfmHist));
    CKC(dalloc(&r->d_banks, (size_t)kMaxRsClasses));
#undef CKC
    r->used = slot_state_bytes(r) * M + (uint64_t)max_block * 8 * (kFrames + kInRing) + sizeof(RsBank) * kMaxRsClasses;
    *out = r;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_destroy(gpud_runner *r) {
    if (!r) return 0;
    for (auto &f : r->fr) {
        if (f.s) cudaStreamSynchronize(f.s);
    }
    if (r->stream) cudaStreamSynchronize(r->stream);
    if (r->admin) cudaStreamSynchronize(r->admin);
    if (r->in_s) {
        cudaStreamSynchronize(r->in_s);
        cudaStreamDestroy(r->in_s);
    }
    for (int i = 0; i < kInRing; ++i) {
        cudaFree(r->d_ring[i]);
        for (auto e : {r->ring_t0[i], r->ring_copied[i], r->ring_free[i]})
            if (e) cudaEventDestroy(e);
    }
    for (auto &f : r->fr) {
        cudaFree(f.d_desc);
        cudaFree(f.d_out);
        cudaFree(f.d_wk);
        cudaFree(f.d_block);
        cudaFree(f.d_rs);
        cudaFree(f.d_gb);
        cudaFree(f.d_bank);
        if (f.h_desc) cudaFreeHost(f.h_desc);
        if (f.h_out) cudaFreeHost(f.h_out);
        if (f.h_stage) cudaFreeHost(f.h_stage);
        if (f.h_in) cudaFreeHost(f.h_in);
        for (auto e : {f.ev_front, f.ev_ext, f.ev_back, f.ev_done, f.ev0, f.ev1, f.ev_fork, f.ev_join})
            if (e) cudaEventDestroy(e);
        for (auto e : f.prof_ev) cudaEventDestroy(e);
        if (f.s2) {
            cudaStreamSynchronize(f.s2);
            cudaStreamDestroy(f.s2);
        }
        if (f.s) cudaStreamDestroy(f.s);
    }
    if (r->h_fault) cudaFreeHost(r->h_fault);
    cudaFree(r->d_prm);
    cudaFree(r->d_st);
    cudaFree(r->d_taps);
    cudaFree(r->d_hist);
    cudaFree(r->d_comp_dl);
    cudaFree(r->d_lr_dl);
    cudaFree(r->d_audio_dl);
    cudaFree(r->d_rds_dl);
    cudaFree(r->d_wtaps);
    cudaFree(r->d_tabs);
    cudaFree(r->d_aud);
    cudaFree(r->d_d1taps);
    cudaFree(r->d_d1hist);
    cudaFree(r->d_banks);
    for (double *a : r->rs_arms) cudaFree(a);
    if (r->stream) cudaStreamDestroy(r->stream);
    if (r->admin) cudaStreamDestroy(r->admin);
    delete r;
    return 0;
}

GPUD_API const char *GPUD_CALL gpud_runner_last_error(gpud_runner *r) { return r ? r->err.c_str() : "null runner"; }

GPUD_API int GPUD_CALL gpud_runner_stream(gpud_runner *r, gpud_stream_handle *out) {
    if (!r || !out) return GPUD_E_ARG;
    *out = (gpud_stream_handle)r->stream;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_schedule(gpud_runner *r, int schedule) {
    if (!r || (schedule != GPUD_SCHED_BATCHED && schedule != GPUD_SCHED_PLAIN)) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    int rc = drain(r);
    if (rc) return rc;
    r->schedule = schedule;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_channel_footprint(gpud_runner *r, const gpud_channel_spec *spec, uint64_t *bytes) {
    if (!r || !bytes) return GPUD_E_ARG;
    int D, T;
    int rc = validate_spec(r, spec, &D, &T);
    if (rc) return rc;
    *bytes = slot_block_bytes(r, D, spec->mode, spec->flags);
    return 0;
}

// Extraction form of a channel: arms of at most 4 taps in the modulated-taps
// form (phase groups of raw samples); else the dense kernel when all D phases
// of a 256-output tile fit in shared memory (L <= 16); else phase groups of
// at most pg phases each (large D, long arms); else the wide kernel.
// Largest group of phases within a shared-memory budget (0: none).
static int largest_group(const Slot &s, bool mod, int budget) {
    int pmax = 0;
    for (int lo = 1, hi = s.P; lo <= hi;) {
        int mid = (lo + hi) / 2;
        if ((mod ? mod_smem_bytes_host(mid, s.L) : group_smem_bytes_host(mid, s.L)) <= budget) {
            pmax = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    return pmax;
}

constexpr int kFormSmemCap = 220 * 1024;  // the dynamic shared memory the grouped kernels opt in to

// Whether an autotune entry's form can run a channel of this geometry.
static bool form_valid(int T, int D, int form, int pg) {
    Slot s;
    s.T = T;
    s.D = D;
    s.P = std::min(D, T);
    s.L = (T + D - 1) / D;
    switch (form) {
    case GPUD_FORM_DENSE: return s.L >= 2 && s.L <= kDenseMaxL && dense_smem_bytes_host(s.P, s.L) <= kDenseSmemLimit;
    case GPUD_FORM_WIDE: return wide_smem_bytes_host(T) <= 64 * 1024;
    case GPUD_FORM_GROUP:
        return pg > 0 ? pg <= s.P && group_smem_bytes_host(pg, s.L) <= kFormSmemCap
                      : largest_group(s, false, kGroupSmemTarget) > 0;
    case GPUD_FORM_MOD:
        if (s.L > kModMaxL) return false;
        return pg > 0 ? pg <= s.P && mod_smem_bytes_host(pg, s.L) <= kFormSmemCap
                      : largest_group(s, true, kModSmemTarget) > 0;
    default: return false;
    }
}

static void choose_extraction(gpud_runner *r, Slot &s) {
    s.ng = 1;
    s.pg = s.P;
    for (const auto &e : r->tune) {
        if (e.taps != s.T || e.decim != s.D) continue;
        if (e.form == GPUD_FORM_DENSE || e.form == GPUD_FORM_WIDE) {
            s.ext_kind = e.form == GPUD_FORM_DENSE ? 0 : 1;
            return;
        }
        const bool m = e.form == GPUD_FORM_MOD;
        int pg = e.group_phases > 0 ? e.group_phases : largest_group(s, m, m ? kModSmemTarget : kGroupSmemTarget);
        s.ext_kind = m ? 3 : 2;
        s.ng = (s.P + pg - 1) / pg;
        s.pg = (s.P + s.ng - 1) / s.ng;
        return;
    }
    const bool mod = s.L <= kModMaxL;
    if (!mod && s.L <= kDenseMaxL && dense_smem_bytes_host(s.P, s.L) <= kDenseSmemLimit) {
        s.ext_kind = 0;
        return;
    }
    const int pmax = largest_group(s, mod, mod ? kModSmemTarget : kGroupSmemTarget);
    if (pmax == 0) {
        s.ext_kind = 1;
        return;
    }
    s.ext_kind = mod ? 3 : 2;
    s.ng = (s.P + pmax - 1) / pmax;
    s.pg = (s.P + s.ng - 1) / s.ng;
    // The staging puts a group's phases on lanes (one pass per 32) and its
    // rows on the 8 warps: groups of at most a multiple of 32 phases can keep
    // the lanes full (100 phases as 4 x 25 rather than 3 x 34, whose second
    // lane pass holds 2 of 32) at the price of more groups; take that split
    // when the instructions per thread it needs are fewer.
    if (pmax >= 64 || (pmax >= 32 && pmax % 32 != 0)) {
        const int q = pmax / 32 * 32;
        const int ng = (s.P + q - 1) / q, pg = (s.P + ng - 1) / ng;
        const int Le = mod ? s.L : ((s.L > 16) ? (s.L + 7) & ~7 : s.L);
        const int cols = 256 + Le - 1;
        auto cost = [&](int groups, int phases) {
            const int lane_passes = (phases + 31) / 32, row_rounds = (phases + 7) / 8;
            const int row = 8 + 2 * Le - 1 + (mod ? 4 : 2) * 8 * Le;  // window + taps loads, FMAs of 8 outputs
            return (int64_t)groups * (lane_passes * 14 * cols / 8 + row_rounds * row + 100);
        };
        if (cost(ng, pg) < cost(s.ng, s.pg)) {
            s.ng = ng;
            s.pg = pg;
        }
    }
}

static int admit_core(gpud_runner *r, const gpud_channel_spec *spec, int D, int T, double deemph_us,
                      int *slot_out);

GPUD_API int GPUD_CALL gpud_runner_admit(gpud_runner *r, const gpud_channel_spec *spec, int *slot_out) {
    if (!r || !slot_out) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    int D, T;
    int rc = validate_spec(r, spec, &D, &T);
    if (rc) return rc;
    return admit_core(r, spec, D, T, -1.0, slot_out);
}

// Admission after validation: decimation D and tap count T given (the batch
// entry point passes a rounded decimation the exact-rate rule would refuse).
static int admit_core(gpud_runner *r, const gpud_channel_spec *spec, int D, int T, double deemph_us,
                      int *slot_out) {
    int rc = 0;
    uint64_t fp = slot_block_bytes(r, D, spec->mode, spec->flags);
    if (r->budget && r->used + fp > r->budget) return set_err(r, GPUD_E_BUDGET, "device-memory budget exhausted");
    // a free slot no block in flight still touches; drain if only such slots are left
    int slot = -1;
    bool busy_free = false;
    for (int i = 0; i < r->max_ch; ++i) {
        const Slot &s = r->slots[(size_t)i];
        if (s.active) continue;
        if (s.reusable_after <= r->completed) {
            slot = i;
            break;
        }
        busy_free = true;
    }
    if (slot < 0 && busy_free) {
        rc = drain(r);
        if (rc) return rc;
        for (int i = 0; i < r->max_ch && slot < 0; ++i)
            if (!r->slots[(size_t)i].active) slot = i;
    }
    if (slot < 0) return set_err(r, GPUD_E_SLOTS, "channel cap reached");
    bool wfm = spec->mode == GPUD_MODE_WFM || spec->mode == GPUD_MODE_WFM_STEREO;
    int rclass = -1;
    int d1 = std::max(1, spec->demod_decim);
    int drate = spec->out_rate / d1;  // actualDemodRate (streamer.go:1113)
    if (wfm) {
        rclass = rate_class_for(r, drate);
        if (rclass < 0) return set_err(r, GPUD_E_CUDA, "WFM rate classes exhausted");
    }
    int rsclass = -1;
    if ((spec->flags & GPUD_CH_AUDIO48K) && spec->mode != GPUD_MODE_IQ) {
        rsclass = rs_class_for(r, drate);
        if (rsclass < 0) return set_err(r, GPUD_E_ARG, "no 48 kHz resampler for this output rate");
    }
    drop_pending(r, slot);
    Slot &s = r->slots[(size_t)slot];
    s = Slot{};
    s.spec = *spec;
    s.spec.num_taps = T;
    s.D = D;
    s.T = T;
    s.P = std::min(D, T);
    s.L = (T + D - 1) / D;
    s.hcap = r->max_taps;
    s.taps_off = slot * 2 * r->tapcap;
    s.dtaps_off = s.taps_off + r->tapcap;
    s.hist_off = slot * 2 * r->max_taps;
    s.wfm_idx = wfm ? slot : -1;
    s.rate_class = rclass;
    s.rs_class = rsclass;
    s.aud_ch = spec->mode == GPUD_MODE_WFM_STEREO ? 2 : 1;
    s.deemph_us = deemph_us;
    s.pver = ++r->pver_seq;
    s.d1 = d1;
    s.d1_phase = 0;
    if (rsclass >= 0) {
        s.rs_L = r->rs_lmk[(size_t)rsclass].x;
        s.rs_M = r->rs_lmk[(size_t)rsclass].y;
    }
    choose_extraction(r, s);
    s.footprint = fp;
    // The slot's memory is unused by every block in flight: write it now.
    std::vector<float> pm, h;
    design_taps(r, s, spec->bandwidth, pm, h, &s.cutoff);
    ChanParams p;
    fill_params(r, slot, &p);
    ChanState st{};
    st.pll_freq = 2 * GPUD_PI * 19000 / (double)demod_rate(s);  // stereoDecodeStateful init (streamer.go:1546-1555)
    CK(cudaMemcpyAsync(r->d_taps + s.taps_off, pm.data(), pm.size() * 4, cudaMemcpyHostToDevice, r->admin));
    CK(cudaMemcpyAsync(r->d_taps + s.dtaps_off, h.data(), h.size() * 4, cudaMemcpyHostToDevice, r->admin));
    CK(cudaMemcpyAsync(r->d_prm + slot, &p, sizeof p, cudaMemcpyHostToDevice, r->admin));
    CK(cudaMemcpyAsync(r->d_st + slot, &st, sizeof st, cudaMemcpyHostToDevice, r->admin));
    CK(cudaMemsetAsync(r->d_aud + slot, 0, sizeof(AudState), r->admin));
    if (d1 > 1) {
        // streamer.go:1117-1124: 101 taps of LowpassFIR(cutoff, snip rate),
        // 90 kHz for WFM, else 0.8 x the demod Nyquist
        double cut = wfm ? 90000.0 : (double)drate / 2.0 * 0.8;
        auto h1 = lowpass_fir(cut, spec->out_rate, kD1Taps);
        h1.resize(kD1Taps, 0.0);
        CK(cudaMemcpyAsync(r->d_d1taps + (size_t)slot * kD1Taps, h1.data(), kD1Taps * 8, cudaMemcpyHostToDevice,
                           r->admin));
        CK(cudaMemsetAsync(r->d_d1hist + (size_t)slot * kWfmHist, 0, kWfmHist * sizeof(float2), r->admin));
    }
    if (s.wfm_idx >= 0) {
        CK(cudaMemsetAsync(r->d_comp_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 4, r->admin));
        CK(cudaMemsetAsync(r->d_lr_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 4, r->admin));
        CK(cudaMemsetAsync(r->d_audio_dl + (size_t)s.wfm_idx * kAudioDlStrideH, 0, kAudioDlStrideH * 4, r->admin));
        CK(cudaMemsetAsync(r->d_rds_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 8, r->admin));
    }
    // complete before the next submit, which is the first block to read them
    CK(cudaStreamSynchronize(r->admin));
    s.active = true;
    r->used += fp;
    *slot_out = slot;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_retire(gpud_runner *r, int slot) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    r->used -= s.footprint;
    s.active = false;
    s.reusable_after = r->submitted;
    drop_pending(r, slot);
    for (auto it = r->by_signal.begin(); it != r->by_signal.end(); ++it)
        if (it->second == slot) {
            r->by_signal.erase(it);
            break;
        }
    return 0;
}

// The new taps / parameters are written on the next block's stream once the
// block before it has carried its extraction state.  That block's later
// stages may still be reading ChanParams; of what an update changes (NCO
// increment, taps, the float64-sum flag) only the extraction reads anything.
GPUD_API int GPUD_CALL gpud_runner_update(gpud_runner *r, int slot, double offset_hz, double bandwidth) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    double cutoff = bandwidth / 2;
    if (cutoff < 200) cutoff = 200;
    if (cutoff != s.cutoff) {
        s.pver = ++r->pver_seq;
        std::vector<float> pm, h;
        design_taps(r, s, bandwidth, pm, h, &s.cutoff);
        queue_write(r, slot, r->d_taps + s.taps_off, pm.data(), pm.size() * 4);
        queue_write(r, slot, r->d_taps + s.dtaps_off, h.data(), h.size() * 4);
    }
    bool was_precise = precise_sum(s.spec);
    s.spec.bandwidth = bandwidth;
    if (offset_hz != s.spec.offset_hz || precise_sum(s.spec) != was_precise) {
        s.pver = ++r->pver_seq;
        s.spec.offset_hz = offset_hz;
        ChanParams p;
        fill_params(r, slot, &p);
        queue_write(r, slot, r->d_prm + slot, &p, sizeof p);
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_process_block(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    return run_block(r, iq, n, iq_on_device, true, nullptr);
}

GPUD_API int GPUD_CALL gpud_runner_submit(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device,
                                          uint64_t *ticket) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    return run_block(r, iq, n, iq_on_device, false, ticket);
}

GPUD_API int GPUD_CALL gpud_runner_wait(gpud_runner *r, uint64_t ticket, int timeout_ms) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    // finish blocks in order until `ticket` has completed
    while (r->completed < ticket) {
        const int a = oldest_inflight(r);
        if (a < 0) break;
        int rc = finish_frame(r, a, timeout_ms < 0 ? -1 : timeout_ms);
        if (rc) return rc;
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_host_outputs(gpud_runner *r, int on) {
    if (!r) return GPUD_E_ARG;
    r->host_outputs = on != 0;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_pll_solver(gpud_runner *r, int parallel) {
    if (!r || parallel < 0) return GPUD_E_ARG;
    r->pll_parallel = parallel != 0;
    r->pll_max_iters = parallel > 1 ? std::min(parallel, 4096) : kPllMaxIters;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_profiling(gpud_runner *r, int on) {
    if (!r) return GPUD_E_ARG;
    r->profiling = on != 0;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_stage_times(gpud_runner *r, gpud_stage_time *out, int cap, int *count) {
    if (!r || !count) return GPUD_E_ARG;
    int n = (int)r->stage_times.size();
    *count = n;
    for (int i = 0; i < n && i < cap && out; ++i) out[i] = r->stage_times[(size_t)i];
    return 0;
}

// Results of the most recently completed block (gpud_runner_wait /
// gpud_runner_process_block) that included the slot.
GPUD_API int GPUD_CALL gpud_runner_result(gpud_runner *r, int slot, gpud_channel_result *out) {
    if (!r || !out) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    std::memset(out, 0, sizeof *out);
    out->signal_id = s.spec.signal_id;
    out->rate = s.spec.out_rate;
    out->audio_channels = s.spec.mode == GPUD_MODE_WFM_STEREO ? 2 : (s.spec.mode == GPUD_MODE_IQ ? 0 : 1);
    out->rds_rate = demod_rate(s) / std::max(1, demod_rate(s) / 19000);
    out->phase_count = s.pc;
    out->history_len = s.hist_len;
    if (r->done_frame < 0) {
        if (oldest_inflight(r) >= 0) return set_err(r, GPUD_E_TIMEOUT, "block still in flight");
        return 0;
    }
    Frame &f = r->fr[r->done_frame];
    if (f.row_of_slot.size() != (size_t)r->max_ch) return 0;
    int row = f.row_of_slot[(size_t)slot];
    if (row < 0) return 0;  // admitted after that block
    const SlotBlock &sb = f.plan.sbs[(size_t)row];
    const DevResult *res = (const DevResult *)(f.h_out + f.off_res) + row;
    out->n_iq = sb.n_out;
    out->phase_count = f.after[(size_t)row].pc;
    out->history_len = f.after[(size_t)row].hist_len;
    out->nco_phase = res->nco_phase;
    out->n_audio = sb.n_audio;
    out->n_rds = sb.n_rds;
    out->flags = res->flags;
    out->coherence = res->coherence;
    out->pilot_hz = res->pilot_hz;
    out->err_avg = res->err_avg;
    out->pll_path = res->status;
    out->pll_iters = res->pll_iters;
    const char *base = f.host_outputs ? f.h_out : f.d_out;
    const bool a48 = (s.spec.flags & GPUD_CH_AUDIO48K) != 0 && s.rs_class >= 0;
    out->audio = (a48 && f.host_outputs) ? nullptr : (const float *)(base + f.off_audio) + sb.audio_off;
    if (a48) {
        const int16_t *p = (const int16_t *)(base + f.off_pcm) + sb.pcm_off;
        if (s.spec.flags & GPUD_CH_PCM_F32)
            out->pcm_f32 = reinterpret_cast<const float *>(p);
        else
            out->pcm = p;
        out->n_pcm = sb.rs_nout * s.aud_ch;
        out->pcm_rate = 48000;
    }
    out->rds = (const gpud_float2 *)(base + f.off_rds) + sb.rds_off;
    out->iq = (s.spec.flags & GPUD_CH_EMIT_IQ) ? (const gpud_float2 *)(base + f.off_ext) + sb.ext_off : nullptr;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_stats_get(gpud_runner *r, gpud_runner_stats *out) {
    if (!r || !out) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    std::memset(out, 0, sizeof *out);
    out->blocks = r->blocks;
    int act = 0;
    for (auto &s : r->slots) act += s.active ? 1 : 0;
    out->active_channels = act;
    out->max_channels = r->max_ch;
    out->device_bytes_used = r->used;
    out->device_bytes_budget = r->budget;
    out->last_block_ms = r->last_ms;
    size_t cnt = std::min(r->lat_pos, r->lat_ms.size());
    if (cnt) {
        std::vector<float> v(r->lat_ms.begin(), r->lat_ms.begin() + (long)cnt);
        std::sort(v.begin(), v.end());
        out->p50_block_ms = v[(size_t)((cnt - 1) * 0.50)];
        out->p99_block_ms = v[(size_t)((cnt - 1) * 0.99)];
    }
    out->kernel_launches = r->launches;
    out->graph_rebuilds = r->graph_rebuilds;
    out->ring_copy_ms = r->ring_ms;
    out->ring_copies = r->ring_copies;
    if (r->done_frame >= 0) {
        out->last_h2d_bytes = r->fr[r->done_frame].h2d;
        out->last_d2h_bytes = r->fr[r->done_frame].d2h;
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_reset_stats(gpud_runner *r) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    r->lat_pos = 0;
    r->ring_ms = 0;
    r->ring_copies = 0;
    return 0;
}

// ---------------------------------------------------------------------------
// snapshot / restore
// ---------------------------------------------------------------------------
struct SnapHeader {
    uint32_t magic, version;
    int32_t D, T, mode, wfm;
    int32_t pc, hist_len, hist_sel, comp_hist_len, has_last, pad;
    int64_t rds_count;
    double cutoff;
    int64_t rs_t;  // 48 kHz resampler phase counter
    int32_t d1, d1_phase;  // pre-demod decimation and its phase counter
};

static uint64_t snap_bytes(const Slot &s) {
    uint64_t b = sizeof(SnapHeader) + sizeof(ChanState) + (uint64_t)s.hcap * 8 + sizeof(AudState);
    if (s.wfm_idx >= 0) b += kWfmHist * 4 * 2 + kAudioDlStrideH * 4 + kWfmHist * 8;
    if (s.d1 > 1) b += kWfmHist * 8;
    return b;
}

GPUD_API int GPUD_CALL gpud_runner_snapshot(gpud_runner *r, int slot, void *blob, uint64_t *bytes) {
    if (!r || !bytes) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    uint64_t need = snap_bytes(s);
    if (!blob) {
        *bytes = need;
        return 0;
    }
    if (*bytes < need) return set_err(r, GPUD_E_ARG, "snapshot buffer too small");
    int rc = drain(r);
    if (rc) return rc;
    char *p = (char *)blob;
    SnapHeader h{0x47505544u, 3, s.D, s.T, s.spec.mode, s.wfm_idx >= 0, s.pc, s.hist_len, s.hist_sel,
                 s.comp_hist_len, s.has_last ? 1 : 0, 0, s.rds_count, s.cutoff, s.rs_t, s.d1, s.d1_phase};
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    CK(cudaMemcpy(p, r->d_st + slot, sizeof(ChanState), cudaMemcpyDeviceToHost));
    p += sizeof(ChanState);
    CK(cudaMemcpy(p, r->d_hist + s.hist_off + (size_t)s.hist_sel * s.hcap, (size_t)s.hcap * 8,
                  cudaMemcpyDeviceToHost));
    p += (size_t)s.hcap * 8;
    CK(cudaMemcpy(p, r->d_aud + slot, sizeof(AudState), cudaMemcpyDeviceToHost));
    p += sizeof(AudState);
    if (s.wfm_idx >= 0) {
        size_t w = (size_t)s.wfm_idx;
        CK(cudaMemcpy(p, r->d_comp_dl + w * kWfmHist, kWfmHist * 4, cudaMemcpyDeviceToHost));
        p += kWfmHist * 4;
        CK(cudaMemcpy(p, r->d_lr_dl + w * kWfmHist, kWfmHist * 4, cudaMemcpyDeviceToHost));
        p += kWfmHist * 4;
        CK(cudaMemcpy(p, r->d_audio_dl + w * kAudioDlStrideH, kAudioDlStrideH * 4, cudaMemcpyDeviceToHost));
        p += kAudioDlStrideH * 4;
        CK(cudaMemcpy(p, r->d_rds_dl + w * kWfmHist, kWfmHist * 8, cudaMemcpyDeviceToHost));
        p += kWfmHist * 8;
    }
    if (s.d1 > 1) {
        CK(cudaMemcpy(p, r->d_d1hist + (size_t)slot * kWfmHist, kWfmHist * 8, cudaMemcpyDeviceToHost));
        p += kWfmHist * 8;
    }
    *bytes = need;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_restore(gpud_runner *r, int slot, const void *blob, uint64_t bytes) {
    if (!r || !blob) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    if (bytes < snap_bytes(s)) return set_err(r, GPUD_E_STATE, "snapshot size mismatch");
    const char *p = (const char *)blob;
    SnapHeader h;
    std::memcpy(&h, p, sizeof h);
    p += sizeof h;
    if (h.magic != 0x47505544u || h.version != 3 || h.D != s.D || h.T != s.T || h.mode != s.spec.mode ||
        h.wfm != (s.wfm_idx >= 0) || h.d1 != s.d1)
        return set_err(r, GPUD_E_STATE, "snapshot geometry mismatch");
    int rc = drain(r);
    if (rc) return rc;
    drop_pending(r, slot);  // the restored state replaces queued updates of this slot
    CK(cudaMemcpy(r->d_st + slot, p, sizeof(ChanState), cudaMemcpyHostToDevice));
    p += sizeof(ChanState);
    s.hist_sel = 0;
    CK(cudaMemcpy(r->d_hist + s.hist_off, p, (size_t)s.hcap * 8, cudaMemcpyHostToDevice));
    p += (size_t)s.hcap * 8;
    CK(cudaMemcpy(r->d_aud + slot, p, sizeof(AudState), cudaMemcpyHostToDevice));
    p += sizeof(AudState);
    if (s.wfm_idx >= 0) {
        size_t w = (size_t)s.wfm_idx;
        CK(cudaMemcpy(r->d_comp_dl + w * kWfmHist, p, kWfmHist * 4, cudaMemcpyHostToDevice));
        p += kWfmHist * 4;
        CK(cudaMemcpy(r->d_lr_dl + w * kWfmHist, p, kWfmHist * 4, cudaMemcpyHostToDevice));
        p += kWfmHist * 4;
        CK(cudaMemcpy(r->d_audio_dl + w * kAudioDlStrideH, p, kAudioDlStrideH * 4, cudaMemcpyHostToDevice));
        p += kAudioDlStrideH * 4;
        CK(cudaMemcpy(r->d_rds_dl + w * kWfmHist, p, kWfmHist * 8, cudaMemcpyHostToDevice));
        p += kWfmHist * 8;
    }
    if (s.d1 > 1) {
        CK(cudaMemcpy(r->d_d1hist + (size_t)slot * kWfmHist, p, kWfmHist * 8, cudaMemcpyHostToDevice));
        p += kWfmHist * 8;
    }
    s.d1_phase = h.d1_phase;
    s.pc = h.pc;
    s.hist_len = h.hist_len;
    s.comp_hist_len = h.comp_hist_len;
    s.has_last = h.has_last != 0;
    s.rds_count = h.rds_count;
    s.rs_t = h.rs_t;
    if (h.cutoff != s.cutoff) {
        s.pver = ++r->pver_seq;
        std::vector<float> pm, hh;
        design_taps(r, s, 2 * h.cutoff, pm, hh, &s.cutoff);
        CK(cudaMemcpy(r->d_taps + s.taps_off, pm.data(), pm.size() * 4, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(r->d_taps + s.dtaps_off, hh.data(), hh.size() * 4, cudaMemcpyHostToDevice));
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_reset_signal(gpud_runner *r, int64_t signal_id) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    auto it = r->by_signal.find(signal_id);
    if (it == r->by_signal.end()) return 0;
    return gpud_runner_retire(r, it->second);
}

GPUD_API int GPUD_CALL gpud_runner_reset_all_signals(gpud_runner *r) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    std::vector<int> slots;
    for (auto &kv : r->by_signal) slots.push_back(kv.second);
    for (int s : slots) gpud_runner_retire(r, s);
    r->by_signal.clear();
    return 0;
}

// ---------------------------------------------------------------------------
// BatchRunner.StreamingExtractGPU semantics
// ---------------------------------------------------------------------------
GPUD_API int GPUD_CALL gpud_runner_streaming_extract(gpud_runner *r, const gpud_float2 *iq, int n,
                                                     const gpud_channel_spec *jobs, int n_jobs,
                                                     gpud_channel_result *results, gpud_float2 *iq_out,
                                                     int iq_out_cap) {
    if (!r || n < 0 || n_jobs < 0 || (n_jobs > 0 && (!jobs || !results))) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    std::vector<int> job_slot((size_t)n_jobs, -1);
    std::map<int64_t, bool> active;
    for (int i = 0; i < n_jobs; ++i) {
        gpud_channel_spec spec = jobs[i];
        spec.mode = GPUD_MODE_IQ;
        spec.flags = GPUD_CH_EMIT_IQ;
        active[spec.signal_id] = true;
        int D, T;
        int rc = validate_spec(r, &spec, &D, &T);
        if (rc) return rc;
        auto it = r->by_signal.find(spec.signal_id);
        int slot = -1;
        if (it != r->by_signal.end()) {
            slot = it->second;
            Slot &s = r->slots[(size_t)slot];
            if (s.spec.config_hash != spec.config_hash || s.D != D || s.T != T) {
                // ResetExtractStreamState (streaming_types.go:48-56): geometry may change
                gpud_runner_retire(r, slot);
                slot = -1;
            } else {
                rc = gpud_runner_update(r, slot, spec.offset_hz, spec.bandwidth);
                if (rc) return rc;
            }
        }
        if (slot < 0) {
            int rc2 = gpud_runner_admit(r, &spec, &slot);
            if (rc2) return rc2;
            r->by_signal[spec.signal_id] = slot;
        }
        job_slot[(size_t)i] = slot;
    }
    // prune signals absent from this call (streaming_gpu_prepare.go:38-43)
    std::vector<int> to_retire;
    for (auto &kv : r->by_signal)
        if (!active.count(kv.first)) to_retire.push_back(kv.second);
    for (int s : to_retire) gpud_runner_retire(r, s);
    // channels admitted through the slot API are left untouched: only the jobs' slots run
    int rc = drain(r);
    if (rc) return rc;
    std::vector<int> parked;
    for (int i = 0; i < r->max_ch; ++i) {
        Slot &s = r->slots[(size_t)i];
        if (!s.active) continue;
        bool mine = std::find(job_slot.begin(), job_slot.end(), i) != job_slot.end();
        if (!mine) {
            s.active = false;
            parked.push_back(i);
        }
    }
    rc = run_block(r, iq, n, 0, true, nullptr);
    for (int i : parked) r->slots[(size_t)i].active = true;
    if (rc) return rc;
    int64_t pos = 0;
    for (int i = 0; i < n_jobs; ++i) {
        rc = gpud_runner_result(r, job_slot[(size_t)i], &results[i]);
        if (rc) return rc;
        gpud_channel_result &res = results[i];
        if (iq_out && res.n_iq > 0) {
            if (pos + res.n_iq > iq_out_cap) return set_err(r, GPUD_E_ARG, "iq_out capacity");
            std::memcpy(iq_out + pos, res.iq, (size_t)res.n_iq * sizeof(gpud_float2));
            res.iq = iq_out + pos;
            pos += res.n_iq;
        }
    }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Event-recording batch path (recorder/wfm_batch_stereo.go:10-72)
// ---------------------------------------------------------------------------
// One capture through a one-channel runner: the channel starts fresh (zero
// filter histories, pilot loop at 19 kHz, resampler and de-emphasis at rest),
// its NCO at the first increment (FreqShift pre-increments from phase 0), its
// decimation phase so that the first output is input 0 (Decimate keeps index
// 0), the 101-tap low-pass at max(bw/2, 200) raised to 75 kHz, decimation
// round(fs/192000), the batch stereo decoder and the 48 kHz back end in float.
GPUD_API int GPUD_CALL gpud_wfm_batch_audio(const gpud_float2 *iq, int n, int iq_on_device, int sample_rate,
                                            double offset_hz, double bandwidth, double deemph_us, float *out,
                                            int out_cap, gpud_batch_audio_result *res) {
    if (!iq || n <= 0 || sample_rate <= 0 || !out || out_cap < 0 || !res || deemph_us < 0) return GPUD_E_ARG;
    std::memset(res, 0, sizeof *res);
    int d1 = (int)std::llround((double)sample_rate / 192000.0);
    if (d1 < 1) d1 = 1;
    const int rate = sample_rate / d1;
    res->demod_rate = rate;
    if ((n + d1 - 1) / d1 < 2) return 0;  // fewer than two decimated samples: no audio
    gpud_runner *r = nullptr;
    int rc = gpud_runner_create(sample_rate, n, 1, 101, 0, &r);
    if (rc) return rc;
    gpud_channel_spec sp{};
    sp.signal_id = 1;
    sp.offset_hz = offset_hz;
    sp.bandwidth = 2.0 * std::max(bandwidth / 2.0, 75000.0);
    sp.out_rate = rate;
    sp.num_taps = 101;
    sp.mode = GPUD_MODE_WFM_STEREO;
    sp.flags = GPUD_CH_AUDIO48K | GPUD_CH_PCM_F32 | GPUD_CH_BATCH_STEREO;
    int slot = -1;
    {
        std::lock_guard<std::recursive_mutex> lk(r->mu);
        rc = admit_core(r, &sp, d1, 101, deemph_us, &slot);
        if (!rc && r->slots[(size_t)slot].rs_class < 0) rc = set_err(r, GPUD_E_ARG, "no 48 kHz resampler for the demod rate");
        if (!rc) {
            Slot &s = r->slots[(size_t)slot];
            s.pc = d1 - 1;
            ChanParams p;
            fill_params(r, slot, &p);
            const uint64_t u1 = p.inc_q;  // phase of input 0: one increment
            if (cudaMemcpy(&r->d_st[slot].nco_q, &u1, sizeof u1, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = set_err(r, GPUD_E_CUDA, "batch state");
        }
    }
    if (!rc) rc = gpud_runner_process_block(r, iq, n, iq_on_device);
    if (!rc) {
        gpud_channel_result cr;
        rc = gpud_runner_result(r, slot, &cr);
        if (!rc) {
            if (cr.n_pcm > out_cap) {
                rc = GPUD_E_ARG;
            } else {
                if (cr.n_pcm > 0) std::memcpy(out, cr.pcm_f32, (size_t)cr.n_pcm * sizeof(float));
                res->n_out = cr.n_pcm;
                res->out_rate = 48000;
                res->locked = (cr.flags & 1) ? 1 : 0;
            }
        }
    }
    gpud_runner_destroy(r);
    return rc;
}

// ---------------------------------------------------------------------------
// One-shot segment demod (recorder/cpu_audio.go:10-75, demodAudioCPU): the
// live /api/demod path and event recordings of the other modes
// ---------------------------------------------------------------------------
// A fresh one-channel runner as for the batch path (FreqShift pre-increment,
// Decimate from input 0, 101 taps at max(bw/2, 200), 75 kHz at least for the
// 192 kS/s WFM demodulators, decimation round(fs/demodRate)); WFM is the bare
// discriminator, WFM_STEREO the free-running stereo decoder.  Above 48 kHz the
// audio then takes the 63-tap anti-alias filter and every round(rate/48000)-th
// frame (stereo: whole frames only), on the device.
GPUD_API int GPUD_CALL gpud_demod_audio_segment(int mode, const gpud_float2 *iq, int n, int iq_on_device,
                                                int sample_rate, double offset_hz, double bandwidth, float *out,
                                                int out_cap, gpud_segment_audio_result *res) {
    if (!iq || n <= 0 || sample_rate <= 0 || !out || out_cap < 0 || !res) return GPUD_E_ARG;
    if (mode < GPUD_MODE_NFM || mode > GPUD_MODE_CW) return GPUD_E_MODE;
    std::memset(res, 0, sizeof *res);
    const bool wide = mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    const int C = mode == GPUD_MODE_WFM_STEREO ? 2 : 1;
    res->channels = C;
    const int drate = wide ? 192000 : 48000;
    double cutoff = std::max(bandwidth / 2.0, 200.0);
    if (cutoff < 75000.0 && drate >= 192000) cutoff = 75000.0;
    int d1 = (int)std::llround((double)sample_rate / (double)drate);
    if (d1 < 1) d1 = 1;
    const int rate = sample_rate / d1;
    res->demod_rate = rate;
    res->out_rate = rate;
    gpud_runner *r = nullptr;
    int rc = gpud_runner_create(sample_rate, n, 1, 101, 0, &r);
    if (rc) return rc;
    gpud_channel_spec sp{};
    sp.signal_id = 1;
    sp.offset_hz = offset_hz;
    sp.bandwidth = 2.0 * cutoff;
    sp.out_rate = rate;
    sp.num_taps = 101;
    sp.mode = mode == GPUD_MODE_WFM ? GPUD_MODE_NFM : mode;  // WFM.Demod is the bare discriminator
    sp.flags = mode == GPUD_MODE_WFM_STEREO ? GPUD_CH_FREE_STEREO : 0;
    int slot = -1;
    {
        std::lock_guard<std::recursive_mutex> lk(r->mu);
        rc = admit_core(r, &sp, d1, 101, -1.0, &slot);
        if (!rc) {
            r->slots[(size_t)slot].pc = d1 - 1;
            ChanParams p;
            fill_params(r, slot, &p);
            const uint64_t u1 = p.inc_q;
            if (cudaMemcpy(&r->d_st[slot].nco_q, &u1, sizeof u1, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = set_err(r, GPUD_E_CUDA, "segment state");
        }
    }
    if (!rc) rc = gpud_runner_set_host_outputs(r, 0);
    if (!rc) rc = gpud_runner_process_block(r, iq, n, iq_on_device);
    gpud_channel_result cr{};
    if (!rc) rc = gpud_runner_result(r, slot, &cr);
    if (!rc) {
        const float *d_audio = cr.audio;  // device pointer (host outputs off)
        const int na = cr.n_audio;
        if (rate > 48000 && na > 0) {
            auto aa = lowpass_fir(48000.0 / 2.0 * 0.9, rate, 63);
            int d2 = (int)std::llround((double)rate / 48000.0);
            if (d2 < 1) d2 = 1;
            const int frames = na / C;
            const int of = C == 2 ? frames / d2 : (frames + d2 - 1) / d2;
            if (of * C > out_cap) {
                rc = GPUD_E_ARG;
            } else {
                double *d_taps = nullptr;
                float *d_o = nullptr;
                if (cudaMalloc((void **)&d_taps, aa.size() * sizeof(double)) != cudaSuccess ||
                    cudaMalloc((void **)&d_o, (size_t)std::max(1, of * C) * sizeof(float)) != cudaSuccess ||
                    cudaMemcpy(d_taps, aa.data(), aa.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
                    launch_seg_aa(0, d_audio, C, d_taps, (int)aa.size(), d2, of, d_o) != cudaSuccess ||
                    cudaMemcpy(out, d_o, (size_t)of * C * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
                    rc = GPUD_E_CUDA;
                } else {
                    gpud_count_launch(of * C > 0 ? 1 : 0);
                    res->n_out = of * C;
                    res->out_rate = rate / d2;
                }
                cudaFree(d_taps);
                cudaFree(d_o);
            }
        } else if (na > out_cap) {
            rc = GPUD_E_ARG;
        } else {
            if (na > 0 && cudaMemcpy(out, d_audio, (size_t)na * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = GPUD_E_CUDA;
            res->n_out = na;
        }
    }
    gpud_runner_destroy(r);
    return rc;
}

// ---------------------------------------------------------------------------
// autotune table
// ---------------------------------------------------------------------------
GPUD_API int GPUD_CALL gpud_runner_set_autotune_table(gpud_runner *r, const gpud_autotune_entry *entries, int count) {
    if (!r || count < 0 || (count > 0 && !entries)) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    for (int i = 0; i < count; ++i) {
        const gpud_autotune_entry &e = entries[i];
        if (e.taps <= 0 || e.decim <= 0 || e.group_phases < 0 || !form_valid(e.taps, e.decim, e.form, e.group_phases))
            return set_err(r, GPUD_E_ARG, "autotune entry: form not valid for its geometry");
    }
    r->tune.assign(entries, entries + count);
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_channel_groups(gpud_runner *r, int enable) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    r->channel_groups = enable != 0;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_channel_form(gpud_runner *r, int slot, int *form, int *group_phases, int *groups) {
    if (!r || !form || !group_phases || !groups) return GPUD_E_ARG;
    std::lock_guard<std::recursive_mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    const Slot &s = r->slots[(size_t)slot];
    static const int kind_form[4] = {GPUD_FORM_DENSE, GPUD_FORM_WIDE, GPUD_FORM_GROUP, GPUD_FORM_MOD};
    *form = kind_form[s.ext_kind];
    *group_phases = s.pg;
    *groups = s.ng;
    return 0;
}


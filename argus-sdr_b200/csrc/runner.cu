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
//   - one H2D of the block, one H2D of the descriptors, one D2H of all outputs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
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
cudaError_t launch_extract_wide(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                const float2 *hist, const float *taps, float2 *ext);
cudaError_t launch_demod(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                         const ChanState *st, const float2 *ext, float *comp, float *audio);
cudaError_t launch_am(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const float2 *ext,
                      float *audio);
cudaError_t launch_wfm_fir(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const WfmTaps *taps, float *wk, int W, const float *comp_dl);
cudaError_t launch_pll(int count, cudaStream_t sm, const int *list, const SlotBlock *sbt, const ChanParams *prm,
                       ChanState *st, float *wk, int W, const int *done);
cudaError_t launch_pll_newton(int count, int cluster, cudaStream_t sm, const int *list, const SlotBlock *sbt,
                              const ChanParams *prm, ChanState *st, float *wk, int W, double *traj,
                              const int64_t *traj_off, int *done);
int pll_newton_threads();
cudaError_t launch_wfm_out(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const ChanState *st, const WfmTaps *taps, const float *wk, int W, const float *lr_dl,
                           const float *audio_dl, float *audio);
cudaError_t launch_rds(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                       const ChanParams *prm, const ChanState *st, const WfmTaps *taps, const BinadeTable *tabs,
                       const float *wk, const float2 *rds_dl, float2 *rds_out);
cudaError_t launch_post(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                        const float2 *x, int n, float2 *hist, const float2 *ext, const float *wk, int W,
                        float *comp_dl, float *lr_dl, float *audio_dl, float2 *rds_dl, const BinadeTable *tabs,
                        DevResult *res);
int rds_smem_bytes(int dr);
int dense_smem_bytes_host(int P, int L);

constexpr int kWfmTapsPadH = 104;
struct WfmTapsHost {
    float t[kWfmTapsPadH][4];
    double rds[kWfmTaps];
};
constexpr int kAudioDlStrideH = kWfmHist + 4;
constexpr int kMaxWfmClasses = 16;
constexpr int kDenseMaxL = 16;
constexpr int kDenseSmemLimit = 200 * 1024;

// ---------------------------------------------------------------------------
// DSP design helpers (host) -- restated from the reference
// ---------------------------------------------------------------------------

// dsp.LowpassFIR (internal/dsp/fir.go:6-28): Hann-windowed sinc, odd length.
static std::vector<double> lowpass_fir(double cutoff_hz, int sample_rate, int taps) {
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
static int build_binade_table(double inc, BinadeTable *t) {
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
    gpud_channel_spec spec{};
    int D = 1, T = 1, P = 1, L = 1, hcap = 0;
    int ext_kind = 0;  // 0 dense, 1 wide
    int taps_off = 0, dtaps_off = 0, hist_off = 0, wfm_idx = -1, rate_class = -1;
    double cutoff = 0;
    // host mirrors of device integer state
    int pc = 0, hist_len = 0, hist_sel = 0, comp_hist_len = 0;
    bool has_last = false;
    int64_t rds_count = 0;
    uint64_t footprint = 0;
    // last block bookkeeping
    SlotBlock sb{};
    int res_row = -1;
};

struct BlockPlan {
    int n = 0;
    std::vector<SlotBlock> sbs;
    std::vector<int> sb_slot;  // slot of each sb entry
    // work lists
    std::vector<int2> w_dense[kDenseMaxL + 1];
    int dense_smem[kDenseMaxL + 1] = {};
    std::vector<int2> w_wide;
    int wide_smem = 0;
    std::vector<int2> w_demod, w_am, w_fir, w_out, w_rds;
    int rds_smem = 0;
    std::vector<int> pll_list;
    std::vector<int64_t> pll_traj_off;  // doubles, per pll_list entry
    int64_t tot_traj = 0;
    int64_t tot_ext = 0, tot_emit_ext = 0, tot_comp = 0, tot_audio = 0, tot_rds = 0;
};

}  // namespace gpud

using namespace gpud;

struct gpud_runner {
    int fs = 0, max_block = 0, max_ch = 0, max_taps = 0;
    uint64_t budget = 0, used = 0;
    int schedule = GPUD_SCHED_BATCHED;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    std::mutex mu;

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
    std::vector<int> wfm_free;
    std::vector<int> class_rate;  // rate of each WFM rate class
    // per-block buffers (grown on demand)
    float2 *d_block = nullptr;
    float *d_wk = nullptr;
    int64_t wk_cap = 0;  // W (floats per work array)
    double *d_traj = nullptr;  // PLL trajectories (parallel-in-time solver)
    int64_t traj_cap = 0;
    int *d_done = nullptr;
    int64_t done_cap = 0;
    bool pll_parallel = true;
    int num_sms = 148;
    char *d_out = nullptr, *h_out = nullptr;
    size_t out_cap = 0;
    char *d_desc = nullptr, *h_desc = nullptr;
    size_t desc_cap = 0;
    float2 *h_in = nullptr;
    // last block layout
    BlockPlan plan;
    size_t off_res = 0, off_audio = 0, off_rds = 0, off_ext = 0, out_bytes = 0;
    // stats
    uint64_t blocks = 0, launches = 0;
    int graph_rebuilds = 0;
    std::vector<float> lat_ms;
    size_t lat_pos = 0;
    double last_ms = 0;
    uint64_t pending_ticket = 0, done_ticket = 0;
    cudaEvent_t ev_done = nullptr;
    // StreamingExtractGPU bookkeeping
    std::map<int64_t, int> by_signal;
    bool host_outputs = true;
    uint64_t last_h2d = 0, last_d2h = 0;
    // per-stage profiling
    bool profiling = false;
    std::vector<cudaEvent_t> prof_ev;
    std::vector<std::string> prof_names;
    int prof_n = 0;
    std::vector<gpud_stage_time> stage_times;
};

static void prof_mark(gpud_runner *r, const char *name) {
    if (!r->profiling) return;
    if ((int)r->prof_ev.size() <= r->prof_n) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        r->prof_ev.push_back(e);
        r->prof_names.emplace_back();
    }
    cudaEventRecord(r->prof_ev[(size_t)r->prof_n], r->stream);
    r->prof_names[(size_t)r->prof_n] = name;
    r->prof_n++;
}

static void prof_collect(gpud_runner *r) {
    if (!r->profiling || r->prof_n < 2) return;
    r->stage_times.clear();
    for (int i = 0; i + 1 < r->prof_n; ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, r->prof_ev[(size_t)i], r->prof_ev[(size_t)i + 1]);
        gpud_stage_time t{};
        std::snprintf(t.name, sizeof t.name, "%s", r->prof_names[(size_t)i].c_str());
        t.ms = ms;
        r->stage_times.push_back(t);
    }
}

static int set_err(gpud_runner *r, int code, const char *what, cudaError_t e = cudaSuccess) {
    char buf[256];
    if (e != cudaSuccess)
        std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    else
        std::snprintf(buf, sizeof buf, "%s", what);
    r->err = buf;
    return code;
}

#define CK(call)                                                     \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return set_err(r, GPUD_E_CUDA, #call, e_); \
    } while (0)

template <typename T>
static cudaError_t dalloc(T **p, size_t count) {
    return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

// Bytes of per-block buffers one slot needs at max_block.
static uint64_t slot_block_bytes(const gpud_runner *r, int D, int mode, int flags) {
    uint64_t nout = (uint64_t)r->max_block / (uint64_t)D + 2;
    uint64_t b = nout * 8;  // extracted IQ (in the output arena)
    bool wfm = mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    if (wfm) b += 5 * (nout + 8) * 4;  // composite work arrays
    if (mode != GPUD_MODE_IQ) b += nout * 4 * (mode == GPUD_MODE_WFM_STEREO ? 2 : 1);
    if (wfm && (flags & GPUD_CH_RDS)) b += (nout / 16 + 4) * 8;
    return b;
}

static uint64_t slot_state_bytes(const gpud_runner *r) {
    return sizeof(ChanParams) + sizeof(ChanState) + (uint64_t)r->tapcap * 2 * 4 + (uint64_t)2 * r->max_taps * 8 +
           (kWfmHist * 3 + kAudioDlStrideH) * 8;
}

static int rate_class_for(gpud_runner *r, int rate) {
    for (size_t i = 0; i < r->class_rate.size(); ++i)
        if (r->class_rate[i] == rate) return (int)i;
    if ((int)r->class_rate.size() >= kMaxWfmClasses) return -1;
    int id = (int)r->class_rate.size();
    r->class_rate.push_back(rate);
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
    BinadeTable tab;
    build_binade_table(-2 * GPUD_PI * (-57000.0) / (double)rate, &tab);
    if (cudaMemcpy(r->d_wtaps + id, &h, sizeof h, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (cudaMemcpy(r->d_tabs + id, &tab, sizeof tab, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    return id;
}

// Tap design of gpudemod/stream_state.go:57-77 (cutoff = max(BW/2, 200),
// LowpassFIR in float64, cast to float32, the first T taps applied), laid out
// phase-major (p*L + u -> h[p + u*D]) and direct.
static int upload_taps(gpud_runner *r, int slot, double bandwidth) {
    Slot &s = r->slots[(size_t)slot];
    double cutoff = bandwidth / 2;
    if (cutoff < 200) cutoff = 200;
    auto base = lowpass_fir(cutoff, r->fs, s.T);
    std::vector<float> h((size_t)s.T);
    for (int k = 0; k < s.T; ++k) h[(size_t)k] = (float)base[(size_t)k];
    std::vector<float> pm((size_t)s.P * s.L, 0.f);
    for (int p = 0; p < s.P; ++p)
        for (int u = 0; u < s.L; ++u) {
            int k = p + u * s.D;
            pm[(size_t)p * s.L + u] = k < s.T ? h[(size_t)k] : 0.f;
        }
    CK(cudaMemcpyAsync(r->d_taps + s.taps_off, pm.data(), pm.size() * 4, cudaMemcpyHostToDevice, r->stream));
    CK(cudaMemcpyAsync(r->d_taps + s.dtaps_off, h.data(), h.size() * 4, cudaMemcpyHostToDevice, r->stream));
    CK(cudaStreamSynchronize(r->stream));
    s.cutoff = cutoff;
    return 0;
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
    p->out_rate = s.spec.out_rate;
    p->taps_off = s.taps_off;
    p->dtaps_off = s.dtaps_off;
    p->hist_off = s.hist_off;
    p->hcap = s.hcap;
    p->wfm_idx = s.wfm_idx;
    int rate = s.spec.out_rate;
    p->rds_dr = std::max(1, rate / 19000);
    double bfo = s.spec.mode == GPUD_MODE_LSB ? -700.0 : 700.0;
    p->ssb_inc = 2 * GPUD_PI * bfo / (double)rate;
    pll_coefficients(50, 0.707, rate, &p->pll_alpha, &p->pll_beta);
    p->pll_lpa = 1 - std::exp(-2 * GPUD_PI * 200 / (double)rate);
    p->pll_fmin = 2 * GPUD_PI * 17000 / (double)rate;
    p->pll_fmax = 2 * GPUD_PI * 21000 / (double)rate;
    p->rds_inc = -2 * GPUD_PI * (-57000.0) / (double)rate;
    p->rds_tab = s.rate_class < 0 ? 0 : s.rate_class;
}

// Fresh device state: NCO phase 0, empty histories, PLL as built by
// stereoDecodeStateful's first call (streamer.go:1546-1555).
static int reset_slot_state(gpud_runner *r, int slot) {
    Slot &s = r->slots[(size_t)slot];
    ChanState st{};
    st.pll_freq = 2 * GPUD_PI * 19000 / (double)s.spec.out_rate;
    CK(cudaMemcpyAsync(r->d_st + slot, &st, sizeof st, cudaMemcpyHostToDevice, r->stream));
    if (s.wfm_idx >= 0) {
        CK(cudaMemsetAsync(r->d_comp_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 4, r->stream));
        CK(cudaMemsetAsync(r->d_lr_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 4, r->stream));
        CK(cudaMemsetAsync(r->d_audio_dl + (size_t)s.wfm_idx * kAudioDlStrideH, 0, kAudioDlStrideH * 4, r->stream));
        CK(cudaMemsetAsync(r->d_rds_dl + (size_t)s.wfm_idx * kWfmHist, 0, kWfmHist * 8, r->stream));
    }
    s.pc = 0;
    s.hist_len = 0;
    s.hist_sel = 0;
    s.has_last = false;
    s.comp_hist_len = 0;
    s.rds_count = 0;
    CK(cudaStreamSynchronize(r->stream));
    return 0;
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
    return 0;
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
#define CKC(call)                             \
    do {                                      \
        if ((call) != cudaSuccess) {          \
            gpud_runner_destroy(r);           \
            return GPUD_E_CUDA;               \
        }                                     \
    } while (0)
    CKC(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    {
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
            r->num_sms = sms;
    }
    CKC(cudaEventCreate(&r->ev0));
    CKC(cudaEventCreate(&r->ev1));
    CKC(cudaEventCreateWithFlags(&r->ev_done, cudaEventDisableTiming));
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
    CKC(dalloc(&r->d_tabs, (size_t)kMaxWfmClasses));
    CKC(dalloc(&r->d_block, (size_t)max_block));
    CKC(cudaMallocHost((void **)&r->h_in, (size_t)max_block * sizeof(float2)));
#undef CKC
    r->used = slot_state_bytes(r) * M + (uint64_t)max_block * 8;
    for (int i = max_channels - 1; i >= 0; --i) r->wfm_free.push_back(i);
    *out = r;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_destroy(gpud_runner *r) {
    if (!r) return 0;
    if (r->stream) cudaStreamSynchronize(r->stream);
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
    cudaFree(r->d_block);
    cudaFree(r->d_wk);
    cudaFree(r->d_traj);
    cudaFree(r->d_done);
    cudaFree(r->d_out);
    cudaFree(r->d_desc);
    if (r->h_out) cudaFreeHost(r->h_out);
    if (r->h_desc) cudaFreeHost(r->h_desc);
    if (r->h_in) cudaFreeHost(r->h_in);
    if (r->ev0) cudaEventDestroy(r->ev0);
    if (r->ev1) cudaEventDestroy(r->ev1);
    if (r->ev_done) cudaEventDestroy(r->ev_done);
    for (auto e : r->prof_ev) cudaEventDestroy(e);
    if (r->stream) cudaStreamDestroy(r->stream);
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

GPUD_API int GPUD_CALL gpud_runner_admit(gpud_runner *r, const gpud_channel_spec *spec, int *slot_out) {
    if (!r || !slot_out) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    int D, T;
    int rc = validate_spec(r, spec, &D, &T);
    if (rc) return rc;
    int slot = -1;
    for (int i = 0; i < r->max_ch; ++i)
        if (!r->slots[(size_t)i].active) {
            slot = i;
            break;
        }
    if (slot < 0) return set_err(r, GPUD_E_SLOTS, "channel cap reached");
    uint64_t fp = slot_block_bytes(r, D, spec->mode, spec->flags);
    if (r->budget && r->used + fp > r->budget) return set_err(r, GPUD_E_BUDGET, "device-memory budget exhausted");
    bool wfm = spec->mode == GPUD_MODE_WFM || spec->mode == GPUD_MODE_WFM_STEREO;
    int rclass = -1;
    if (wfm) {
        rclass = rate_class_for(r, spec->out_rate);
        if (rclass < 0) return set_err(r, GPUD_E_CUDA, "WFM rate classes exhausted");
    }
    Slot &s = r->slots[(size_t)slot];
    s = Slot{};
    s.active = true;
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
    int smem = dense_smem_bytes_host(s.P, s.L);
    s.ext_kind = (s.L >= 2 && s.L <= kDenseMaxL && smem <= kDenseSmemLimit) ? 0 : 1;
    s.footprint = fp;
    rc = upload_taps(r, slot, spec->bandwidth);
    if (rc) {
        s.active = false;
        return rc;
    }
    ChanParams p;
    fill_params(r, slot, &p);
    CK(cudaMemcpyAsync(r->d_prm + slot, &p, sizeof p, cudaMemcpyHostToDevice, r->stream));
    rc = reset_slot_state(r, slot);
    if (rc) {
        s.active = false;
        return rc;
    }
    r->used += fp;
    *slot_out = slot;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_retire(gpud_runner *r, int slot) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    r->used -= s.footprint;
    s.active = false;
    for (auto it = r->by_signal.begin(); it != r->by_signal.end(); ++it)
        if (it->second == slot) {
            r->by_signal.erase(it);
            break;
        }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_update(gpud_runner *r, int slot, double offset_hz, double bandwidth) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    double cutoff = bandwidth / 2;
    if (cutoff < 200) cutoff = 200;
    if (cutoff != s.cutoff) {
        int rc = upload_taps(r, slot, bandwidth);
        if (rc) return rc;
    }
    s.spec.bandwidth = bandwidth;
    if (offset_hz != s.spec.offset_hz) {
        s.spec.offset_hz = offset_hz;
        ChanParams p;
        fill_params(r, slot, &p);
        CK(cudaMemcpyAsync(r->d_prm + slot, &p, sizeof p, cudaMemcpyHostToDevice, r->stream));
        CK(cudaStreamSynchronize(r->stream));
    }
    return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// block planning
// ---------------------------------------------------------------------------
int gpud::dense_smem_bytes_host(int P, int L) {
    int M = 256 + L - 1;
    int Mp = (M + (M >> 3) + 1) | 1;
    int z = P * Mp * 8;
    int red = 8 * (256 + 32) * 8;
    return std::max(z, red) + P * L * 4 + 16;
}

static void plan_slot(gpud_runner *r, BlockPlan &pl, int slot, int n) {
    Slot &s = r->slots[(size_t)slot];
    SlotBlock sb{};
    sb.slot = slot;
    sb.pc = s.pc;
    sb.n_out = (s.pc + n) / s.D;
    sb.hist_len = s.hist_len;
    sb.hist_sel = s.hist_sel;
    int mode = s.spec.mode;
    bool fm = mode == GPUD_MODE_NFM || mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    bool wfm = mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO;
    sb.n_disc = 0;
    sb.bridge = 0;
    if (fm && sb.n_out > 0) {
        sb.bridge = s.has_last ? 1 : 0;
        sb.n_disc = s.has_last ? sb.n_out : sb.n_out - 1;
    }
    switch (mode) {
    case GPUD_MODE_NFM:
    case GPUD_MODE_WFM: sb.n_audio = sb.n_disc; break;
    case GPUD_MODE_WFM_STEREO: sb.n_audio = 2 * sb.n_disc; break;
    case GPUD_MODE_AM:
    case GPUD_MODE_USB:
    case GPUD_MODE_LSB:
    case GPUD_MODE_CW: sb.n_audio = sb.n_out; break;
    default: sb.n_audio = 0;
    }
    sb.comp_hist_len = s.comp_hist_len;
    sb.n_rds = 0;
    sb.rds_first = -1;
    if (wfm && (s.spec.flags & GPUD_CH_RDS) && sb.n_disc > 0) {
        int dr = std::max(1, s.spec.out_rate / 19000);
        int64_t c0 = s.rds_count;
        int qf = (int)((dr - c0 % dr) % dr);
        if (qf < sb.n_disc) {
            sb.rds_first = qf;
            sb.n_rds = (sb.n_disc - 1 - qf) / dr + 1;
        }
    }
    sb.res_idx = (int)pl.sbs.size();
    pl.sbs.push_back(sb);
    pl.sb_slot.push_back(slot);
}

// Offsets (emitting slots' IQ first so one D2H covers it) and work lists.
static void finish_plan(gpud_runner *r, BlockPlan &pl) {
    int64_t ext = 0;
    for (int pass = 0; pass < 2; ++pass)
        for (auto &sb : pl.sbs) {
            bool emit = (r->slots[(size_t)sb.slot].spec.flags & GPUD_CH_EMIT_IQ) != 0;
            if (emit != (pass == 0)) continue;
            sb.ext_off = (int)ext;
            ext += (sb.n_out + 3) & ~3;
            if (pass == 0) pl.tot_emit_ext = ext;
        }
    pl.tot_ext = ext;
    int64_t comp = 0, audio = 0, rds = 0;
    for (auto &sb : pl.sbs) {
        Slot &s = r->slots[(size_t)sb.slot];
        sb.comp_off = (int)comp;
        if (s.wfm_idx >= 0) comp += (sb.n_disc + 8 + 7) & ~7;
        sb.audio_off = (int)audio;
        audio += (sb.n_audio + 3) & ~3;
        sb.rds_off = (int)rds;
        rds += (sb.n_rds + 1) & ~1;
    }
    pl.tot_comp = comp;
    pl.tot_audio = audio;
    pl.tot_rds = rds;
    for (int L = 0; L <= kDenseMaxL; ++L) {
        pl.w_dense[L].clear();
        pl.dense_smem[L] = 0;
    }
    pl.w_wide.clear();
    pl.wide_smem = 0;
    pl.w_demod.clear();
    pl.w_am.clear();
    pl.w_fir.clear();
    pl.w_out.clear();
    pl.w_rds.clear();
    pl.pll_list.clear();
    pl.pll_traj_off.clear();
    pl.tot_traj = 0;
    pl.rds_smem = 0;
    for (int i = 0; i < (int)pl.sbs.size(); ++i) {
        const SlotBlock &sb = pl.sbs[(size_t)i];
        Slot &s = r->slots[(size_t)sb.slot];
        if (sb.n_out > 0) {
            if (s.ext_kind == 0) {
                for (int t = 0; t * 256 < sb.n_out; ++t) pl.w_dense[s.L].push_back(make_int2(i, t));
                pl.dense_smem[s.L] = std::max(pl.dense_smem[s.L], dense_smem_bytes_host(s.P, s.L));
            } else {
                for (int t = 0; t * 32 < sb.n_out; ++t) pl.w_wide.push_back(make_int2(i, t));
                pl.wide_smem = std::max(pl.wide_smem, s.T * 4);
            }
        }
        int mode = s.spec.mode;
        int nd = (mode == GPUD_MODE_USB || mode == GPUD_MODE_LSB || mode == GPUD_MODE_CW) ? sb.n_out : sb.n_disc;
        if ((mode >= GPUD_MODE_NFM && mode <= GPUD_MODE_WFM_STEREO) || mode >= GPUD_MODE_USB)
            for (int t = 0; t * 1024 < nd; ++t) pl.w_demod.push_back(make_int2(i, t));
        if (mode == GPUD_MODE_AM && sb.n_out > 0) pl.w_am.push_back(make_int2(i, 0));
        if (mode == GPUD_MODE_WFM_STEREO && sb.n_disc > 0) {
            for (int t = 0; t * 1024 < sb.n_disc; ++t) pl.w_fir.push_back(make_int2(i, t));
            pl.pll_list.push_back(i);
            pl.pll_traj_off.push_back(pl.tot_traj);
            pl.tot_traj += 8 * ((int64_t)sb.n_disc + 1);
        }
        if ((mode == GPUD_MODE_WFM || mode == GPUD_MODE_WFM_STEREO) && sb.n_disc > 0)
            for (int t = 0; t * 1024 < sb.n_disc; ++t) pl.w_out.push_back(make_int2(i, t));
        if (sb.n_rds > 0) {
            for (int t = 0; t * 64 < sb.n_rds; ++t) pl.w_rds.push_back(make_int2(i, t));
            pl.rds_smem = std::max(pl.rds_smem, rds_smem_bytes(std::max(1, s.spec.out_rate / 19000)));
        }
    }
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static int ensure_buffers(gpud_runner *r, const BlockPlan &pl) {
    int64_t W = std::max<int64_t>(pl.tot_comp, 8);
    if (W > r->wk_cap) {
        cudaFree(r->d_wk);
        r->d_wk = nullptr;
        int64_t cap = std::max<int64_t>(W * 5 / 4, 1 << 16);
        CK(dalloc(&r->d_wk, (size_t)cap * 5));
        r->wk_cap = cap;
        r->graph_rebuilds++;
    }
    if (pl.tot_traj > r->traj_cap) {
        cudaFree(r->d_traj);
        r->d_traj = nullptr;
        int64_t cap = std::max<int64_t>(pl.tot_traj * 5 / 4, 1 << 16);
        CK(dalloc(&r->d_traj, (size_t)cap));
        r->traj_cap = cap;
    }
    if ((int64_t)pl.pll_list.size() > r->done_cap) {
        cudaFree(r->d_done);
        r->d_done = nullptr;
        int64_t cap = std::max<int64_t>((int64_t)pl.pll_list.size() * 2, 64);
        CK(dalloc(&r->d_done, (size_t)cap));
        r->done_cap = cap;
    }
    size_t res = align256(pl.sbs.size() * sizeof(DevResult));
    size_t need = res + align256((size_t)pl.tot_audio * 4) + align256((size_t)pl.tot_rds * 8) +
                  align256((size_t)pl.tot_ext * 8);
    if (need > r->out_cap) {
        cudaFree(r->d_out);
        if (r->h_out) cudaFreeHost(r->h_out);
        r->d_out = nullptr;
        r->h_out = nullptr;
        size_t cap = need * 5 / 4 + 4096;
        CK(cudaMalloc((void **)&r->d_out, cap));
        CK(cudaMallocHost((void **)&r->h_out, cap));
        r->out_cap = cap;
        r->graph_rebuilds++;
    }
    size_t nw = 0;
    for (int L = 0; L <= kDenseMaxL; ++L) nw += pl.w_dense[L].size();
    nw += pl.w_wide.size() + pl.w_demod.size() + pl.w_am.size() + pl.w_fir.size() + pl.w_out.size() +
          pl.w_rds.size();
    size_t dneed = align256(pl.sbs.size() * sizeof(SlotBlock)) + align256(nw * sizeof(int2)) +
                   align256(pl.pll_list.size() * 4) + align256(pl.pll_list.size() * 8) + 4096;
    if (dneed > r->desc_cap) {
        cudaFree(r->d_desc);
        if (r->h_desc) cudaFreeHost(r->h_desc);
        r->d_desc = nullptr;
        r->h_desc = nullptr;
        size_t cap = dneed * 5 / 4 + 4096;
        CK(cudaMalloc((void **)&r->d_desc, cap));
        CK(cudaMallocHost((void **)&r->h_desc, cap));
        r->desc_cap = cap;
    }
    return 0;
}

// Host mirrors advance exactly as the device state does.
static void advance_mirrors(gpud_runner *r, const BlockPlan &pl, int n) {
    for (const SlotBlock &sb : pl.sbs) {
        Slot &s = r->slots[(size_t)sb.slot];
        s.pc = (s.pc + n) % s.D;
        s.hist_len = std::min(s.T - 1, s.hist_len + n);
        s.hist_sel = 1 - s.hist_sel;
        if (sb.n_out > 0) s.has_last = true;
        if (s.wfm_idx >= 0) {
            s.comp_hist_len = std::min(kWfmHist, s.comp_hist_len + sb.n_disc);
            s.rds_count += sb.n_disc;
        }
        s.sb = sb;
    }
}

// Enqueue descriptor upload, kernels and the output D2H for the slots in pl.
static int enqueue_block(gpud_runner *r, BlockPlan &pl, const float2 *x_dev, int n) {
    // descriptor staging
    char *hd = r->h_desc;
    size_t o_sb = 0, o_w = align256(pl.sbs.size() * sizeof(SlotBlock));
    std::memcpy(hd + o_sb, pl.sbs.data(), pl.sbs.size() * sizeof(SlotBlock));
    int2 *hw = (int2 *)(hd + o_w);
    size_t cnt = 0;
    size_t w_dense_off[kDenseMaxL + 1];
    for (int L = 0; L <= kDenseMaxL; ++L) {
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
           o_out = put(pl.w_out), o_rds = put(pl.w_rds);
    size_t o_pll = o_w + align256(cnt * sizeof(int2));
    std::memcpy(hd + o_pll, pl.pll_list.data(), pl.pll_list.size() * 4);
    size_t o_traj = o_pll + align256(pl.pll_list.size() * 4);
    std::memcpy(hd + o_traj, pl.pll_traj_off.data(), pl.pll_traj_off.size() * 8);
    size_t dbytes = o_traj + pl.pll_traj_off.size() * 8;
    CK(cudaMemcpyAsync(r->d_desc, hd, dbytes, cudaMemcpyHostToDevice, r->stream));
    const SlotBlock *d_sb = (const SlotBlock *)(r->d_desc + o_sb);
    const int2 *d_w = (const int2 *)(r->d_desc + o_w);
    const int *d_pll = (const int *)(r->d_desc + o_pll);
    const int64_t *d_traj_off = (const int64_t *)(r->d_desc + o_traj);

    r->off_res = 0;
    r->off_audio = align256(pl.sbs.size() * sizeof(DevResult));
    r->off_rds = r->off_audio + align256((size_t)pl.tot_audio * 4);
    r->off_ext = r->off_rds + align256((size_t)pl.tot_rds * 8);
    DevResult *d_res = (DevResult *)(r->d_out + r->off_res);
    float *d_audio = (float *)(r->d_out + r->off_audio);
    float2 *d_rds = (float2 *)(r->d_out + r->off_rds);
    float2 *d_ext = (float2 *)(r->d_out + r->off_ext);
    const int W = (int)r->wk_cap;
    const WfmTaps *wt = (const WfmTaps *)r->d_wtaps;
    int nl = 0;
    for (int L = 0; L <= kDenseMaxL; ++L) {
        if (pl.w_dense[L].empty()) continue;
        prof_mark(r, L < 10 ? (std::string("extract_dense_L") + char('0' + L)).c_str() : (std::string("extract_dense_L1") + char('0' + L - 10)).c_str());
        CK(launch_extract_dense(L, (int)pl.w_dense[L].size(), pl.dense_smem[L], r->stream, d_w + w_dense_off[L],
                                d_sb, r->d_prm, r->d_st, x_dev, n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    if (!pl.w_wide.empty()) {
        prof_mark(r, "extract_wide");
        CK(launch_extract_wide((int)pl.w_wide.size(), pl.wide_smem, r->stream, d_w + o_wide, d_sb, r->d_prm, r->d_st,
                               x_dev, n, r->d_hist, r->d_taps, d_ext));
        nl++;
    }
    if (!pl.w_demod.empty()) {
        prof_mark(r, "demod");
        CK(launch_demod((int)pl.w_demod.size(), r->stream, d_w + o_dem, d_sb, r->d_prm, r->d_st, d_ext, r->d_wk,
                        d_audio));
        nl++;
    }
    if (!pl.w_am.empty()) {
        prof_mark(r, "am");
        CK(launch_am((int)pl.w_am.size(), r->stream, d_w + o_am, d_sb, d_ext, d_audio));
        nl++;
    }
    if (!pl.w_fir.empty()) {
        prof_mark(r, "wfm_fir");
        CK(launch_wfm_fir((int)pl.w_fir.size(), r->stream, d_w + o_fir, d_sb, r->d_prm, wt, r->d_wk, W, r->d_comp_dl));
        nl++;
    }
    if (!pl.pll_list.empty()) {
        const int *done = nullptr;
        if (r->pll_parallel) {
            // cluster size: enough CTAs to cover the SMs, no more than 8 per
            // channel, at least 8 steps per thread
            int nch = (int)pl.pll_list.size();
            int max_n = 0;
            for (int i : pl.pll_list) max_n = std::max(max_n, pl.sbs[(size_t)i].n_disc);
            int cluster = 1;
            while (cluster < 8 && nch * cluster * 2 <= 3 * r->num_sms &&
                   max_n / (cluster * 2 * pll_newton_threads()) >= 8)
                cluster *= 2;
            prof_mark(r, "pll_newton");
            CK(launch_pll_newton(nch, cluster, r->stream, d_pll, d_sb, r->d_prm, r->d_st, r->d_wk, W, r->d_traj,
                                 d_traj_off, r->d_done));
            nl++;
            done = r->d_done;
        }
        prof_mark(r, "pll_serial");
        CK(launch_pll((int)pl.pll_list.size(), r->stream, d_pll, d_sb, r->d_prm, r->d_st, r->d_wk, W, done));
        nl++;
    }
    if (!pl.w_out.empty()) {
        prof_mark(r, "wfm_out");
        CK(launch_wfm_out((int)pl.w_out.size(), r->stream, d_w + o_out, d_sb, r->d_prm, r->d_st, wt, r->d_wk, W,
                          r->d_lr_dl, r->d_audio_dl, d_audio));
        nl++;
    }
    if (!pl.w_rds.empty()) {
        prof_mark(r, "rds");
        CK(launch_rds((int)pl.w_rds.size(), pl.rds_smem, r->stream, d_w + o_rds, d_sb, r->d_prm, r->d_st, wt,
                      r->d_tabs, r->d_wk, r->d_rds_dl, d_rds));
        nl++;
    }
    if (!pl.sbs.empty()) {
        prof_mark(r, "post");
        CK(launch_post((int)pl.sbs.size(), r->stream, d_sb, r->d_prm, r->d_st, x_dev, n, r->d_hist, d_ext, r->d_wk, W,
                       r->d_comp_dl, r->d_lr_dl, r->d_audio_dl, r->d_rds_dl, r->d_tabs, d_res));
        nl++;
    }
    prof_mark(r, "d2h");
    r->launches += (uint64_t)nl;
    gpud_count_launch(nl);
    r->out_bytes = r->off_ext + (size_t)pl.tot_emit_ext * 8;
    if (r->host_outputs) {
        CK(cudaMemcpyAsync(r->h_out, r->d_out, r->out_bytes, cudaMemcpyDeviceToHost, r->stream));
        r->last_d2h += r->out_bytes;
    } else {
        // keep the results table on the host (small); payload stays on the device
        CK(cudaMemcpyAsync(r->h_out, r->d_out, r->off_audio, cudaMemcpyDeviceToHost, r->stream));
        r->last_d2h += r->off_audio;
    }
    r->last_h2d += dbytes;
    prof_mark(r, "end");
    return 0;
}

static int stage_input(gpud_runner *r, const gpud_float2 *iq, int n, int on_device, const float2 **x_dev) {
    if (n == 0) {
        *x_dev = r->d_block;
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
        std::memcpy(r->h_in, iq, (size_t)n * sizeof(float2));
        src = r->h_in;
    }
    CK(cudaMemcpyAsync(r->d_block, src, (size_t)n * sizeof(float2), cudaMemcpyHostToDevice, r->stream));
    r->last_h2d += (uint64_t)n * sizeof(float2);
    *x_dev = r->d_block;
    return 0;
}

static void record_latency(gpud_runner *r) {
    float ms = 0;
    cudaEventElapsedTime(&ms, r->ev0, r->ev1);
    r->last_ms = ms;
    r->lat_ms[r->lat_pos % r->lat_ms.size()] = ms;
    r->lat_pos++;
}

static int run_block(gpud_runner *r, const gpud_float2 *iq, int n, int on_device, bool wait) {
    if (n < 0 || n > r->max_block) return set_err(r, GPUD_E_BLOCK, "block larger than max_block");
    if (r->pending_ticket != r->done_ticket) {
        CK(cudaEventSynchronize(r->ev_done));
        r->done_ticket = r->pending_ticket;
    }
    r->prof_n = 0;
    r->last_h2d = r->last_d2h = 0;
    CK(cudaEventRecord(r->ev0, r->stream));
    prof_mark(r, "h2d");
    const float2 *x = nullptr;
    int rc = stage_input(r, iq, n, on_device, &x);
    if (rc) return rc;
    if (r->schedule == GPUD_SCHED_BATCHED) {
        BlockPlan &pl = r->plan;
        pl.sbs.clear();
        pl.sb_slot.clear();
        pl.n = n;
        for (int i = 0; i < r->max_ch; ++i)
            if (r->slots[(size_t)i].active) plan_slot(r, pl, i, n);
        finish_plan(r, pl);
        rc = ensure_buffers(r, pl);
        if (rc) return rc;
        if (!pl.sbs.empty()) {
            rc = enqueue_block(r, pl, x, n);
            if (rc) return rc;
        }
        advance_mirrors(r, pl, n);
        for (size_t i = 0; i < pl.sbs.size(); ++i) r->slots[(size_t)pl.sbs[i].slot].res_row = (int)i;
    } else {
        // Plain per-signal schedule (mirrors executeStreamingGPUNativePrepared,
        // streaming_gpu_native_prepare.go:25-106): each channel alone, its own
        // descriptor upload, launches and D2H, synchronised before the next.
        // Results are gathered into the same host arena layout.
        BlockPlan full;
        full.n = n;
        for (int i = 0; i < r->max_ch; ++i)
            if (r->slots[(size_t)i].active) plan_slot(r, full, i, n);
        finish_plan(r, full);
        rc = ensure_buffers(r, full);
        if (rc) return rc;
        std::vector<char> gathered;
        size_t res_b = align256(full.sbs.size() * sizeof(DevResult));
        size_t a_off = res_b, r_off = a_off + align256((size_t)full.tot_audio * 4),
               e_off = r_off + align256((size_t)full.tot_rds * 8);
        gathered.assign(e_off + align256((size_t)full.tot_ext * 8), 0);
        for (size_t k = 0; k < full.sbs.size(); ++k) {
            BlockPlan one;
            one.n = n;
            SlotBlock sb = full.sbs[k];
            int slot = sb.slot;
            Slot &s = r->slots[(size_t)slot];
            if (!on_device && n > 0) {  // the reference copies the whole block per signal
                rc = stage_input(r, iq, n, 0, &x);
                if (rc) return rc;
            }
            plan_slot(r, one, slot, n);
            finish_plan(r, one);
            rc = enqueue_block(r, one, x, n);
            if (rc) return rc;
            CK(cudaStreamSynchronize(r->stream));
            const SlotBlock &o = one.sbs[0];
            const SlotBlock &f = full.sbs[k];
            std::memcpy(gathered.data() + k * sizeof(DevResult), r->h_out + r->off_res, sizeof(DevResult));
            std::memcpy(gathered.data() + a_off + (size_t)f.audio_off * 4, r->h_out + r->off_audio +
                        (size_t)o.audio_off * 4, (size_t)o.n_audio * 4);
            std::memcpy(gathered.data() + r_off + (size_t)f.rds_off * 8, r->h_out + r->off_rds + (size_t)o.rds_off * 8,
                        (size_t)o.n_rds * 8);
            if (s.spec.flags & GPUD_CH_EMIT_IQ)
                std::memcpy(gathered.data() + e_off + (size_t)f.ext_off * 8,
                            r->h_out + r->off_ext + (size_t)o.ext_off * 8, (size_t)o.n_out * 8);
            advance_mirrors(r, one, n);
        }
        std::memcpy(r->h_out, gathered.data(), gathered.size());
        r->off_res = 0;
        r->off_audio = a_off;
        r->off_rds = r_off;
        r->off_ext = e_off;
        r->plan = full;
        for (size_t i = 0; i < full.sbs.size(); ++i) {
            Slot &s = r->slots[(size_t)full.sbs[i].slot];
            s.res_row = (int)i;
            s.sb = full.sbs[i];
        }
    }
    CK(cudaEventRecord(r->ev1, r->stream));
    CK(cudaEventRecord(r->ev_done, r->stream));
    r->pending_ticket++;
    r->blocks++;
    if (wait) {
        CK(cudaEventSynchronize(r->ev_done));
        r->done_ticket = r->pending_ticket;
        record_latency(r);
        prof_collect(r);
    }
    return 0;
}

extern "C" {

GPUD_API int GPUD_CALL gpud_runner_process_block(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    return run_block(r, iq, n, iq_on_device, true);
}

GPUD_API int GPUD_CALL gpud_runner_submit(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device,
                                          uint64_t *ticket) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    int rc = run_block(r, iq, n, iq_on_device, false);
    if (rc) return rc;
    if (ticket) *ticket = r->pending_ticket;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_wait(gpud_runner *r, uint64_t ticket, int timeout_ms) {
    if (!r) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (ticket <= r->done_ticket) return 0;
    // bounded poll: never block past timeout_ms
    double waited = 0;
    while (true) {
        cudaError_t q = cudaEventQuery(r->ev_done);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) return set_err(r, GPUD_E_CUDA, "event query", q);
        if (timeout_ms >= 0 && waited >= timeout_ms) return set_err(r, GPUD_E_TIMEOUT, "wait timed out");
        struct timespec ts{0, 50000};
        nanosleep(&ts, nullptr);
        waited += 0.05;
    }
    r->done_ticket = r->pending_ticket;
    record_latency(r);
    prof_collect(r);
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_host_outputs(gpud_runner *r, int on) {
    if (!r) return GPUD_E_ARG;
    r->host_outputs = on != 0;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_set_pll_solver(gpud_runner *r, int parallel) {
    if (!r) return GPUD_E_ARG;
    r->pll_parallel = parallel != 0;
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

GPUD_API int GPUD_CALL gpud_runner_result(gpud_runner *r, int slot, gpud_channel_result *out) {
    if (!r || !out) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    if (r->pending_ticket != r->done_ticket) return set_err(r, GPUD_E_TIMEOUT, "block still in flight");
    Slot &s = r->slots[(size_t)slot];
    std::memset(out, 0, sizeof *out);
    out->signal_id = s.spec.signal_id;
    out->rate = s.spec.out_rate;
    out->phase_count = s.pc;
    out->history_len = s.hist_len;
    out->audio_channels = s.spec.mode == GPUD_MODE_WFM_STEREO ? 2 : (s.spec.mode == GPUD_MODE_IQ ? 0 : 1);
    out->rds_rate = s.spec.out_rate / std::max(1, s.spec.out_rate / 19000);
    if (s.res_row < 0 || s.res_row >= (int)r->plan.sbs.size() || r->plan.sbs[(size_t)s.res_row].slot != slot) {
        return 0;  // admitted after the last block: no outputs yet
    }
    const SlotBlock &sb = s.sb;
    const DevResult *res = (const DevResult *)(r->h_out + r->off_res) + s.res_row;
    out->n_iq = sb.n_out;
    out->nco_phase = res->nco_phase;
    out->n_audio = sb.n_audio;
    out->n_rds = sb.n_rds;
    out->flags = res->flags;
    out->coherence = res->coherence;
    out->pilot_hz = res->pilot_hz;
    out->err_avg = res->err_avg;
    out->pll_path = res->status;
    out->pll_iters = res->pll_iters;
    const char *base = r->host_outputs ? r->h_out : r->d_out;
    out->audio = (const float *)(base + r->off_audio) + sb.audio_off;
    out->rds = (const gpud_float2 *)(base + r->off_rds) + sb.rds_off;
    out->iq = (s.spec.flags & GPUD_CH_EMIT_IQ) ? (const gpud_float2 *)(base + r->off_ext) + sb.ext_off : nullptr;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_stats_get(gpud_runner *r, gpud_runner_stats *out) {
    if (!r || !out) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
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
    out->last_h2d_bytes = r->last_h2d;
    out->last_d2h_bytes = r->last_d2h;
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
};

static uint64_t snap_bytes(const Slot &s) {
    uint64_t b = sizeof(SnapHeader) + sizeof(ChanState) + (uint64_t)s.hcap * 8;
    if (s.wfm_idx >= 0) b += kWfmHist * 4 * 2 + kAudioDlStrideH * 4 + kWfmHist * 8;
    return b;
}

GPUD_API int GPUD_CALL gpud_runner_snapshot(gpud_runner *r, int slot, void *blob, uint64_t *bytes) {
    if (!r || !bytes) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    uint64_t need = snap_bytes(s);
    if (!blob) {
        *bytes = need;
        return 0;
    }
    if (*bytes < need) return set_err(r, GPUD_E_ARG, "snapshot buffer too small");
    CK(cudaStreamSynchronize(r->stream));
    char *p = (char *)blob;
    SnapHeader h{0x47505544u, 1, s.D, s.T, s.spec.mode, s.wfm_idx >= 0, s.pc, s.hist_len, s.hist_sel,
                 s.comp_hist_len, s.has_last ? 1 : 0, 0, s.rds_count, s.cutoff};
    std::memcpy(p, &h, sizeof h);
    p += sizeof h;
    CK(cudaMemcpy(p, r->d_st + slot, sizeof(ChanState), cudaMemcpyDeviceToHost));
    p += sizeof(ChanState);
    CK(cudaMemcpy(p, r->d_hist + s.hist_off + (size_t)s.hist_sel * s.hcap, (size_t)s.hcap * 8,
                  cudaMemcpyDeviceToHost));
    p += (size_t)s.hcap * 8;
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
    *bytes = need;
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_restore(gpud_runner *r, int slot, const void *blob, uint64_t bytes) {
    if (!r || !blob) return GPUD_E_ARG;
    std::lock_guard<std::mutex> lk(r->mu);
    if (slot < 0 || slot >= r->max_ch || !r->slots[(size_t)slot].active) return set_err(r, GPUD_E_SLOT, "bad slot");
    Slot &s = r->slots[(size_t)slot];
    if (bytes < snap_bytes(s)) return set_err(r, GPUD_E_STATE, "snapshot size mismatch");
    const char *p = (const char *)blob;
    SnapHeader h;
    std::memcpy(&h, p, sizeof h);
    p += sizeof h;
    if (h.magic != 0x47505544u || h.D != s.D || h.T != s.T || h.mode != s.spec.mode || h.wfm != (s.wfm_idx >= 0))
        return set_err(r, GPUD_E_STATE, "snapshot geometry mismatch");
    CK(cudaStreamSynchronize(r->stream));
    CK(cudaMemcpy(r->d_st + slot, p, sizeof(ChanState), cudaMemcpyHostToDevice));
    p += sizeof(ChanState);
    s.hist_sel = 0;
    CK(cudaMemcpy(r->d_hist + s.hist_off, p, (size_t)s.hcap * 8, cudaMemcpyHostToDevice));
    p += (size_t)s.hcap * 8;
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
    s.pc = h.pc;
    s.hist_len = h.hist_len;
    s.comp_hist_len = h.comp_hist_len;
    s.has_last = h.has_last != 0;
    s.rds_count = h.rds_count;
    if (h.cutoff != s.cutoff) {
        int rc = upload_taps(r, slot, 2 * h.cutoff);
        if (rc) return rc;
    }
    return 0;
}

GPUD_API int GPUD_CALL gpud_runner_reset_signal(gpud_runner *r, int64_t signal_id) {
    if (!r) return GPUD_E_ARG;
    auto it = r->by_signal.find(signal_id);
    if (it == r->by_signal.end()) return 0;
    return gpud_runner_retire(r, it->second);
}

GPUD_API int GPUD_CALL gpud_runner_reset_all_signals(gpud_runner *r) {
    if (!r) return GPUD_E_ARG;
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
    // channels admitted through the slot API stay untouched but only the jobs' slots run
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
    int rc;
    {
        std::lock_guard<std::mutex> lk(r->mu);
        rc = run_block(r, iq, n, 0, true);
    }
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

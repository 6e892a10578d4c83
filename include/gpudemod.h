/*
 * gpudemod.h -- C ABI of libgpudemod_kernels.so, the B200 (sm_100a)
 * implementation of Argus SDR's per-signal extraction and demod runner.
 *
 * Part 1 is the drop-in for the reference's `gpudemod_kernels` library: the
 * sixteen `gpud_*` entry points of internal/demod/gpudemod/native/exports.cu
 * with identical C signatures and return codes (0 ok; n<=0 is a no-op that
 * returns 0; positive = cudaError_t; negative = argument error).  The Linux
 * cgo preamble of the reference (internal/demod/gpudemod/gpudemod.go:33-39)
 * binds seven of them; the Windows loader (windows_bridge.go:56-82) resolves
 * all sixteen.
 *
 * Part 2 is the batched / serving runner that replaces the reference's
 * per-signal Go loop (BatchRunner.StreamingExtractGPU ->
 * executeStreamingGPUNativePrepared, streaming_gpu_native_prepare.go:17-108)
 * with one device-resident channel table, one launch sequence per IQ block
 * for all channels (up to three blocks in flight on their own streams,
 * ordered by events), and the demod chain (FM discriminator,
 * AM, SSB, CW, WFM stereo with pilot PLL, RDS baseband) on the device.
 * Its return-code space extends the reference's with new negative codes only
 * (GPUD_E_*), none reused with another meaning.
 *
 * All device pointers are plain CUDA device pointers; host pointers are
 * marked `host`.  No torch types cross this boundary.
 */
#ifndef GPUDEMOD_H
#define GPUDEMOD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define GPUD_API __declspec(dllexport)
#define GPUD_CALL __stdcall
#else
#define GPUD_API __attribute__((visibility("default")))
#define GPUD_CALL
#endif

/* exports.cu:4-12 and gpudemod.go:10 (`gpud_float2`), exports.cu:12
 * (`gpud_stream_handle`). */
typedef struct {
    float x;
    float y;
} gpud_float2;
typedef void *gpud_stream_handle;

/* ======================================================================== */
/* Part 1: reference entry points (native/exports.cu)                        */
/* ======================================================================== */

/* exports.cu:18-25 -- create a CUDA stream; -1 on a null out pointer. */
GPUD_API int GPUD_CALL gpud_stream_create(gpud_stream_handle *out);
/* exports.cu:27-30 */
GPUD_API int GPUD_CALL gpud_stream_destroy(gpud_stream_handle stream);
/* exports.cu:32-35 -- a null stream synchronizes the device. */
GPUD_API int GPUD_CALL gpud_stream_sync(gpud_stream_handle stream);

/* exports.cu:37-76 -- out[i] = in[i] * exp(j*(phase_start + i*phase_inc)). */
GPUD_API int GPUD_CALL gpud_launch_freq_shift_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n,
                                                          double phase_inc, double phase_start,
                                                          gpud_stream_handle stream);
/* exports.cu:78-85 (legacy default stream); also kernels.cu:26-37. */
GPUD_API int GPUD_CALL gpud_launch_freq_shift_cuda(const gpud_float2 *in, gpud_float2 *out, int n,
                                                   double phase_inc, double phase_start);

/* exports.cu:87-112 -- out[i] = arg(conj(in[i]) * in[i+1]), n-1 outputs. */
GPUD_API int GPUD_CALL gpud_launch_fm_discrim_cuda(const gpud_float2 *in, float *out, int n);

/* exports.cu:169-173 -- process-global taps for gpud_launch_fir[_stream]_cuda;
 * -1 unless 1 <= n <= 256. */
GPUD_API int GPUD_CALL gpud_upload_fir_taps_cuda(const float *taps, int n);
/* exports.cu:175-186 -- complex x real FIR, zero history, n outputs. */
GPUD_API int GPUD_CALL gpud_launch_fir_cuda(const gpud_float2 *in, gpud_float2 *out, int n, int num_taps);
/* exports.cu:188-196 */
GPUD_API int GPUD_CALL gpud_launch_fir_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n, int num_taps,
                                                   gpud_stream_handle stream);
/* exports.cu:198-244 -- as gpud_launch_fir_stream_cuda with a device taps
 * pointer per call. */
GPUD_API int GPUD_CALL gpud_launch_fir_v2_stream_cuda(const gpud_float2 *in, gpud_float2 *out, const float *taps,
                                                      int n, int num_taps, gpud_stream_handle stream);

/* exports.cu:246-257 -- out[i] = in[i*factor]. */
GPUD_API int GPUD_CALL gpud_launch_decimate_cuda(const gpud_float2 *in, gpud_float2 *out, int n_out, int factor);
/* exports.cu:259-271 */
GPUD_API int GPUD_CALL gpud_launch_decimate_stream_cuda(const gpud_float2 *in, gpud_float2 *out, int n_out,
                                                        int factor, gpud_stream_handle stream);

/* exports.cu:273-294 -- |in[i]| (no mean removal, as the reference kernel). */
GPUD_API int GPUD_CALL gpud_launch_am_envelope_cuda(const gpud_float2 *in, float *out, int n);

/* exports.cu:296-326 -- Re(in[i] * exp(j*(phase_start + i*phase_inc))). */
GPUD_API int GPUD_CALL gpud_launch_ssb_product_cuda(const gpud_float2 *in, float *out, int n, double phase_inc,
                                                    double phase_start);

/* exports.cu:356-460 -- transitional one-shot polyphase prepare (shift, FIR,
 * decimate, history tail).  Codes -1..-5 as the reference.  Unlike the
 * reference it allocates no device memory: the shifted samples are produced
 * inside the fused kernel. */
GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_prepare_cuda(
    const gpud_float2 *in_new, int n_new, const gpud_float2 *history_in, int history_len, const float *polyphase_taps,
    int polyphase_len, int decim, int num_taps, int phase_count_in, double phase_start, double phase_inc,
    gpud_float2 *out, int *n_out /*host*/, int *phase_count_out /*host*/, double *phase_end_out /*host*/,
    gpud_float2 *history_out);

/* exports.cu:533-631 -- production stateful streaming extractor for one
 * signal.  history_len_io, phase_count_state, phase_state and n_out are host
 * pointers read before and written after the launches; everything else is
 * device memory.  Codes -10..-16 as the reference.  Taps follow the CPU
 * oracle: the layout stride is polyphase_len/decim and taps with
 * p + k*decim >= num_taps are not applied (gpudemod/streaming_host_core.go). */
GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_stateful_cuda(
    const gpud_float2 *in_new, int n_new, gpud_float2 *shifted_new_tmp, const float *polyphase_taps,
    int polyphase_len, int decim, int num_taps, gpud_float2 *history_state, gpud_float2 *history_scratch,
    int history_cap, int *history_len_io /*host*/, int *phase_count_state /*host*/, double *phase_state /*host*/,
    double phase_inc, gpud_float2 *out, int out_cap, int *n_out /*host*/);

/* No counterpart in the reference: an allocation-free variant of
 * gpud_launch_streaming_polyphase_stateful_cuda for callers that cannot
 * allocate device memory around the call (a real-time loop that must not stall
 * on cudaMalloc/cudaFree, which can synchronize the device; a process whose
 * device memory is committed to a fixed budget).  Same arguments minus the two
 * caller scratch buffers, same results and codes (-10 and -11 are checked
 * first), plus GPUD_E_SCRATCH (-32) when n_new > GPUD_NOALLOC_MAX_NEW or
 * history_cap > GPUD_NOALLOC_MAX_HISTORY.  The scratch is one file-scope device
 * array (about 2.1 MB) that every GPU loading the library holds until exit;
 * its device address is resolved on the first call made on each device (make
 * that call before any stream capture) and kept, so after cudaDeviceReset the
 * entry point must not be called on that device again.  All calls share that
 * array: calls that overlap on the GPU race. */
#define GPUD_NOALLOC_MAX_NEW 262144
#define GPUD_NOALLOC_MAX_HISTORY 4096
#define GPUD_E_SCRATCH (-32)
GPUD_API int GPUD_CALL gpud_launch_streaming_polyphase_stateful_noalloc_cuda(
    const gpud_float2 *in_new, int n_new, const float *polyphase_taps, int polyphase_len, int decim, int num_taps,
    gpud_float2 *history_state, int history_cap, int *history_len_io /*host*/, int *phase_count_state /*host*/,
    double *phase_state /*host*/, double phase_inc, gpud_float2 *out, int out_cap, int *n_out /*host*/);

/* ======================================================================== */
/* Part 2: batched / serving runner                                          */
/* ======================================================================== */

/* New error codes (all below the reference's -16). */
#define GPUD_E_ARG (-20)           /* null pointer / bad size */
#define GPUD_E_DECIM (-21)         /* sample_rate % out_rate != 0 (ExactIntegerDecimation) */
#define GPUD_E_TAPS (-22)          /* tap count or polyphase layout beyond the runner's caps */
#define GPUD_E_BUDGET (-23)        /* admission refused: device-memory budget exhausted */
#define GPUD_E_SLOTS (-24)         /* admission refused: channel cap reached */
#define GPUD_E_SLOT (-25)          /* slot id not active */
#define GPUD_E_BLOCK (-26)         /* block larger than the runner's max_block */
#define GPUD_E_TIMEOUT (-27)       /* wait timed out */
#define GPUD_E_CUDA (-28)          /* CUDA call failed (details via gpud_runner_last_error) */
#define GPUD_E_MODE (-29)          /* unknown demod mode */
#define GPUD_E_DEVICE_STATUS (-30) /* a kernel reported a bounds/status failure */
#define GPUD_E_STATE (-31)         /* snapshot blob does not match the slot geometry */
#define GPUD_E_IO (-33)            /* a snapshot file cannot be opened, mapped or written */
#define GPUD_E_FORMAT (-34)        /* not an SDRIQ001 file, or shorter than its header says */

/* Demod modes: DemodType of gpudemod.go:69-76 plus WFM_STEREO and IQ-only. */
enum {
    GPUD_MODE_IQ = 0,
    GPUD_MODE_NFM = 1,
    GPUD_MODE_WFM = 2,
    GPUD_MODE_WFM_STEREO = 3,
    GPUD_MODE_AM = 4,
    GPUD_MODE_USB = 5,
    GPUD_MODE_LSB = 6,
    GPUD_MODE_CW = 7
};

/* channel flags */
#define GPUD_CH_EMIT_IQ 1 /* copy the extracted IQ back every block */
#define GPUD_CH_RDS 2     /* WFM modes: produce the 57 kHz RDS baseband */
/* 48 kHz audio stream (recorder/streamer.go:1408-1470, 569-575): the channel's
 * audio resampled to 48 kHz by the rational polyphase resampler of
 * dsp/resample.go (32 taps per arm, Kaiser beta 6), for WFM modes de-emphasised
 * (one-pole, 50 us unless GPUD_CH_DEEMPH75 / GPUD_CH_NO_DEEMPH) and scaled by
 * 0.35, encoded as s16le PCM.  With this flag only the PCM comes back to the
 * host; the demod-rate audio stays in the device arena. */
#define GPUD_CH_AUDIO48K 4
#define GPUD_CH_DEEMPH75 8    /* 75 us de-emphasis (US/Japan) */
#define GPUD_CH_NO_DEEMPH 16  /* no de-emphasis */
#define GPUD_CH_PCM_F32 32    /* with GPUD_CH_AUDIO48K: float samples (pcm_f32) instead of s16le */
/* WFM_STEREO: the event-recording batch decoder (recorder/wfm_batch_stereo.go:74-155)
 * instead of the streaming one -- locked per block by the pilot-band share of
 * the composite's power, no hysteresis, the discriminator output on both
 * channels when not locked. */
#define GPUD_CH_BATCH_STEREO 64
/* WFM_STEREO: WFMStereo.Demod (demod/fm.go:92-123) -- a free-running 38 kHz
 * carrier instead of the pilot loop, always stereo. */
#define GPUD_CH_FREE_STEREO 128

/* Schedules for gpud_runner_set_schedule. */
#define GPUD_SCHED_BATCHED 0 /* one launch sequence per block for all channels */
#define GPUD_SCHED_PLAIN 1   /* per-signal, synchronous: H2D, launches, D2H per channel */

/* StreamingExtractJob (gpudemod/streaming_types.go:8-15) plus the demod mode. */
typedef struct {
    int64_t signal_id;
    double offset_hz;
    double bandwidth;
    int32_t out_rate;
    int32_t num_taps; /* <= 0 selects 101 (stream_state.go:51-53) */
    uint64_t config_hash;
    int32_t mode;  /* GPUD_MODE_* */
    int32_t flags; /* GPUD_CH_* */
    /* pre-demod decimation (recorder/streamer.go:1098-1146): > 1 puts the
     * stateful 101-tap decimating low-pass of dsp/decimating_fir.go (cutoff
     * 90 kHz for WFM modes, else 0.8 x the demod Nyquist) between the
     * extraction at out_rate and the demodulator, which then runs at
     * out_rate / demod_decim; 0 or 1: none. */
    int32_t demod_decim;
    int32_t reserved;
} gpud_channel_spec;

/* Per-channel result of the last processed block.  The pointers reference
 * the runner's pinned host output arena and stay valid until the next block
 * is submitted.  Mirrors StreamingExtractResult (streaming_types.go:17-24)
 * plus the demod outputs. */
typedef struct {
    int64_t signal_id;
    int32_t rate;        /* extraction output rate */
    int32_t n_iq;        /* NOut */
    int32_t phase_count; /* PhaseCount after the block */
    int32_t history_len; /* HistoryLen after the block */
    double nco_phase;    /* NCO phase after the block, [-pi, pi) */
    int32_t n_audio;     /* floats in audio (2 per frame for WFM_STEREO) */
    int32_t audio_channels;
    int32_t n_rds;    /* complex RDS baseband samples */
    int32_t rds_rate; /* out_rate / floor(out_rate / 19000) */
    int32_t flags;    /* bit0 pilot locked this block, bit1 stereo enabled */
    float coherence;  /* pilot lock margins of this block */
    float pilot_hz;
    float err_avg;
    const gpud_float2 *iq; /* host; NULL unless GPUD_CH_EMIT_IQ */
    const float *audio;    /* host; NULL with GPUD_CH_AUDIO48K (it stays on the device) */
    const gpud_float2 *rds;
    int32_t pll_path;      /* WFM_STEREO: 1 parallel-in-time PLL solver, 2 serial loop */
    int32_t pll_iters;     /* Newton iterations of the last parallel solve */
    const int16_t *pcm;    /* GPUD_CH_AUDIO48K: s16le samples, interleaved per audio channel */
    int32_t n_pcm;         /* int16 samples in pcm (frames x audio_channels) */
    int32_t pcm_rate;      /* 48000 with GPUD_CH_AUDIO48K, else 0 */
    const float *pcm_f32;  /* GPUD_CH_AUDIO48K | GPUD_CH_PCM_F32: float samples (then pcm is NULL) */
} gpud_channel_result;

/* Extraction kernel forms (gpud_autotune_entry.form). */
#define GPUD_FORM_DENSE 0 /* all D phases of a 256-output tile in shared memory (2 <= ceil(T/D) <= 16) */
#define GPUD_FORM_WIDE 1  /* one warp per output, lanes over taps */
#define GPUD_FORM_GROUP 2 /* phase groups of rotated samples; long arms in sliding windows */
#define GPUD_FORM_MOD 3   /* phase groups of raw samples, NCO folded into the taps (ceil(T/D) <= 4) */

/* One autotune override: channels with this applied tap count and decimation
 * use `form`; group_phases (GROUP / MOD) fixes the phases per group, 0 lets
 * the runner size it. */
typedef struct {
    int32_t taps;
    int32_t decim;
    int32_t form;
    int32_t group_phases;
} gpud_autotune_entry;

/* Runner statistics. */
typedef struct {
    uint64_t blocks;
    int32_t active_channels;
    int32_t max_channels;
    uint64_t device_bytes_used;
    uint64_t device_bytes_budget;
    double last_block_ms;   /* device time of the last block (CUDA events) */
    double p50_block_ms;    /* over the last 4096 blocks */
    double p99_block_ms;
    uint64_t kernel_launches; /* kernels launched by the runner since creation */
    int32_t graph_rebuilds;   /* regrowths of the per-block work arrays and output arena (the
                                 launch sequence is not graph-captured; a captured one would be
                                 rebuilt on exactly these) */
    int32_t pad;
    uint64_t last_h2d_bytes;  /* host->device bytes of the last block */
    uint64_t last_d2h_bytes;  /* device->host bytes of the last block */
    double ring_copy_ms;      /* device time of the input-ring copies (blocks from pinned host
                                 memory) completed since the last reset */
    uint64_t ring_copies;     /* their count */
} gpud_runner_stats;

typedef struct gpud_runner gpud_runner;

/* Create a runner for one wideband stream.  max_block: largest IQ block;
 * max_channels: slot count (<= 4096); max_taps: largest FIR (<= 4096);
 * device_mem_budget: bytes the runner may allocate for channel state and
 * buffers (0 = no limit).  Returns 0 or a GPUD_E_* code. */
GPUD_API int GPUD_CALL gpud_runner_create(int sample_rate, int max_block, int max_channels, int max_taps,
                                          uint64_t device_mem_budget, gpud_runner **out);
GPUD_API int GPUD_CALL gpud_runner_destroy(gpud_runner *r);

/* Admit a channel (slot state resident on the device).  Refused with
 * GPUD_E_BUDGET when the channel's device footprint would exceed the budget,
 * GPUD_E_SLOTS at the channel cap.  New channels join at the next block. */
/* Replaces the autotune table (count 0: none; the built-in rule then picks
 * every channel's form).  Entries whose form cannot run their geometry are
 * refused (GPUD_E_ARG).  Applies to channels admitted afterwards; a
 * channel's form depends on its class alone, so (with channel groups off,
 * below) its output is the same alone and in any mix under one table. */
GPUD_API int GPUD_CALL gpud_runner_set_autotune_table(gpud_runner *r, const gpud_autotune_entry *entries, int count);
/* The extraction form, phases per group and group count of an admitted channel. */
GPUD_API int GPUD_CALL gpud_runner_channel_form(gpud_runner *r, int slot, int *form, int *group_phases, int *groups);
/* Channel groups on the tensor cores (no reference counterpart; on by
 * default).  Dense-form channels of one decimation (a multiple of 4), tap
 * count and phase count, at least 4 of them, are extracted together as one
 * TF32x3 GEMM per 128-output tile from output 256 on.  A grouped channel's
 * IQ then depends on whether its class has company in the block (a different
 * summation order, within the 1e-5 parity bar of the ungrouped result); with
 * groups off (enable 0) every channel's output is bit-identical alone and in
 * any mix.  Takes effect at the next block. */
GPUD_API int GPUD_CALL gpud_runner_set_channel_groups(gpud_runner *r, int enable);
GPUD_API int GPUD_CALL gpud_runner_admit(gpud_runner *r, const gpud_channel_spec *spec, int *slot_out);
GPUD_API int GPUD_CALL gpud_runner_retire(gpud_runner *r, int slot);
/* Offset / bandwidth drift: the NCO increment follows the offset with the
 * phase kept; taps are rebuilt when the cutoff changes, history kept
 * (stream_state.go:57-77, Q11). */
GPUD_API int GPUD_CALL gpud_runner_update(gpud_runner *r, int slot, double offset_hz, double bandwidth);
GPUD_API int GPUD_CALL gpud_runner_set_schedule(gpud_runner *r, int schedule);
/* Bytes of device memory one more channel of this spec would take. */
GPUD_API int GPUD_CALL gpud_runner_channel_footprint(gpud_runner *r, const gpud_channel_spec *spec,
                                                     uint64_t *bytes);

/* Process one IQ block through every active channel, synchronously.  iq is a
 * host pointer unless iq_on_device != 0 (pinned host memory is copied
 * straight into the runner's input ring, pageable memory through the
 * runner's pinned staging buffer). */
GPUD_API int GPUD_CALL gpud_runner_process_block(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device);
/* Asynchronous form: enqueue the block and return a ticket; wait returns 0
 * once the outputs of every block up to that ticket are in host memory
 * (GPUD_E_TIMEOUT after timeout_ms).  Three blocks may be in flight: block
 * k+1's extraction / demod / stereo FIR / RDS stages run while block k's pilot
 * PLL and stereo output finish, and their copies overlap; a fourth submit
 * first completes the oldest block.  A block in pinned host memory starts its copy into one of the
 * runner's four input-ring buffers when it is submitted, before that wait.
 * A pinned host iq buffer is read asynchronously and must stay unchanged until
 * its block completed; pageable buffers are copied before submit returns. */
GPUD_API int GPUD_CALL gpud_runner_submit(gpud_runner *r, const gpud_float2 *iq, int n, int iq_on_device,
                                          uint64_t *ticket);
GPUD_API int GPUD_CALL gpud_runner_wait(gpud_runner *r, uint64_t ticket, int timeout_ms);
/* Outputs of the most recently completed block (process_block or wait).  The
 * pointers stay valid until the third submit after that block;
 * GPUD_E_TIMEOUT when blocks are in flight and none has completed since. */
GPUD_API int GPUD_CALL gpud_runner_result(gpud_runner *r, int slot, gpud_channel_result *out);
GPUD_API int GPUD_CALL gpud_runner_stats_get(gpud_runner *r, gpud_runner_stats *out);
/* Clears the block-latency window behind p50_block_ms / p99_block_ms and the
 * ring-copy totals. */
GPUD_API int GPUD_CALL gpud_runner_reset_stats(gpud_runner *r);
/* Stream that joins every submitted block: an event recorded on it after a
 * submit completes when that block and all earlier ones have completed (for
 * external event timing). */
GPUD_API int GPUD_CALL gpud_runner_stream(gpud_runner *r, gpud_stream_handle *out);
GPUD_API const char *GPUD_CALL gpud_runner_last_error(gpud_runner *r);

/* Output placement: with on == 0 the per-block outputs stay in the runner's
 * device arena (no D2H; for consumers that read them on the GPU) and the
 * pointers of gpud_channel_result are device pointers.  Default on. */
GPUD_API int GPUD_CALL gpud_runner_set_host_outputs(gpud_runner *r, int on);

/* Stereo pilot PLL solver: 1 (default) solves each block's loop trajectory in
 * parallel (multiple-shooting Newton over one segment per thread with an
 * associative scan) and falls back per channel to the serial loop when it has
 * not converged within 64 iterations (keeping the consistent prefix of the
 * trajectory and running the serial loop over the rest); a value n > 1 sets
 * that limit to n
 * (at most 4096); 0 runs the serial loop only.  Both compute the same
 * recurrence (recorder/streamer.go:1588-1613). */
GPUD_API int GPUD_CALL gpud_runner_set_pll_solver(gpud_runner *r, int parallel);

/* Per-kernel device time of the last block (CUDA events between the
 * launches on the runner stream); enable with gpud_runner_set_profiling. */
typedef struct {
    char name[24];
    double ms;
} gpud_stage_time;
GPUD_API int GPUD_CALL gpud_runner_set_profiling(gpud_runner *r, int on);
GPUD_API int GPUD_CALL gpud_runner_stage_times(gpud_runner *r, gpud_stage_time *out, int cap, int *count);

/* Slot snapshot / restore (checkpoint across segment rotation; mirrors
 * recorder/streamer.go:1646-1752 captureDSPState/restoreDSPState).  The blob
 * holds the complete device state of the slot; size via *bytes with
 * blob == NULL. */
GPUD_API int GPUD_CALL gpud_runner_snapshot(gpud_runner *r, int slot, void *blob /*host*/, uint64_t *bytes);
GPUD_API int GPUD_CALL gpud_runner_restore(gpud_runner *r, int slot, const void *blob /*host*/, uint64_t bytes);

/* BatchRunner.StreamingExtractGPU (streaming_gpu_stub.go:21-26) semantics:
 * jobs keyed by signal_id; state reset when config_hash changes
 * (stream_state.go:41-47); signals absent from the call are pruned
 * (streaming_gpu_prepare.go:38-43).  Extracted IQ is written back to iq_out
 * (host, capacity iq_out_cap complex samples) job after job; results[i].iq
 * points into it. */
GPUD_API int GPUD_CALL gpud_runner_streaming_extract(gpud_runner *r, const gpud_float2 *iq /*host*/, int n,
                                                     const gpud_channel_spec *jobs, int n_jobs,
                                                     gpud_channel_result *results, gpud_float2 *iq_out /*host*/,
                                                     int iq_out_cap);

/* BatchRunner.ResetSignalState / ResetAllSignalStates (stream_state.go:9-24):
 * forget the streaming state of one signal id (or of all signals admitted
 * through gpud_runner_streaming_extract); the next job for it starts fresh. */
GPUD_API int GPUD_CALL gpud_runner_reset_signal(gpud_runner *r, int64_t signal_id);
GPUD_API int GPUD_CALL gpud_runner_reset_all_signals(gpud_runner *r);

/* gpudemod/streaming_types.go:58-72 StreamingConfigHash. */
GPUD_API uint64_t GPUD_CALL gpud_streaming_config_hash(int64_t signal_id, int out_rate, int num_taps,
                                                       int sample_rate);

/* ------------------------------------------------------------------------
 * Part 3: long-window stereo pilot detector
 * classifier.StereoPilotPresent / estimateWFMPilot (internal/classifier/
 * pll.go:75-131, 170-196) for a batch of FM-multiplex basebands (complex,
 * carrier at DC), each analysed on the device: float64 discriminator,
 * spectrum magnitude at 19 kHz +- 1 kHz in 10 Hz steps (201 bins), pilot
 * present when max / median > threshold.
 * ------------------------------------------------------------------------ */
typedef struct gpud_pilot gpud_pilot;

typedef struct {
    const gpud_float2 *iq; /* device pointer to n samples */
    int32_t n;
    int32_t sample_rate;   /* below 40000: no decision (not present) */
    int32_t window;        /* 1: the last sample_rate/2 samples (StereoPilotPresent); 0: all of them */
    int32_t pad;
} gpud_pilot_job;

typedef struct {
    int32_t present;  /* stereo pilot: median > 0 and ratio > threshold */
    int32_t best_bin; /* 0..200, frequency 18000 + 10 * best_bin Hz (the first maximum) */
    double ratio;     /* largest magnitude / median magnitude */
    double best_hz;
    double median;
} gpud_pilot_result;

/* max_samples bounds n (after the window) of every job. */
GPUD_API int GPUD_CALL gpud_pilot_create(int max_jobs, int max_samples, gpud_pilot **out);
GPUD_API int GPUD_CALL gpud_pilot_destroy(gpud_pilot *p);
/* threshold <= 0 selects the reference's 4.0.  Runs on `stream` (NULL: the
 * legacy default stream) and returns once results (host, count entries) are
 * written. */
GPUD_API int GPUD_CALL gpud_pilot_run(gpud_pilot *p, const gpud_pilot_job *jobs, int count, double threshold,
                                      gpud_stream_handle stream, gpud_pilot_result *results);

/* Number of kernels this library has launched in the process (all entry
 * points). */
GPUD_API uint64_t GPUD_CALL gpud_kernel_launch_count(void);

/* ======================================================================
 * Part 4 -- event-recording batch WFM stereo (no counterpart in the
 * reference's C ABI: it replaces the Go function demodWFMStereoBatchAudio,
 * recorder/wfm_batch_stereo.go:10-72, called by demodWFMStereoHybrid,
 * recorder/wfm_hybrid.go:18-19, for recorded events)
 * ====================================================================== */
typedef struct {
    int32_t n_out;       /* floats written: frames x 2, interleaved L/R */
    int32_t out_rate;    /* 48000 */
    int32_t demod_rate;  /* sample_rate / round(sample_rate / 192000) */
    int32_t locked;      /* the batch decoder's lock decision */
} gpud_batch_audio_result;

/* One capture, stateless: shift by offset_hz, 101-tap low-pass, decimate to
 * ~192 kS/s, discriminator, batch stereo decode (duplicated mono when not
 * locked), 48 kHz resample, de-emphasis (deemph_us, 0: none), x0.35.  iq is a
 * host pointer unless iq_on_device.  Returns 0, GPUD_E_ARG (bad argument,
 * out_cap too small) or a runner error. */
GPUD_API int GPUD_CALL gpud_wfm_batch_audio(const gpud_float2 *iq, int n, int iq_on_device, int sample_rate,
                                            double offset_hz, double bandwidth, double deemph_us, float *out,
                                            int out_cap, gpud_batch_audio_result *res);

typedef struct {
    int32_t n_out;       /* floats written (frames x channels) */
    int32_t channels;    /* 2 for WFM_STEREO, else 1 */
    int32_t out_rate;    /* demod rate / round(demod rate / 48000) when above 48 kHz, else the demod rate */
    int32_t demod_rate;  /* sample_rate / round(sample_rate / mode's demod rate) */
} gpud_segment_audio_result;

/* One segment, stateless, any GPUD_MODE_* but IQ (no counterpart in the
 * reference's C ABI: it replaces the Go function demodAudioCPU,
 * recorder/cpu_audio.go:10-75, behind the live /api/demod path,
 * recorder/demod_live.go:40-70, and event recordings, recorder/demod.go:
 * 21-60): shift, 101-tap low-pass, decimation to ~48 kHz (~192 kHz for WFM),
 * the mode's demodulator (WFM_STEREO: free-running 38 kHz stereo), and above
 * 48 kHz a 63-tap anti-alias filter and integer decimation. */
GPUD_API int GPUD_CALL gpud_demod_audio_segment(int mode, const gpud_float2 *iq, int n, int iq_on_device,
                                                int sample_rate, double offset_hz, double bandwidth, float *out,
                                                int out_cap, gpud_segment_audio_result *res);

/* ======================================================================
 * Part 5 -- SDRIQ001 snapshots (internal/iqfile/iqfile.go): write, mapped
 * read and a looping replay source feeding host or device blocks
 * ====================================================================== */
typedef struct gpud_iqfile gpud_iqfile;
typedef struct {
    int64_t sample_rate;
    double center_hz;
    int64_t samples;
} gpud_iqfile_meta;

/* iqfile.Write (iqfile.go:33-59): magic, rate, centre, count, cf32 samples. */
GPUD_API int GPUD_CALL gpud_iqfile_write(const char *path, const gpud_float2 *iq, int64_t n, int64_t sample_rate,
                                         double center_hz);
/* iqfile.Read / NewSource (iqfile.go:62-116): GPUD_E_FORMAT on a bad magic or
 * a file shorter than its header's count, GPUD_E_IO when it cannot be opened. */
GPUD_API int GPUD_CALL gpud_iqfile_open(const char *path, gpud_iqfile **out, gpud_iqfile_meta *meta);
GPUD_API void GPUD_CALL gpud_iqfile_close(gpud_iqfile *f);
/* Source.ReadIQ (iqfile.go:128-148): the next n samples, looping at the end
 * (zeros for an empty file), into host memory or, with dst_on_device, device
 * memory on `stream` (a cudaStream_t; NULL: the legacy default stream). */
GPUD_API int GPUD_CALL gpud_iqfile_read(gpud_iqfile *f, gpud_float2 *dst, int64_t n, int dst_on_device,
                                        void *stream);
GPUD_API int GPUD_CALL gpud_iqfile_seek(gpud_iqfile *f, int64_t pos);
GPUD_API int64_t GPUD_CALL gpud_iqfile_tell(const gpud_iqfile *f);

/* ======================================================================
 * Part 6 -- RDS decoder for a batch of stations (internal/rds/rds.go:78-636,
 * rds.Decoder.Decode, called per station and RDS window by
 * cmd/sdrd/pipeline_runtime.go:1137): symbol timing, Costas loop,
 * differential decoding, block sync with one-bit correction and flywheel,
 * PI / PS (group 0A) / RT (group 2A).  State per station stays on the device.
 * ====================================================================== */
typedef struct gpud_rds_decoder gpud_rds_decoder;

typedef struct {
    const gpud_float2 *samples; /* device pointer: RDS baseband (RDSBasebandComplex output) */
    int32_t n;                  /* below 104: ignored, as the reference does */
    int32_t sample_rate;
    int32_t station;            /* 0 .. max_stations-1, distinct within one run */
    int32_t pad;
} gpud_rds_job;

typedef struct {
    int32_t groups;        /* groups applied by this call */
    int32_t groups_total;  /* over all calls of the station */
    int32_t status;        /* 0; 1: the timing loop stopped advancing (input far out of range) */
    uint16_t pi;
    uint16_t pad;
    char ps[9];            /* Program Service name, trailing spaces trimmed */
    char rt[65];           /* RadioText */
    char pad2[2];
} gpud_rds_result;

/* max_samples bounds n of every job. */
GPUD_API int GPUD_CALL gpud_rds_decoder_create(int max_stations, int max_samples, gpud_rds_decoder **out);
GPUD_API int GPUD_CALL gpud_rds_decoder_destroy(gpud_rds_decoder *r);
/* A new decoder state for the station (rds.Decoder{} of a newly found station). */
GPUD_API int GPUD_CALL gpud_rds_decoder_reset(gpud_rds_decoder *r, int station);
/* One Decode call per job, all jobs in one launch on `stream`; returns once
 * results (host, count entries) are written. */
GPUD_API int GPUD_CALL gpud_rds_decode_run(gpud_rds_decoder *r, const gpud_rds_job *jobs, int count,
                                           gpud_stream_handle stream, gpud_rds_result *results);

/* ======================================================================
 * Part 7 -- surveillance spectrum (internal/fft/fft.go:19-55 Spectrum,
 * internal/fft/welch.go:15-66 WelchPSD, called per frame by
 * cmd/sdrd/pipeline_runtime.go:294-341; cuFFT or gonum there): float64
 * transforms in shared memory, power-of-two sizes up to 8192, fftshifted dB.
 * ====================================================================== */
typedef struct gpud_spectrum gpud_spectrum;

/* max_fft: a power of two <= 8192; max_segments: Welch segments per call. */
GPUD_API int GPUD_CALL gpud_spectrum_create(int max_fft, int max_segments, gpud_spectrum **out);
GPUD_API int GPUD_CALL gpud_spectrum_destroy(gpud_spectrum *s);
/* Spectrum(iq, Hann(n) when hann, else none): n dB values, 20 log10(|X|/n + 1e-12),
 * DC at index n/2.  iq: device pointer. */
GPUD_API int GPUD_CALL gpud_spectrum_single(gpud_spectrum *s, const gpud_float2 *iq, int n, int hann,
                                            gpud_stream_handle stream, double *out_db);
/* WelchPSD(iq, seg_size, overlap, Hann when hann): segments at
 * step = int(seg_size (1 - overlap)), overlap clamped to [0, 0.95], mean power,
 * 10 log10(. + 1e-24), DC at seg_size/2; *n_out = seg_size.  Fewer samples than
 * one segment: Spectrum of the whole vector without window (*n_out = n). */
GPUD_API int GPUD_CALL gpud_spectrum_welch(gpud_spectrum *s, const gpud_float2 *iq, int64_t n, int seg_size,
                                           double overlap, int hann, gpud_stream_handle stream, double *out_db,
                                           int *n_out);

/* ======================================================================
 * Part 8 -- the single-signal Engine's front end on the device
 * (internal/demod/gpudemod/gpudemod.go:325-427).  The reference runs these
 * stages with its CPU dsp functions; these entry points give the same
 * results on the device so Engine.ShiftFilterDecimate / Engine.Demod and the
 * legacy batch paths need no CPU stage.
 * ====================================================================== */

/* dsp.LowpassFIR (internal/dsp/fir.go:6-28): Hann-windowed sinc taps of
 * odd length (taps | 1) into out (host, out_cap entries).  Returns the length
 * or GPUD_E_ARG. */
GPUD_API int GPUD_CALL gpud_lowpass_fir(double cutoff_hz, int sample_rate, int taps, double *out, int out_cap);

/* dsp.Decimate(dsp.ApplyFIR(dsp.FreqShift(in, sample_rate, offset_hz), taps), decim)
 * (gpudemod.go:336-350; dsp/freqshift.go:6-23, dsp/fir.go:31-95): the shift's
 * phase restarts at 0 and is incremented before use by the reference's exact
 * sequence of float64 additions; the FIR (num_taps <= 4096 float64 taps,
 * device) has zero history and a float64 accumulator and is evaluated at the
 * kept samples only; *n_out = ceil(n / decim) samples, every decim-th from
 * index 0.  in, shifted_tmp (n samples), out (out_cap) and taps are device
 * pointers; n_out is a host pointer.  Returns 0, GPUD_E_ARG or GPUD_E_CUDA;
 * n <= 0 is a no-op. */
GPUD_API int GPUD_CALL gpud_shift_fir_decimate_cuda(const gpud_float2 *in, int n, int sample_rate, double offset_hz,
                                                    const double *taps, int num_taps, int decim,
                                                    gpud_float2 *shifted_tmp, gpud_float2 *out, int out_cap,
                                                    int *n_out /*host*/, gpud_stream_handle stream);

#ifdef __cplusplus
}
#endif

#endif /* GPUDEMOD_H */

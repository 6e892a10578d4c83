/*
 * oracle.c -- CPU restatement of the Argus SDR `gpudemod` extraction and demod
 * path, written in plain C99.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only as
 * the checker or the timed CPU baseline.  The product (libgpudemod_kernels.so)
 * never links, loads or calls it.
 *
 * Every function cites the reference Go source it restates (paths are relative
 * to the svabi79/argus-sdr tree).  The reference is Go 1.23; the arithmetic
 * conventions that matter for parity are reproduced explicitly:
 *
 *   - complex64 * complex64 in Go is evaluated in float64 and rounded once per
 *     component to float32 (the gc compiler widens complex64 products to
 *     minimise cancellation); complex64 + complex64 is a float32 add per
 *     component.  cmul_go() and cadd_go() below restate that.
 *   - float32(x) conversions round-to-nearest; build with -ffp-contract=off so
 *     that no expression is fused into an FMA the Go code does not perform.
 *   - Go's math.Sin/Cos/Atan2/Hypot/Exp are replaced by glibc libm.  The two can
 *     differ by an ulp in float64; every value that crosses into float32 hides
 *     that, and no reference test pins raw stdlib values (parity at that
 *     boundary is unpinned, stated in the module header of the tests).
 *
 * Pinning: the restatement is checked against every known-answer test the
 * reference holds for this path (polyphase layout, exact decimation,
 * monolithic == chunked, direct == polyphase, RDS baseband chunked == plain,
 * stereo lock/separation/no-false-lock properties) -- see tests/test_oracle.py.
 * The reference itself cannot run here (Go toolchain absent), so raw sample
 * values are pinned only through those KATs.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    float re, im;
} cf32;

#define OR_PI 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Go arithmetic helpers                                                     */
/* ------------------------------------------------------------------------ */

static inline cf32 cmul_go(cf32 a, cf32 b) {
    cf32 r;
    r.re = (float)((double)a.re * (double)b.re - (double)a.im * (double)b.im);
    r.im = (float)((double)a.re * (double)b.im + (double)a.im * (double)b.re);
    return r;
}

static inline cf32 cadd_go(cf32 a, cf32 b) {
    cf32 r;
    r.re = a.re + b.re;
    r.im = a.im + b.im;
    return r;
}

/* ------------------------------------------------------------------------ */
/* internal/dsp/fir.go:6-28  LowpassFIR                                      */
/* ------------------------------------------------------------------------ */

/* Returns the tap count actually produced (taps bumped to odd).  `out` must
 * hold taps|1 values. */
int or_lowpass_fir(double cutoff_hz, int sample_rate, int taps, double *out) {
    if (taps % 2 == 0) taps++;
    for (int i = 0; i < taps; i++) out[i] = 0.0;
    double fc = cutoff_hz / (double)sample_rate;
    if (fc <= 0) return taps;
    double m = (double)(taps - 1) / 2.0;
    for (int n = 0; n < taps; n++) {
        double x = (double)n - m;
        double sinc;
        if (x == 0) {
            sinc = 2 * fc;
        } else {
            sinc = sin(2 * OR_PI * fc * x) / (OR_PI * x);
        }
        double w = 0.5 * (1 - cos(2 * OR_PI * (double)n / (double)(taps - 1)));
        out[n] = sinc * w;
    }
    return taps;
}

/* gpudemod/cpu_oracle.go:155-163  ExactIntegerDecimation: D or -1. */
int or_exact_decim(int sample_rate, int out_rate) {
    if (sample_rate <= 0 || out_rate <= 0) return -1;
    if (sample_rate % out_rate != 0) return -1;
    return sample_rate / out_rate;
}

/* gpudemod/polyphase.go:22-28 PolyphasePhaseLen */
int or_polyphase_phase_len(int base_len, int decim) {
    if (decim <= 0 || base_len <= 0) return 0;
    return (base_len + decim - 1) / decim;
}

/* gpudemod/polyphase.go:6-20 BuildPolyphaseTapsPhaseMajor.  Returns D*L. */
int or_build_polyphase(const float *base, int n, int decim, float *out) {
    if (decim <= 0 || n == 0) return 0;
    int L = (n + decim - 1) / decim;
    for (int p = 0; p < decim; p++) {
        for (int k = 0; k < L; k++) {
            int src = p + k * decim;
            out[p * L + k] = src < n ? base[src] : 0.0f;
        }
    }
    return decim * L;
}

/* gpudemod/streaming_types.go:58-72  StreamingConfigHash: FNV-1a 64 over
 * "sig=%d|out=%d|taps=%d|sr=%d" (offset and bandwidth deliberately excluded). */
uint64_t or_config_hash(int64_t signal_id, int out_rate, int num_taps, int sample_rate) {
    char buf[160];
    int len = snprintf(buf, sizeof buf, "sig=%lld|out=%d|taps=%d|sr=%d", (long long)signal_id, out_rate,
                       num_taps, sample_rate);
    uint64_t h = 14695981039346656037ULL;
    for (int i = 0; i < len; i++) {
        h ^= (uint8_t)buf[i];
        h *= 1099511628211ULL;
    }
    return h;
}

/* ------------------------------------------------------------------------ */
/* gpudemod/streaming_host_core.go:5-64  runStreamingPolyphaseHostCore       */
/* ------------------------------------------------------------------------ */

/*
 * The NCO phase is used before it is incremented and wrapped once into
 * [-pi, pi).  The rotator is computed in float64 and rounded to complex64; the
 * product with the input is a complex64 product.  Outputs are accumulated in
 * complex64 in phase-major order (p outer, k inner), skipping taps that are zero
 * and samples older than the retained history.
 *
 * hist_io holds up to num_taps-1 shifted samples (oldest first) and is updated
 * in place; *hist_len_io, *phase_io and *pc_io carry the rest of the state.
 * Returns the number of outputs written to out.
 */
int or_extract_host_core(const cf32 *in, int n, int sample_rate, double offset_hz, double *phase_io,
                         int *pc_io, int num_taps, int decim, cf32 *hist_io, int *hist_len_io,
                         const float *poly, int poly_len, cf32 *out) {
    int D = decim > 1 ? decim : 1;
    int phase_len = or_polyphase_phase_len(poly_len / D * D, decim);
    if (phase_len == 0) phase_len = or_polyphase_phase_len(poly_len, decim);
    double phase = *phase_io;
    int pc = *pc_io;
    int keep = num_taps - 1;
    int hlen = *hist_len_io;
    /* work buffer: history followed by every new shifted sample.  `start` is the
     * index of the oldest retained sample; trimming just advances it. */
    cf32 *buf = (cf32 *)malloc(sizeof(cf32) * (size_t)(hlen + n + 1));
    memcpy(buf, hist_io, sizeof(cf32) * (size_t)hlen);
    int start = 0, end = hlen; /* retained window is buf[start:end] */
    double inc = -2.0 * OR_PI * offset_hz / (double)sample_rate;
    int nout = 0;
    for (int i = 0; i < n; i++) {
        cf32 rot;
        rot.re = (float)cos(phase);
        rot.im = (float)sin(phase);
        cf32 s = cmul_go(in[i], rot);
        buf[end++] = s;
        pc++;
        if (pc == decim) {
            cf32 y = {0.0f, 0.0f};
            int len = end - start;
            for (int p = 0; p < decim; p++) {
                for (int k = 0; k < phase_len; k++) {
                    int idx_tap = p * phase_len + k;
                    if (idx_tap >= poly_len) continue;
                    float tap = poly[idx_tap];
                    if (tap == 0) continue;
                    int src_back = p + k * decim;
                    int idx = len - 1 - src_back;
                    if (idx < 0) continue;
                    cf32 t = {tap, 0.0f};
                    y = cadd_go(y, cmul_go(t, buf[start + idx]));
                }
            }
            out[nout++] = y;
            pc = 0;
        }
        if (end - start > keep) start = end - (keep > 0 ? keep : 0);
        phase += inc;
        if (phase >= OR_PI) {
            phase -= 2 * OR_PI;
        } else if (phase < -OR_PI) {
            phase += 2 * OR_PI;
        }
    }
    int new_len = end - start;
    if (new_len > keep) new_len = keep > 0 ? keep : 0;
    memcpy(hist_io, buf + end - new_len, sizeof(cf32) * (size_t)new_len);
    *hist_len_io = new_len;
    *phase_io = phase;
    *pc_io = pc;
    free(buf);
    return nout;
}

/* gpudemod/cpu_oracle.go:32-75  CPUOracleExtract (direct form; NumTaps taps of
 * BaseTaps, samples older than the history read as zero). */
int or_extract_direct(const cf32 *in, int n, double phase_inc, double *phase_io, int *pc_io, int num_taps,
                      int decim, cf32 *hist_io, int *hist_len_io, const float *base_taps, cf32 *out) {
    double phase = *phase_io;
    int pc = *pc_io;
    int keep = num_taps - 1;
    int hlen = *hist_len_io;
    cf32 *buf = (cf32 *)malloc(sizeof(cf32) * (size_t)(hlen + n + 1));
    memcpy(buf, hist_io, sizeof(cf32) * (size_t)hlen);
    int start = 0, end = hlen;
    int nout = 0;
    for (int i = 0; i < n; i++) {
        cf32 rot;
        rot.re = (float)cos(phase);
        rot.im = (float)sin(phase);
        buf[end++] = cmul_go(in[i], rot);
        pc++;
        if (pc == decim) {
            cf32 y = {0.0f, 0.0f};
            int len = end - start;
            for (int k = 0; k < num_taps; k++) {
                int idx = len - 1 - k;
                cf32 smp = {0.0f, 0.0f};
                if (idx >= 0) smp = buf[start + idx];
                cf32 t = {base_taps[k], 0.0f};
                y = cadd_go(y, cmul_go(t, smp));
            }
            out[nout++] = y;
            pc = 0;
        }
        if (end - start > keep) start = end - (keep > 0 ? keep : 0);
        phase += phase_inc;
        if (phase >= OR_PI) {
            phase -= 2 * OR_PI;
        } else if (phase < -OR_PI) {
            phase += 2 * OR_PI;
        }
    }
    int new_len = end - start;
    if (new_len > keep) new_len = keep > 0 ? keep : 0;
    memcpy(hist_io, buf + end - new_len, sizeof(cf32) * (size_t)new_len);
    *hist_len_io = new_len;
    *phase_io = phase;
    *pc_io = pc;
    free(buf);
    return nout;
}

/* Polyphase variant of the direct form: gpudemod/cpu_oracle.go:77-130
 * CPUOracleExtractPolyphase (phase_inc given directly, layout from base). */
int or_extract_polyphase(const cf32 *in, int n, double phase_inc, double *phase_io, int *pc_io, int num_taps,
                         int decim, cf32 *hist_io, int *hist_len_io, const float *base_taps, int base_len,
                         cf32 *out) {
    int L = or_polyphase_phase_len(base_len, decim);
    float *poly = (float *)calloc((size_t)(decim * L + 1), sizeof(float));
    or_build_polyphase(base_taps, base_len, decim, poly);
    double phase = *phase_io;
    int pc = *pc_io;
    int keep = num_taps - 1;
    int hlen = *hist_len_io;
    cf32 *buf = (cf32 *)malloc(sizeof(cf32) * (size_t)(hlen + n + 1));
    memcpy(buf, hist_io, sizeof(cf32) * (size_t)hlen);
    int start = 0, end = hlen;
    int nout = 0;
    for (int i = 0; i < n; i++) {
        cf32 rot;
        rot.re = (float)cos(phase);
        rot.im = (float)sin(phase);
        buf[end++] = cmul_go(in[i], rot);
        pc++;
        if (pc == decim) {
            cf32 y = {0.0f, 0.0f};
            int len = end - start;
            for (int p = 0; p < decim; p++) {
                for (int k = 0; k < L; k++) {
                    float tap = poly[p * L + k];
                    if (tap == 0) continue;
                    int idx = len - 1 - (p + k * decim);
                    if (idx < 0) continue;
                    cf32 t = {tap, 0.0f};
                    y = cadd_go(y, cmul_go(t, buf[start + idx]));
                }
            }
            out[nout++] = y;
            pc = 0;
        }
        if (end - start > keep) start = end - (keep > 0 ? keep : 0);
        phase += phase_inc;
        if (phase >= OR_PI) {
            phase -= 2 * OR_PI;
        } else if (phase < -OR_PI) {
            phase += 2 * OR_PI;
        }
    }
    int new_len = end - start;
    if (new_len > keep) new_len = keep > 0 ? keep : 0;
    memcpy(hist_io, buf + end - new_len, sizeof(cf32) * (size_t)new_len);
    *hist_len_io = new_len;
    *phase_io = phase;
    *pc_io = pc;
    free(buf);
    free(poly);
    return nout;
}

/* ------------------------------------------------------------------------ */
/* Demodulators                                                              */
/* ------------------------------------------------------------------------ */

/* internal/demod/fm.go:179-196  fmDiscrimInto: float64 cross/dot products of
 * float32 inputs, float64 atan2, float32 output.  Returns n-1 (or 0). */
int or_fm_discrim(const cf32 *iq, int n, float *out) {
    if (n < 2) return 0;
    for (int i = 1; i < n; i++) {
        cf32 p = iq[i - 1], c = iq[i];
        double num = (double)p.re * (double)c.im - (double)p.im * (double)c.re;
        double den = (double)p.re * (double)c.re + (double)p.im * (double)c.im;
        out[i - 1] = (float)atan2(num, den);
    }
    return n - 1;
}

/* internal/demod/am.go:11-27  AM.Demod: hypot minus the per-call mean. */
int or_am_demod(const cf32 *iq, int n, float *out) {
    if (n == 0) return 0;
    double mean = 0;
    for (int i = 0; i < n; i++) {
        double mag = hypot((double)iq[i].re, (double)iq[i].im);
        mean += mag;
        out[i] = (float)mag;
    }
    mean /= (double)n;
    float fm = (float)mean;
    for (int i = 0; i < n; i++) out[i] = out[i] - fm;
    return n;
}

/* internal/demod/ssb.go:19-39  product detector, BFO +-700 Hz, phase
 * incremented before use and restarted at 0 on every call. */
int or_ssb_demod(const cf32 *iq, int n, int sample_rate, int usb, float *out) {
    if (n == 0) return 0;
    double bfo = usb ? 700.0 : -700.0;
    double phase = 0.0;
    double inc = 2 * OR_PI * bfo / (double)sample_rate;
    for (int i = 0; i < n; i++) {
        phase += inc;
        double c = cos(phase), s = sin(phase);
        out[i] = (float)((double)iq[i].re * c - (double)iq[i].im * s);
    }
    return n;
}

/* internal/demod/cw.go:11-26  Re(v) * cos(700 Hz BFO), pre-increment, restart
 * per call. */
int or_cw_demod(const cf32 *iq, int n, int sample_rate, float *out) {
    if (n == 0) return 0;
    double phase = 0.0;
    double inc = 2 * OR_PI * 700.0 / (double)sample_rate;
    for (int i = 0; i < n; i++) {
        phase += inc;
        out[i] = (float)((double)iq[i].re * cos(phase));
    }
    return n;
}

/* ------------------------------------------------------------------------ */
/* internal/dsp/fir_stateful.go:6-54  StatefulFIRReal                        */
/* ------------------------------------------------------------------------ */

/* The Go filter shifts a float64 delay line by one per sample (delay[0] is the
 * newest) and accumulates sum_k delay[k]*taps[k] for k = 0..n-1 in float64.
 * A circular buffer gives the same values in the same order. */
typedef struct {
    int n;
    double taps[1025];
    double delay[1025]; /* circular; delay[pos] is the newest */
    int pos;
} or_fir_real;

static void fir_real_init(or_fir_real *f, const double *taps, int n) {
    f->n = n;
    memcpy(f->taps, taps, sizeof(double) * (size_t)n);
    memset(f->delay, 0, sizeof f->delay);
    f->pos = 0;
}

static void fir_real_process(or_fir_real *f, const float *x, int len, float *out) {
    int n = f->n;
    if (len == 0 || n == 0) return;
    for (int i = 0; i < len; i++) {
        f->pos = (f->pos + n - 1) % n;
        f->delay[f->pos] = (double)x[i];
        double acc = 0;
        int p = f->pos;
        for (int k = 0; k < n; k++) {
            acc += f->delay[p] * f->taps[k];
            p++;
            if (p == n) p = 0;
        }
        out[i] = (float)acc;
    }
}

/* ------------------------------------------------------------------------ */
/* internal/recorder/streamer.go:1496-1644  stereoDecodeStateful + PLL       */
/* ------------------------------------------------------------------------ */

typedef struct {
    int rate; /* 0 until the filters are built */
    or_fir_real lpf, bphi, bplo, lrlpf, plhi, pllo;
    double phase, freq, alpha, beta, err_avg, i_state, q_state, lp_alpha;
    /* lock bookkeeping of the last call (streamer.go:1632-1635) */
    double coherence, freq_hz;
    int locked;
    /* hysteresis (streamer.go:1363-1400) and the mono fallback LPF
     * (streamer.go:1511-1520) */
    int on_count, off_count, enabled;
    int audio_rate;
    or_fir_real audio_lpf;
} or_stereo;

/* streamer.go:1496-1509 pllCoefficients */
void or_pll_coefficients(double loop_bw, double damping, int sample_rate, double *alpha, double *beta) {
    if (sample_rate <= 0 || loop_bw <= 0) {
        *alpha = 0;
        *beta = 0;
        return;
    }
    double bl = loop_bw / (double)sample_rate;
    double theta = bl / (damping + 0.25 / damping);
    double d = 1 + 2 * damping * theta + theta * theta;
    *alpha = (4 * damping * theta) / d;
    *beta = (4 * theta * theta) / d;
}

size_t or_stereo_size(void) { return sizeof(or_stereo); }

void or_stereo_init(or_stereo *s) { memset(s, 0, sizeof *s); }

static void lpf101(double cutoff, int fs, double *taps) { or_lowpass_fir(cutoff, fs, 101, taps); }

/* Returns n; writes 2n interleaved L/R floats; *locked receives the per-call
 * lock decision.  lr_out (n floats, may be NULL) receives the L-R product
 * before its 15 kHz filter, pilot_out the pilot band signal (diagnostics). */
int or_stereo_decode(or_stereo *s, const float *mono, int n, int sample_rate, float *out, int *locked) {
    if (n == 0 || sample_rate <= 0) {
        *locked = 0;
        return 0;
    }
    if (s->rate != sample_rate) {
        double t[101];
        lpf101(15000, sample_rate, t);
        fir_real_init(&s->lpf, t, 101);
        fir_real_init(&s->lrlpf, t, 101);
        lpf101(53000, sample_rate, t);
        fir_real_init(&s->bphi, t, 101);
        lpf101(23000, sample_rate, t);
        fir_real_init(&s->bplo, t, 101);
        lpf101(21000, sample_rate, t);
        fir_real_init(&s->plhi, t, 101);
        lpf101(17000, sample_rate, t);
        fir_real_init(&s->pllo, t, 101);
        s->rate = sample_rate;
        s->phase = 0;
        s->freq = 2 * OR_PI * 19000 / (double)sample_rate;
        or_pll_coefficients(50, 0.707, sample_rate, &s->alpha, &s->beta);
        s->err_avg = 0;
        s->i_state = 0;
        s->q_state = 0;
        s->lp_alpha = 1 - exp(-2 * OR_PI * 200 / (double)sample_rate);
    }
    float *lpr = (float *)malloc(sizeof(float) * (size_t)n * 5);
    float *bpf = lpr + n, *lr = lpr + 2 * n, *w1 = lpr + 3 * n, *w2 = lpr + 4 * n;
    fir_real_process(&s->lpf, mono, n, lpr);
    fir_real_process(&s->bphi, mono, n, w1);
    fir_real_process(&s->bplo, mono, n, w2);
    for (int i = 0; i < n; i++) bpf[i] = w1[i] - w2[i];
    fir_real_process(&s->plhi, mono, n, w1);
    fir_real_process(&s->pllo, mono, n, w2);
    for (int i = 0; i < n; i++) w1[i] = w1[i] - w2[i];
    const float *pilot = w1;

    double phase = s->phase, freq = s->freq, alpha = s->alpha, beta = s->beta;
    double is = s->i_state, qs = s->q_state, lpa = s->lp_alpha;
    double min_f = 2 * OR_PI * 17000 / (double)sample_rate;
    double max_f = 2 * OR_PI * 21000 / (double)sample_rate;
    double pilot_power = 0, err_sum = 0;
    for (int i = 0; i < n; i++) {
        double p = (double)pilot[i];
        double sp = sin(phase), cp = cos(phase);
        double imix = p * cp;
        double qmix = p * -sp;
        is += lpa * (imix - is);
        qs += lpa * (qmix - qs);
        double err = atan2(qs, is);
        freq += beta * err;
        if (freq < min_f) {
            freq = min_f;
        } else if (freq > max_f) {
            freq = max_f;
        }
        phase += freq + alpha * err;
        if (phase > 2 * OR_PI) {
            phase -= 2 * OR_PI;
        } else if (phase < 0) {
            phase += 2 * OR_PI;
        }
        pilot_power += p * p;
        err_sum += fabs(err);
        lr[i] = bpf[i] * (float)(2 * sin(2 * phase));
    }
    s->phase = phase;
    s->freq = freq;
    s->i_state = is;
    s->q_state = qs;
    double block_err = err_sum / (double)n;
    s->err_avg = 0.9 * s->err_avg + 0.1 * block_err;
    fir_real_process(&s->lrlpf, lr, n, lr);
    double coherence = 0;
    if (pilot_power > 1e-12) coherence = (is * is + qs * qs) * (double)n / pilot_power;
    double freq_hz = s->freq * (double)sample_rate / (2 * OR_PI);
    int lk = coherence > 0.15 && fabs(freq_hz - 19000) < 250 && s->err_avg < 0.35;
    s->coherence = coherence;
    s->freq_hz = freq_hz;
    s->locked = lk;
    for (int i = 0; i < n; i++) {
        out[2 * i] = 0.5f * (lpr[i] + lr[i]);
        out[2 * i + 1] = 0.5f * (lpr[i] - lr[i]);
    }
    free(lpr);
    *locked = lk;
    return n;
}

/* streamer.go:1511-1520 wfmAudioFilter: 15 kHz stateful LPF, rebuilt when the
 * rate changes. */
static void wfm_audio_filter(or_stereo *s, const float *x, int n, int rate, float *out) {
    if (s->audio_rate != rate) {
        double t[101];
        lpf101(15000, rate, t);
        fir_real_init(&s->audio_lpf, t, 101);
        s->audio_rate = rate;
    }
    fir_real_process(&s->audio_lpf, x, n, out);
}

/* streamer.go:1355-1404 WFM_STEREO branch of processSnippet: stereo decode,
 * lock hysteresis (on after 4 locked calls, off after 10 unlocked), and the
 * dual-mono 15 kHz fallback.  Writes 2n floats.  Returns n. */
int or_wfm_stereo_stage(or_stereo *s, const float *mono, int n, int rate, float *out, int *locked,
                        int *enabled) {
    if (n == 0) {
        *locked = 0;
        *enabled = s->enabled;
        return 0;
    }
    float *st = (float *)malloc(sizeof(float) * 2 * (size_t)n);
    int lk = 0;
    or_stereo_decode(s, mono, n, rate, st, &lk);
    if (lk) {
        s->on_count++;
        s->off_count = 0;
        if (s->on_count >= 4) s->enabled = 1;
    } else {
        s->on_count = 0;
        s->off_count++;
        if (s->off_count >= 10) s->enabled = 0;
    }
    if (s->enabled) {
        memcpy(out, st, sizeof(float) * 2 * (size_t)n);
    } else {
        float *m = (float *)malloc(sizeof(float) * (size_t)n);
        wfm_audio_filter(s, mono, n, rate, m);
        for (int i = 0; i < n; i++) {
            out[2 * i] = m[i];
            out[2 * i + 1] = m[i];
        }
        free(m);
    }
    free(st);
    *locked = lk;
    *enabled = s->enabled;
    return n;
}

/* Plain WFM (mono) branch: streamer.go:1401-1404. */
int or_wfm_mono_stage(or_stereo *s, const float *mono, int n, int rate, float *out) {
    if (n == 0) return 0;
    wfm_audio_filter(s, mono, n, rate, out);
    return n;
}

void or_stereo_margins(const or_stereo *s, double *coherence, double *freq_hz, double *err_avg) {
    *coherence = s->coherence;
    *freq_hz = s->freq_hz;
    *err_avg = s->err_avg;
}

/* ------------------------------------------------------------------------ */
/* RDS baseband: internal/demod/fm.go:143-163 and 234-271, with              */
/* dsp/freqshift.go:6-23, dsp/fir.go:31-95                                    */
/* ------------------------------------------------------------------------ */

/* Monolithic RDSBasebandComplex over an IQ vector.  Returns the number of
 * outputs; *rate_out gets fs / Dr. */
int or_rds_baseband_complex(const cf32 *iq, int n, int sample_rate, cf32 *out, int *rate_out) {
    if (n < 2 || sample_rate <= 0) {
        *rate_out = 0;
        return 0;
    }
    int m = n - 1;
    float *disc = (float *)malloc(sizeof(float) * (size_t)m);
    or_fm_discrim(iq, n, disc);
    cf32 *cplx = (cf32 *)malloc(sizeof(cf32) * (size_t)m);
    /* FreqShift(x, fs, -57000): inc = +2 pi 57000 / fs, incremented before use,
     * never wrapped. */
    double phase = 0.0;
    double inc = -2 * OR_PI * (-57000.0) / (double)sample_rate;
    for (int i = 0; i < m; i++) {
        phase += inc;
        double re = cos(phase), im = sin(phase);
        double b = (double)disc[i];
        cplx[i].re = (float)(b * re);
        cplx[i].im = (float)(b * im);
    }
    double taps[101];
    or_lowpass_fir(7500, sample_rate, 101, taps);
    int dr = sample_rate / 19000;
    if (dr < 1) dr = 1;
    int nout = 0;
    for (int i = 0; i < m; i += dr) {
        double ar = 0, ai = 0;
        for (int k = 0; k < 101; k++) {
            int idx = i - k;
            if (idx < 0) break;
            ar += (double)cplx[idx].re * taps[k];
            ai += (double)cplx[idx].im * taps[k];
        }
        out[nout].re = (float)ar;
        out[nout].im = (float)ai;
        nout++;
    }
    *rate_out = sample_rate / dr;
    free(disc);
    free(cplx);
    return nout;
}

/* Streaming form over the discriminator stream.  Feeding consecutive chunks of
 * one stream produces exactly the outputs of a single RDSBasebandComplex call
 * over the concatenated stream: the FreqShift phase (float64, accumulated by
 * repeated addition from 0), the last 100 shifted samples and the decimation
 * phase are carried. */
typedef struct {
    int rate;
    int dr;
    double taps[101];
    double phase;
    double inc;
    int64_t count; /* stream samples seen */
    cf32 hist[100];
    int hist_len; /* valid samples in hist (oldest first), <= 100 */
} or_rds;

size_t or_rds_size(void) { return sizeof(or_rds); }

void or_rds_init(or_rds *r, int sample_rate) {
    memset(r, 0, sizeof *r);
    r->rate = sample_rate;
    r->dr = sample_rate / 19000;
    if (r->dr < 1) r->dr = 1;
    or_lowpass_fir(7500, sample_rate, 101, r->taps);
    r->inc = -2 * OR_PI * (-57000.0) / (double)sample_rate;
}

int or_rds_process(or_rds *r, const float *disc, int n, cf32 *out) {
    cf32 *w = (cf32 *)malloc(sizeof(cf32) * (size_t)(r->hist_len + n + 1));
    memcpy(w, r->hist, sizeof(cf32) * (size_t)r->hist_len);
    int h = r->hist_len;
    for (int i = 0; i < n; i++) {
        r->phase += r->inc;
        double re = cos(r->phase), im = sin(r->phase);
        double b = (double)disc[i];
        w[h + i].re = (float)(b * re);
        w[h + i].im = (float)(b * im);
    }
    int nout = 0;
    for (int i = 0; i < n; i++) {
        int64_t gi = r->count + i;
        if (gi % r->dr != 0) continue;
        double ar = 0, ai = 0;
        for (int k = 0; k < 101; k++) {
            int64_t gidx = gi - k;
            if (gidx < 0) break;
            const cf32 v = w[h + i - k];
            ar += (double)v.re * r->taps[k];
            ai += (double)v.im * r->taps[k];
        }
        out[nout].re = (float)ar;
        out[nout].im = (float)ai;
        nout++;
    }
    int tot = h + n;
    int keep = tot < 100 ? tot : 100;
    memmove(r->hist, w + tot - keep, sizeof(cf32) * (size_t)keep);
    r->hist_len = keep;
    r->count += n;
    free(w);
    return nout;
}

/* ------------------------------------------------------------------------ */
/* internal/rds/rds.go:78-636  RDS decoder                                    */
/* ------------------------------------------------------------------------ */

#define OFF_A 0x0FC
#define OFF_B 0x198
#define OFF_C 0x168
#define OFF_CP 0x350
#define OFF_D 0x1B4

typedef struct {
    char ps[8];
    char rt[64];
    uint16_t last_pi;
    double costas_phase, costas_freq;
    double sync_mu;
    cf32 sync_prev, sync_prev_decision;
    int sync_has_prev;
    int last_sample_rate;
    int last_hard_bit, has_last_hard_bit;
    int total_decodes, groups_found_calls;
    int groups_total; /* groups applied over all calls */
} or_rds_dec;

size_t or_rds_dec_size(void) { return sizeof(or_rds_dec); }
void or_rds_dec_init(or_rds_dec *d) { memset(d, 0, sizeof *d); }

/* rds.go:590-599 crcSyndrome.  Note the reduction polynomial constant lacks the
 * x^10 term, so the tested bit is never cleared; the map is still linear over
 * GF(2) and is restated exactly. */
uint16_t or_rds_syndrome(uint32_t raw) {
    uint32_t poly = 0x1B9;
    uint32_t reg = raw;
    for (int i = 25; i >= 10; i--) {
        if ((reg >> i) & 1) reg ^= poly << (i - 10);
    }
    return (uint16_t)(reg & 0x3FF);
}

static int decode_raw_block(uint32_t raw, uint16_t *data, uint16_t *off) {
    uint16_t s = or_rds_syndrome(raw);
    if (s == OFF_A || s == OFF_B || s == OFF_C || s == OFF_CP || s == OFF_D) {
        *data = (uint16_t)(raw >> 10);
        *off = s;
        return 1;
    }
    return 0;
}

static uint32_t bits_to_raw(const uint8_t *bits) {
    uint32_t raw = 0;
    for (int i = 0; i < 26; i++) raw = (raw << 1) | (uint32_t)(bits[i] & 1);
    return raw;
}

static int off_allowed(uint16_t off, const uint16_t *allowed, int na) {
    for (int i = 0; i < na; i++)
        if (off == allowed[i]) return 1;
    return 0;
}

/* rds.go:538-576 decodeBlockExpected; returns ok, sets *data. */
static int decode_block_expected(const uint8_t *bits, const uint16_t *allowed, int na, int use_fec,
                                 uint16_t *data) {
    uint32_t raw = bits_to_raw(bits);
    uint16_t d, o;
    if (decode_raw_block(raw, &d, &o) && off_allowed(o, allowed, na)) {
        *data = d;
        return 1;
    }
    if (!use_fec) return 0;
    int count = 0;
    uint16_t cand = 0;
    for (int i = 0; i < 26; i++) {
        uint32_t flipped = raw ^ (1u << (25 - i));
        if (!decode_raw_block(flipped, &d, &o) || !off_allowed(o, allowed, na)) continue;
        cand = d;
        count++;
        if (count > 1) return 0;
    }
    if (count == 1) {
        *data = cand;
        return 1;
    }
    return 0;
}

/* rds.go:432-475 decodeGroupAt */
static int decode_group_at(const uint8_t *bits, int nbits, int start, int use_fec, uint16_t grp[4]) {
    static const uint16_t a[1] = {OFF_A}, b[1] = {OFF_B}, c[2] = {OFF_C, OFF_CP}, dd[1] = {OFF_D};
    if (start < 0 || start + 104 > nbits) return 0;
    if (!decode_block_expected(bits + start, a, 1, use_fec, &grp[0])) return 0;
    if (!decode_block_expected(bits + start + 26, b, 1, use_fec, &grp[1])) return 0;
    if (!decode_block_expected(bits + start + 52, c, 2, use_fec, &grp[2])) return 0;
    if (!decode_block_expected(bits + start + 78, dd, 1, use_fec, &grp[3])) return 0;
    return 1;
}

static char sanitize(uint8_t b) { return (b < 32 || b > 126) ? ' ' : (char)b; }

/* rds.go:477-502 applyGroup */
static void apply_group(or_rds_dec *d, const uint16_t g[4]) {
    uint16_t pi = g[0];
    if (pi != 0) d->last_pi = pi;
    int gtype = (g[1] >> 12) & 0xF;
    int version_a = ((g[1] >> 11) & 1) == 0;
    if (gtype == 0 && version_a) {
        int addr = g[1] & 0x3;
        int idx = addr * 2;
        if (idx + 1 < 8) {
            d->ps[idx] = sanitize((uint8_t)(g[3] >> 8));
            d->ps[idx + 1] = sanitize((uint8_t)(g[3] & 0xFF));
        }
    }
    if (gtype == 2 && version_a) {
        int addr = g[1] & 0xF;
        uint8_t ch[4] = {(uint8_t)(g[2] >> 8), (uint8_t)(g[2] & 0xFF), (uint8_t)(g[3] >> 8),
                         (uint8_t)(g[3] & 0xFF)};
        int idx = addr * 4;
        for (int j = 0; j < 4 && idx + j < 64; j++) d->rt[idx + j] = sanitize(ch[j]);
    }
}

/* rds.go:365-430 tryDecode (flywheel +-3) */
static int try_decode(or_rds_dec *d, const uint8_t *bits, int nbits, int use_fec) {
    int groups = 0;
    uint16_t g[4];
    for (int i = 0; i + 104 <= nbits;) {
        if (!decode_group_at(bits, nbits, i, use_fec, g)) {
            i++;
            continue;
        }
        groups++;
        apply_group(d, g);
        int next = i + 104;
        int locked = 1;
        while (locked && next + 104 <= nbits) {
            if (decode_group_at(bits, nbits, next, use_fec, g)) {
                apply_group(d, g);
                groups++;
                next += 104;
                continue;
            }
            int matched = 0;
            for (int delta = 1; delta <= 3 && !matched; delta++) {
                int left = next - delta;
                if (left >= 0 && decode_group_at(bits, nbits, left, use_fec, g)) {
                    apply_group(d, g);
                    groups++;
                    next = left + 104;
                    matched = 1;
                    break;
                }
                int right = next + delta;
                if (right + 104 <= nbits && decode_group_at(bits, nbits, right, use_fec, g)) {
                    apply_group(d, g);
                    groups++;
                    next = right + 104;
                    matched = 1;
                    break;
                }
            }
            if (!matched) locked = 0;
        }
        int resume = next - 3;
        if (resume <= i) resume = i + 1;
        i = resume;
    }
    return groups;
}

/* rds.go:78-264 Decode (diagnostic counters and strings omitted; they do not
 * feed back into decoding).  Returns the number of groups applied by this call. */
int or_rds_decode(or_rds_dec *d, const cf32 *samples, int n, int sample_rate) {
    if (n < 104 || sample_rate <= 0) return 0;
    d->total_decodes++;
    if (d->last_sample_rate != 0 && d->last_sample_rate != sample_rate) {
        d->costas_phase = 0;
        d->costas_freq = 0;
        d->sync_mu = 0;
        d->sync_prev.re = d->sync_prev.im = 0;
        d->sync_prev_decision.re = d->sync_prev_decision.im = 0;
        d->sync_has_prev = 0;
        d->last_hard_bit = 0;
        d->has_last_hard_bit = 0;
    }
    d->last_sample_rate = sample_rate;
    double sps = (double)sample_rate / 1187.5;
    double mu = d->sync_mu;
    if (mu < 0 || mu >= sps || isnan(mu) || isinf(mu)) mu = sps / 2;
    int cap = (int)((double)n / sps) + 8;
    cf32 *sym = (cf32 *)malloc(sizeof(cf32) * (size_t)cap);
    int ns = 0;
    cf32 prev = d->sync_prev, prev_dec = d->sync_prev_decision;
    int have_prev = d->sync_has_prev;
    while (mu < (double)(n - 1)) {
        int idx = (int)mu;
        double frac = mu - (double)idx;
        if (idx + 1 >= n) break;
        cf32 sm;
        sm.re = (float)((double)samples[idx].re * (1 - frac) + (double)samples[idx + 1].re * frac);
        sm.im = (float)((double)samples[idx].im * (1 - frac) + (double)samples[idx + 1].im * frac);
        cf32 dec;
        dec.re = sm.re >= 0 ? 1.0f : -1.0f;
        dec.im = 0.0f;
        if (have_prev) {
            double err_r = (double)(dec.re - prev_dec.re) * (double)prev.re -
                           (double)(sm.re - prev.re) * (double)prev_dec.re;
            mu += sps + 0.01 * err_r;
        } else {
            mu += sps;
            have_prev = 1;
        }
        prev_dec = dec;
        prev = sm;
        if (ns == cap) {
            cap *= 2;
            sym = (cf32 *)realloc(sym, sizeof(cf32) * (size_t)cap);
        }
        sym[ns++] = sm;
    }
    double res = mu - (double)n;
    while (res < 0) res += sps;
    while (res >= sps) res -= sps;
    d->sync_mu = res;
    d->sync_prev = prev;
    d->sync_prev_decision = prev_dec;
    d->sync_has_prev = have_prev;
    if (ns < 104) {
        free(sym);
        return 0;
    }
    double alpha = 0.132, beta = alpha * alpha / 4.0;
    double phase = d->costas_phase, freq = d->costas_freq;
    uint8_t *hard = (uint8_t *)malloc((size_t)ns);
    for (int i = 0; i < ns; i++) {
        float cp = (float)cos(phase), sp = (float)sin(phase);
        cf32 s = sym[i];
        cf32 y;
        y.re = s.re * cp + s.im * sp;
        y.im = s.im * cp - s.re * sp;
        double err = y.re >= 0 ? (double)y.im : -(double)y.im;
        freq += beta * err;
        phase += freq + alpha * err;
        while (phase > OR_PI) phase -= 2 * OR_PI;
        while (phase < -OR_PI) phase += 2 * OR_PI;
        hard[i] = y.re >= 0 ? 1 : 0;
    }
    d->costas_phase = phase;
    d->costas_freq = freq;
    int nb = 0;
    uint8_t *bits = (uint8_t *)malloc((size_t)ns + 1);
    if (d->has_last_hard_bit) {
        bits[0] = hard[0] ^ (uint8_t)d->last_hard_bit;
        for (int i = 1; i < ns; i++) bits[i] = hard[i] ^ hard[i - 1];
        nb = ns;
    } else if (ns >= 2) {
        for (int i = 1; i < ns; i++) bits[i - 1] = hard[i] ^ hard[i - 1];
        nb = ns - 1;
    }
    d->last_hard_bit = hard[ns - 1];
    d->has_last_hard_bit = 1;
    uint8_t *inv = (uint8_t *)malloc((size_t)nb + 1);
    for (int i = 0; i < nb; i++) inv[i] = 1 - bits[i];
    int groups = try_decode(d, bits, nb, 1);
    if (groups == 0) groups = try_decode(d, inv, nb, 1);
    if (groups > 0) d->groups_found_calls++;
    d->groups_total += groups;
    free(sym);
    free(hard);
    free(bits);
    free(inv);
    return groups;
}

void or_rds_dec_result(const or_rds_dec *d, uint16_t *pi, char *ps9, char *rt65) {
    *pi = d->last_pi;
    /* psString / rtString: zero runes become spaces, trailing spaces trimmed. */
    int end = 8;
    for (int i = 0; i < 8; i++) ps9[i] = d->ps[i] ? d->ps[i] : ' ';
    while (end > 0 && ps9[end - 1] == ' ') end--;
    ps9[end] = 0;
    end = 64;
    for (int i = 0; i < 64; i++) rt65[i] = d->rt[i] ? d->rt[i] : ' ';
    while (end > 0 && rt65[end - 1] == ' ') end--;
    rt65[end] = 0;
}

/* ------------------------------------------------------------------------ */
/* Per-channel pipeline (one block at a time)                                 */
/* ------------------------------------------------------------------------ */

/*
 * The chain a channel runs per block, composed from the reference stages:
 * extraction (streaming_host_core.go), then by mode the demod of
 * recorder/streamer.go processSnippet with decim1 == 1 (the extraction rate is
 * the demod rate): discriminator with the one-sample bridge
 * (streamer.go:1287-1302), the WFM mono LPF (streamer.go:1401-1404), the
 * WFM_STEREO stage with hysteresis (streamer.go:1355-1400), AM / SSB / CW per
 * call; RDS baseband for WFM channels in streaming form.
 */
enum {
    OR_MODE_IQ = 0,
    OR_MODE_NFM = 1,
    OR_MODE_WFM = 2,
    OR_MODE_WFM_STEREO = 3,
    OR_MODE_AM = 4,
    OR_MODE_USB = 5,
    OR_MODE_LSB = 6,
    OR_MODE_CW = 7
};

/* internal/dsp/decimating_fir.go:6-95 StatefulDecimatingFIRComplex: float64
 * delay line (delay[0] newest), emit when the phase counter is 0 (then it
 * restarts at factor-1), float64 accumulate, complex64 output. */
typedef struct {
    int n, factor, phase;
    double taps[128];
    double dr[128], di[128];
} or_decim_fir;

static void decim_fir_init(or_decim_fir *f, const double *taps, int n, int factor) {
    memset(f, 0, sizeof *f);
    f->n = n;
    f->factor = factor < 1 ? 1 : factor;
    memcpy(f->taps, taps, sizeof(double) * (size_t)n);
}

static int decim_fir_process(or_decim_fir *f, const cf32 *iq, int len, cf32 *out) {
    int n = f->n, nout = 0;
    if (len == 0 || n == 0) return 0;
    for (int i = 0; i < len; i++) {
        memmove(f->dr + 1, f->dr, sizeof(double) * (size_t)(n - 1));
        memmove(f->di + 1, f->di, sizeof(double) * (size_t)(n - 1));
        f->dr[0] = (double)iq[i].re;
        f->di[0] = (double)iq[i].im;
        if (f->factor <= 1 || f->phase == 0) {
            double ar = 0, ai = 0;
            for (int k = 0; k < n; k++) {
                ar += f->dr[k] * f->taps[k];
                ai += f->di[k] * f->taps[k];
            }
            out[nout].re = (float)ar;
            out[nout].im = (float)ai;
            nout++;
            if (f->factor > 1) f->phase = f->factor - 1;
        } else {
            f->phase--;
        }
    }
    return nout;
}

size_t or_decim_fir_size(void) { return sizeof(or_decim_fir); }
int or_decim_fir_init(or_decim_fir *f, const double *taps, int n, int factor) {
    if (n < 1 || n > 128) return -1;
    decim_fir_init(f, taps, n, factor);
    return 0;
}
int or_decim_fir_process(or_decim_fir *f, const cf32 *iq, int len, cf32 *out) { return decim_fir_process(f, iq, len, out); }
int or_decim_fir_phase(const or_decim_fir *f) { return f->phase; }

typedef struct {
    int sample_rate, out_rate, num_taps, decim, mode, rds_on;
    int demod_decim, demod_rate;
    or_decim_fir pre;
    double offset_hz;
    double nco_phase;
    int phase_count;
    int hist_len;
    cf32 hist[4096];
    int poly_len;
    float poly[8192 + 4096];
    cf32 last_iq;
    int has_last;
    or_stereo st;
    or_rds rds;
} or_channel;

size_t or_channel_size(void) { return sizeof(or_channel); }

/* gpudemod/stream_state.go:25-85 getOrInitExtractState (tap design part):
 * cutoff = max(BW/2, 200), LowpassFIR(cutoff, fs, T) cast to float32, laid out
 * phase-major.  Returns 0 or -1 for a non-integer decimation. */
int or_channel_init(or_channel *ch, int sample_rate, double offset_hz, double bandwidth, int out_rate, int num_taps,
                    int mode, int rds_on) {
    memset(ch, 0, sizeof *ch);
    int D = or_exact_decim(sample_rate, out_rate);
    if (D <= 0) return -1;
    if (num_taps <= 0) num_taps = 101;
    ch->sample_rate = sample_rate;
    ch->out_rate = out_rate;
    ch->num_taps = num_taps;
    ch->decim = D;
    ch->mode = mode;
    ch->rds_on = rds_on;
    ch->offset_hz = offset_hz;
    double cutoff = bandwidth / 2;
    if (cutoff < 200) cutoff = 200;
    double base[4097];
    int blen = or_lowpass_fir(cutoff, sample_rate, num_taps, base);
    float basef[4097];
    for (int i = 0; i < blen; i++) basef[i] = (float)base[i];
    ch->poly_len = or_build_polyphase(basef, blen, D, ch->poly);
    or_stereo_init(&ch->st);
    or_rds_init(&ch->rds, out_rate);
    ch->demod_decim = 1;
    ch->demod_rate = out_rate;
    return 0;
}

/* recorder/streamer.go:1098-1146: the stateful anti-alias FIR + decimation
 * by decim1 ahead of the demodulator: 101 taps of LowpassFIR(cutoff, snip
 * rate), cutoff 90 kHz for WFM modes, else 0.8 x the demod Nyquist.  The demod
 * stages then run at out_rate / decim1. */
int or_channel_set_demod_decim(or_channel *ch, int decim1) {
    if (decim1 <= 1) return 0;
    int drate = ch->out_rate / decim1;
    int wfm = ch->mode == OR_MODE_WFM || ch->mode == OR_MODE_WFM_STEREO;
    double cutoff = wfm ? 90000.0 : (double)drate / 2.0 * 0.8;
    double taps[128];
    int n = or_lowpass_fir(cutoff, ch->out_rate, 101, taps);
    decim_fir_init(&ch->pre, taps, n, decim1);
    ch->demod_decim = decim1;
    ch->demod_rate = drate;
    or_rds_init(&ch->rds, drate);
    return 0;
}

/* Runs one block.  Output capacities: iq_out n/D+2, audio 2*(n/D+2), rds
 * n/D/dr+2.  Counts are returned through the pointers; flags (bit0 locked,
 * bit1 stereo enabled) through *flags. */
int or_channel_process(or_channel *ch, const cf32 *in, int n, cf32 *iq_out, int *n_iq, float *audio,
                       int *n_audio, cf32 *rds_out, int *n_rds, int *flags) {
    int nout = or_extract_host_core(in, n, ch->sample_rate, ch->offset_hz, &ch->nco_phase, &ch->phase_count,
                                    ch->num_taps, ch->decim, ch->hist, &ch->hist_len, ch->poly, ch->poly_len,
                                    iq_out);
    *n_iq = nout;
    *n_audio = 0;
    *n_rds = 0;
    *flags = 0;
    int rate = ch->demod_rate;
    cf32 *dec = NULL;
    if (ch->demod_decim > 1) {
        /* the demodulator sees the decimated stream; iq_out keeps the extraction output */
        dec = (cf32 *)malloc(sizeof(cf32) * (size_t)(nout + 2));
        int nd = decim_fir_process(&ch->pre, iq_out, nout, dec);
        nout = nd;
    }
    const cf32 *dq = dec ? dec : iq_out;
    switch (ch->mode) {
    case OR_MODE_NFM:
    case OR_MODE_WFM:
    case OR_MODE_WFM_STEREO: {
        float *disc = (float *)malloc(sizeof(float) * (size_t)(nout + 2));
        int nd = 0;
        if (ch->has_last && nout > 0) {
            cf32 *br = (cf32 *)malloc(sizeof(cf32) * (size_t)(nout + 1));
            br[0] = ch->last_iq;
            memcpy(br + 1, dq, sizeof(cf32) * (size_t)nout);
            nd = or_fm_discrim(br, nout + 1, disc);
            free(br);
        } else {
            nd = or_fm_discrim(dq, nout, disc);
        }
        if (nout > 0) {
            ch->last_iq = dq[nout - 1];
            ch->has_last = 1;
        }
        if (nd > 0) {
            if (ch->mode == OR_MODE_NFM) {
                memcpy(audio, disc, sizeof(float) * (size_t)nd);
                *n_audio = nd;
            } else if (ch->mode == OR_MODE_WFM) {
                *n_audio = or_wfm_mono_stage(&ch->st, disc, nd, rate, audio);
            } else {
                int lk = 0, en = 0;
                or_wfm_stereo_stage(&ch->st, disc, nd, rate, audio, &lk, &en);
                *n_audio = 2 * nd;
                *flags = (lk ? 1 : 0) | (en ? 2 : 0);
            }
            if (ch->rds_on && ch->mode != OR_MODE_NFM) *n_rds = or_rds_process(&ch->rds, disc, nd, rds_out);
        }
        free(disc);
        break;
    }
    case OR_MODE_AM:
        *n_audio = or_am_demod(dq, nout, audio);
        break;
    case OR_MODE_USB:
        *n_audio = or_ssb_demod(dq, nout, rate, 1, audio);
        break;
    case OR_MODE_LSB:
        *n_audio = or_ssb_demod(dq, nout, rate, 0, audio);
        break;
    case OR_MODE_CW:
        *n_audio = or_cw_demod(dq, nout, rate, audio);
        break;
    default:
        break;
    }
    free(dec);
    return 0;
}

void or_channel_state(const or_channel *ch, double *nco_phase, int *phase_count, int *hist_len) {
    *nco_phase = ch->nco_phase;
    *phase_count = ch->phase_count;
    *hist_len = ch->hist_len;
}

void or_channel_stereo_margins(const or_channel *ch, double *coherence, double *freq_hz, double *err_avg) {
    or_stereo_margins(&ch->st, coherence, freq_hz, err_avg);
}

void or_channel_set_offset(or_channel *ch, double offset_hz) { ch->offset_hz = offset_hz; }

/* ------------------------------------------------------------------------ */
/* Audio back end: internal/dsp/resample.go:45-232 (rational polyphase        */
/* resampler), recorder/streamer.go:1408-1470 (48 kHz resample, de-emphasis,  */
/* x0.35 for WFM) and :569-575 with wavwriter.go:77-85 (s16le encoding).      */
/* ------------------------------------------------------------------------ */

static int or_gcd(int a, int b) {
    while (b != 0) {
        int t = a % b;
        a = b;
        b = t;
    }
    return a < 0 ? -a : a;
}

/* resample.go bessel0: series until the term drops below 1e-12 of the sum. */
static double or_bessel0(double x) {
    double sum = 1.0, term = 1.0;
    for (int k = 1; k < 30; k++) {
        term *= (x / (2 * (double)k)) * (x / (2 * (double)k));
        sum += term;
        if (term < 1e-12 * sum) break;
    }
    return sum;
}

#define OR_RS_MAXL 512
#define OR_RS_MAXK 40
typedef struct {
    int l, m, taps; /* upsample L, downsample M, taps per arm */
    double bank_in[OR_RS_MAXL * OR_RS_MAXK]; /* arms of small banks, bank[p*taps + t] */
    double *bank;                            /* bank_in, or a heap bank for L > OR_RS_MAXL */
    double delay[OR_RS_MAXK];                /* delay[0] newest */
    int out_time;
} or_resampler;

size_t or_resampler_size(void) { return sizeof(or_resampler); }

/* NewResampler (resample.go:45-93): L/M from the gcd, prototype of odd length
 * L*tapsPerPhase(+1), windowed sinc fc = 0.90/max(L,M) with Kaiser beta 6 and
 * gain L, split into L arms of ceil(len/L) taps.  Returns 0, or -1 when the
 * bank does not fit. */
static int resampler_init(or_resampler *r, int in_rate, int out_rate, int taps_per_phase, int heap_ok);

int or_resampler_init(or_resampler *r, int in_rate, int out_rate, int taps_per_phase) {
    return resampler_init(r, in_rate, out_rate, taps_per_phase, 0);
}

/* Same with any L: banks above OR_RS_MAXL arms on the heap (or_resampler_release). */
int or_resampler_init_any(or_resampler *r, int in_rate, int out_rate, int taps_per_phase) {
    return resampler_init(r, in_rate, out_rate, taps_per_phase, 1);
}

void or_resampler_release(or_resampler *r) {
    if (r->bank && r->bank != r->bank_in) free(r->bank);
    r->bank = r->bank_in;
}

static int resampler_init(or_resampler *r, int in_rate, int out_rate, int taps_per_phase, int heap_ok) {
    memset(r, 0, sizeof *r);
    r->bank = r->bank_in;
    if (in_rate <= 0 || out_rate <= 0) in_rate = out_rate = 1;
    if (taps_per_phase < 4) taps_per_phase = 4;
    int g = or_gcd(in_rate, out_rate);
    int l = out_rate / g, m = in_rate / g;
    int plen = l * taps_per_phase;
    if (plen % 2 == 0) plen++;
    int k = (plen + l - 1) / l;
    if (k > OR_RS_MAXK) return -1;
    if (l > OR_RS_MAXL) {
        if (!heap_ok) return -1;
        r->bank = (double *)malloc(sizeof(double) * (size_t)l * (size_t)k);
        if (!r->bank) {
            r->bank = r->bank_in;
            return -1;
        }
    }
    double fc = 0.90 / (double)(l > m ? l : m);
    double mid = (double)(plen - 1) / 2.0;
    double b0 = or_bessel0(6.0);
    for (int p = 0; p < l; p++)
        for (int t = 0; t < k; t++) {
            int n = p + t * l;
            double v = 0.0;
            if (n < plen) {
                double x = (double)n - mid;
                double s = fabs(x) < 1e-12 ? 2 * OR_PI * fc : sin(2 * OR_PI * fc * x) / x;
                double xx = ((double)n - mid) / mid;
                double w = or_bessel0(6.0 * sqrt(1 - xx * xx)) / b0;
                v = s * w * (double)l;
            }
            r->bank[p * k + t] = v;
        }
    r->l = l;
    r->m = m;
    r->taps = k;
    return 0;
}

void or_resampler_ratio(const or_resampler *r, int *l, int *m, int *taps, int *out_time) {
    *l = r->l;
    *m = r->m;
    *taps = r->taps;
    *out_time = r->out_time;
}

void or_resampler_bank(const or_resampler *r, double *out) {
    memcpy(out, r->bank, sizeof(double) * (size_t)(r->l * r->taps));
}

/* Resampler.Process (resample.go:105-153), including its exits: when the input
 * runs out inside the consume loop the phase counter has already been reduced
 * by L for the sample it could not consume.  Returns the output count. */
int or_resampler_process(or_resampler *r, const float *in, int n, float *out) {
    if (n == 0) return 0;
    if (r->l == r->m) {
        memcpy(out, in, sizeof(float) * (size_t)n);
        return n;
    }
    int L = r->l, M = r->m, K = r->taps;
    int pos = 0, t = r->out_time, nout = 0;
    while (pos < n) {
        while (t >= L) {
            t -= L;
            if (pos >= n) {
                r->out_time = t;
                return nout;
            }
            memmove(r->delay + 1, r->delay, sizeof(double) * (size_t)(K - 1));
            r->delay[0] = (double)in[pos++];
        }
        const double *arm = r->bank + t * K;
        double acc = 0;
        for (int k = 0; k < K; k++) acc += r->delay[k] * arm[k];
        out[nout++] = (float)acc;
        t += M;
    }
    r->out_time = t;
    return nout;
}

/* The 48 kHz back end of one channel: a resampler per audio channel
 * (StereoResampler for 2), then for WFM modes the one-pole de-emphasis
 * y = a*y + (1-a)*x, a = exp(-1/(48000*tau)) in float64 per channel and the
 * x0.35 gain, then s16le: int16(clip(s*32767)) with Go's truncating
 * conversion. */
typedef struct {
    int channels, wfm;
    double deemph_us, y[2];
    or_resampler rs[2];
} or_audio48;

size_t or_audio48_size(void) { return sizeof(or_audio48); }

int or_audio48_init(or_audio48 *a, int in_rate, int channels, int wfm, double deemph_us) {
    memset(a, 0, sizeof *a);
    a->channels = channels;
    a->wfm = wfm;
    a->deemph_us = deemph_us;
    for (int c = 0; c < channels; c++)
        if (or_resampler_init(&a->rs[c], in_rate, 48000, 32) != 0) return -1;
    return 0;
}

/* in: frames x channels interleaved at the demod rate.  Writes interleaved
 * float audio (out_f, may be NULL) and s16le samples; returns the sample
 * count (frames x channels). */
int or_audio48_process(or_audio48 *a, const float *in, int frames, float *out_f, int16_t *pcm) {
    int C = a->channels;
    /* per-channel output capacity: frames * L / M plus the phase slack */
    size_t cap = (size_t)((double)frames * (double)a->rs[0].l / (double)a->rs[0].m) + (size_t)frames / 1000 + 64;
    float *tmp = (float *)malloc(sizeof(float) * (size_t)(frames + 8));
    float *res = (float *)malloc(sizeof(float) * (size_t)C * cap);
    int nf = -1;
    float *outs[2] = {NULL, NULL};
    int cnt[2] = {0, 0};
    for (int c = 0; c < C; c++) {
        for (int i = 0; i < frames; i++) tmp[i] = in[i * C + c];
        outs[c] = res + (size_t)c * cap;
        cnt[c] = or_resampler_process(&a->rs[c], tmp, frames, outs[c]);
        if (nf < 0 || cnt[c] < nf) nf = cnt[c];
    }
    if (nf < 0) nf = 0;
    float *audio = (float *)malloc(sizeof(float) * (size_t)(nf * C + 1));
    for (int i = 0; i < nf; i++)
        for (int c = 0; c < C; c++) audio[i * C + c] = outs[c][i];
    if (a->wfm && a->deemph_us > 0) {
        double tau = a->deemph_us * 1e-6;
        double al = exp(-1.0 / (48000.0 * tau));
        for (int c = 0; c < C; c++) {
            double y = a->y[c];
            for (int i = 0; i < nf; i++) {
                y = al * y + (1 - al) * (double)audio[i * C + c];
                audio[i * C + c] = (float)y;
            }
            a->y[c] = y;
        }
    }
    if (a->wfm)
        for (int i = 0; i < nf * C; i++) audio[i] *= 0.35f;
    for (int i = 0; i < nf * C; i++) {
        float v = audio[i] * 32767.0f;
        if (v > 32767.0f) v = 32767.0f;
        if (v < -32768.0f) v = -32768.0f;
        pcm[i] = (int16_t)v; /* truncation toward zero, as Go's conversion */
        if (out_f) out_f[i] = audio[i];
    }
    free(tmp);
    free(res);
    free(audio);
    return nf * C;
}

/* ------------------------------------------------------------------------ */
/* internal/classifier/pll.go:35-42, 75-131, 170-196  StereoPilotPresent /    */
/* estimateWFMPilot: float64 FM discriminator, 201 Goertzel magnitudes at      */
/* 19 kHz +-1 kHz in 10 Hz steps, locked when max / median > threshold.        */
/* ------------------------------------------------------------------------ */

static int or_cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* window != 0: StereoPilotPresent (the last sample_rate/2 samples); else the
 * whole vector (estimateWFMPilot as EstimateExactFrequency calls it).
 * Returns the lock decision; *ratio, *best_hz, *median and mags[201] (may be
 * NULL) receive the intermediate values. */
int or_stereo_pilot(const cf32 *iq, int n, int sample_rate, int window, double threshold, double *ratio,
                    double *best_hz, double *median, double *mags) {
    *ratio = 0;
    *best_hz = 19000.0;
    *median = 0;
    if (window) {
        int mx = sample_rate / 2;
        if (mx > 0 && n > mx) {
            iq += n - mx;
            n = mx;
        }
    }
    if (sample_rate < 40000 || n < 2) return 0;
    int nd = n - 1;
    double *d = (double *)malloc(sizeof(double) * (size_t)nd);
    for (int i = 1; i < n; i++) {
        cf32 p = iq[i - 1], c = iq[i];
        double num = (double)p.re * (double)c.im - (double)p.im * (double)c.re;
        double den = (double)p.re * (double)c.re + (double)p.im * (double)c.im;
        d[i - 1] = atan2(num, den);
    }
    double m[201], best = 0.0, bestf = 19000.0;
    int cnt = 0;
    for (double off = -1000.0; off <= 1000.0; off += 10.0) {
        double f = 19000.0 + off;
        double k = f / ((double)sample_rate / (double)nd);
        double w = 2.0 * OR_PI * k / (double)nd;
        double coeff = 2.0 * cos(w);
        double s1 = 0.0, s2 = 0.0;
        for (int i = 0; i < nd; i++) {
            double s0 = d[i] + coeff * s1 - s2;
            s2 = s1;
            s1 = s0;
        }
        double mag = sqrt(s1 * s1 + s2 * s2 - coeff * s1 * s2);
        m[cnt++] = mag;
        if (mag > best) {
            best = mag;
            bestf = f;
        }
    }
    free(d);
    if (mags) memcpy(mags, m, sizeof m);
    double c[201];
    memcpy(c, m, sizeof m);
    qsort(c, 201, sizeof(double), or_cmp_double);
    double med = c[201 / 2];
    *median = med;
    *best_hz = bestf;
    if (med > 0) *ratio = best / med;
    return med > 0 && *ratio > threshold;
}

/* ------------------------------------------------------------------------ */
/* Event-recording batch path (recorder/wfm_batch_stereo.go:10-168): one call
 * over a whole capture, every stage stateless.                             */

/* dsp.ApplyFIRReal (dsp/fir_real.go:4-20): float64 taps and accumulation from
 * a zero history, float32 out. */
static void apply_fir_real(const float *x, int n, const double *taps, int nt, float *out) {
    for (int i = 0; i < n; i++) {
        double acc = 0;
        for (int k = 0; k < nt; k++) {
            int idx = i - k;
            if (idx < 0) break;
            acc += (double)x[idx] * taps[k];
        }
        out[i] = (float)acc;
    }
}

/* wfmStereoDecodeBatch (wfm_batch_stereo.go:74-155): the streaming decoder's
 * filters and pilot loop from a fresh state over one call, locked when the
 * pilot-band power is above 0.3 % of the composite's, the loop frequency
 * within 250 Hz of 19 kHz and the mean |phase error| below 0.35.  out: 2n
 * interleaved L/R (written whatever the decision).  Returns locked. */
int or_wfm_stereo_decode_batch(const float *mono, int n, int rate, float *out, double *ratio_out,
                               double *freq_hz_out, double *err_out) {
    if (n <= 0 || rate <= 0) return 0;
    double lp[101], h53[101], h23[101], h21[101], h17[101];
    or_lowpass_fir(15000, rate, 101, lp);
    or_lowpass_fir(53000, rate, 101, h53);
    or_lowpass_fir(23000, rate, 101, h23);
    or_lowpass_fir(21000, rate, 101, h21);
    or_lowpass_fir(17000, rate, 101, h17);
    float *lpr = (float *)malloc(sizeof(float) * (size_t)n * 6);
    float *hi = lpr + n, *lo = lpr + 2 * (size_t)n, *pilot = lpr + 3 * (size_t)n, *bpf = lpr + 4 * (size_t)n,
          *lr = lpr + 5 * (size_t)n;
    apply_fir_real(mono, n, lp, 101, lpr);
    apply_fir_real(mono, n, h53, 101, hi);
    apply_fir_real(mono, n, h23, 101, lo);
    for (int i = 0; i < n; i++) bpf[i] = hi[i] - lo[i];
    apply_fir_real(mono, n, h21, 101, hi);
    apply_fir_real(mono, n, h17, 101, lo);
    for (int i = 0; i < n; i++) pilot[i] = hi[i] - lo[i];
    double phase = 0.0, freq = 2 * OR_PI * 19000 / (double)rate, alpha, beta;
    or_pll_coefficients(50, 0.707, rate, &alpha, &beta);
    double lpa = 1 - exp(-2 * OR_PI * 200 / (double)rate);
    double is = 0, qs = 0;
    double fmin = 2 * OR_PI * 17000 / (double)rate, fmax = 2 * OR_PI * 21000 / (double)rate;
    double pp = 0, tp = 0, es = 0;
    for (int i = 0; i < n; i++) {
        double p = (double)pilot[i];
        double sp = sin(phase), cp = cos(phase);
        double im = p * cp, qm = p * -sp;
        is += lpa * (im - is);
        qs += lpa * (qm - qs);
        double err = atan2(qs, is);
        freq += beta * err;
        if (freq < fmin) freq = fmin;
        else if (freq > fmax) freq = fmax;
        phase += freq + alpha * err;
        if (phase > 2 * OR_PI) phase -= 2 * OR_PI;
        else if (phase < 0) phase += 2 * OR_PI;
        tp += (double)mono[i] * (double)mono[i];
        pp += p * p;
        es += fabs(err);
        lr[i] = bpf[i] * (float)(2 * sin(2 * phase));
    }
    apply_fir_real(lr, n, lp, 101, hi);  /* lr filtered */
    double ratio = tp > 0 ? pp / tp : 0.0;
    double fhz = freq * (double)rate / (2 * OR_PI);
    double berr = es / (double)n;
    int locked = ratio > 0.003 && fabs(fhz - 19000) < 250 && berr < 0.35;
    for (int i = 0; i < n; i++) {
        out[2 * i] = 0.5f * (lpr[i] + hi[i]);
        out[2 * i + 1] = 0.5f * (lpr[i] - hi[i]);
    }
    if (ratio_out) *ratio_out = ratio;
    if (freq_hz_out) *freq_hz_out = fhz;
    if (err_out) *err_out = berr;
    free(lpr);
    return locked;
}

/* demodWFMStereoBatchAudio (wfm_batch_stereo.go:10-72): FreqShift by the
 * offset (float64 phase accumulated from 0, product rounded once), 101-tap
 * LowpassFIR at max(bw/2, 200) raised to 75 kHz (the WFM demodulator's
 * 192 kS/s output), ApplyFIR over every sample, Decimate by
 * decim1 = round(fs/192000) from index 0, the discriminator, the batch stereo
 * decoder (duplicated mono when not locked), the stereo resampler to 48 kHz
 * unless the demod rate is 48 kHz, de-emphasis at the output rate, x0.35.
 * Writes interleaved float L/R to out (capacity out_cap floats); returns the
 * float count, or -1 (capacity, resampler). */
int or_wfm_batch_audio(const cf32 *iq, int n, int fs, double offset, double bw, double deemph_us, float *out,
                       int out_cap, int *out_rate, int *locked_out, int *demod_rate_out) {
    *out_rate = 0;
    *locked_out = 0;
    if (n <= 0 || fs <= 0) return 0;
    double cutoff = bw / 2;
    if (cutoff < 200) cutoff = 200;
    if (cutoff < 75000) cutoff = 75000;
    double taps[128];
    int nt = or_lowpass_fir(cutoff, fs, 101, taps);
    int d1 = (int)round((double)fs / 192000.0);
    if (d1 < 1) d1 = 1;
    int rate = fs / d1;
    if (demod_rate_out) *demod_rate_out = rate;
    int nd = (n + d1 - 1) / d1;
    cf32 *dec = (cf32 *)malloc(sizeof(cf32) * (size_t)nd);
    double inc = offset != 0 ? -2 * OR_PI * offset / (double)fs : 0.0;
    /* shifted samples feeding the decimated outputs only (ApplyFIR then Decimate) */
    cf32 *sh = (cf32 *)malloc(sizeof(cf32) * (size_t)n);
    double ph = 0.0;
    for (int i = 0; i < n; i++) {
        if (offset == 0) {
            sh[i] = iq[i];
            continue;
        }
        ph += inc;
        double re = cos(ph), im = sin(ph);
        sh[i].re = (float)((double)iq[i].re * re - (double)iq[i].im * im);
        sh[i].im = (float)((double)iq[i].re * im + (double)iq[i].im * re);
    }
    for (int j = 0; j < nd; j++) {
        int i = j * d1;
        double ar = 0, ai = 0;
        for (int k = 0; k < nt; k++) {
            int idx = i - k;
            if (idx < 0) break;
            ar += (double)sh[idx].re * taps[k];
            ai += (double)sh[idx].im * taps[k];
        }
        dec[j].re = (float)ar;
        dec[j].im = (float)ai;
    }
    free(sh);
    if (nd < 2) {
        free(dec);
        return 0;
    }
    int nm = nd - 1;
    float *mono = (float *)malloc(sizeof(float) * (size_t)nm);
    or_fm_discrim(dec, nd, mono);
    free(dec);
    float *st = (float *)malloc(sizeof(float) * (size_t)nm * 2);
    int locked = or_wfm_stereo_decode_batch(mono, nm, rate, st, NULL, NULL, NULL);
    if (!locked)
        for (int i = 0; i < nm; i++) st[2 * i] = st[2 * i + 1] = mono[i];
    free(mono);
    int orate = rate, nf = nm;
    float *audio = st;
    if (rate != 48000) {
        or_resampler *rs = (or_resampler *)malloc(sizeof(or_resampler) * 2);
        if (or_resampler_init_any(&rs[0], rate, 48000, 32) != 0 || or_resampler_init_any(&rs[1], rate, 48000, 32) != 0) {
            free(rs);
            free(st);
            return -1;
        }
        size_t cap = (size_t)((double)nm * 48000.0 / (double)rate) + 64;
        float *tmp = (float *)malloc(sizeof(float) * (size_t)nm);
        float *o0 = (float *)malloc(sizeof(float) * cap), *o1 = (float *)malloc(sizeof(float) * cap);
        for (int i = 0; i < nm; i++) tmp[i] = st[2 * i];
        int c0 = or_resampler_process(&rs[0], tmp, nm, o0);
        for (int i = 0; i < nm; i++) tmp[i] = st[2 * i + 1];
        int c1 = or_resampler_process(&rs[1], tmp, nm, o1);
        nf = c0 < c1 ? c0 : c1;
        audio = (float *)malloc(sizeof(float) * (size_t)(2 * nf + 1));
        for (int i = 0; i < nf; i++) {
            audio[2 * i] = o0[i];
            audio[2 * i + 1] = o1[i];
        }
        or_resampler_release(&rs[0]);
        or_resampler_release(&rs[1]);
        free(rs);
        free(tmp);
        free(o0);
        free(o1);
        free(st);
        orate = 48000;
    }
    if (2 * nf > out_cap) {
        free(audio);
        return -1;
    }
    if (deemph_us > 0 && orate > 0) {
        double tau = deemph_us * 1e-6;
        double al = exp(-1.0 / ((double)orate * tau));
        double yl = 0, yr = 0;
        for (int i = 0; i < nf; i++) {
            yl = al * yl + (1 - al) * (double)audio[2 * i];
            audio[2 * i] = (float)yl;
            yr = al * yr + (1 - al) * (double)audio[2 * i + 1];
            audio[2 * i + 1] = (float)yr;
        }
    }
    for (int i = 0; i < 2 * nf; i++) out[i] = audio[i] * 0.35f;
    free(audio);
    *out_rate = orate;
    *locked_out = locked;
    return 2 * nf;
}

/* demod.wfmStereo (demod/fm.go:92-123), WFMStereo.Demod: discriminator, 15 kHz
 * L+R, 53k-23k band, a free-running 38 kHz carrier pre-incremented from phase
 * 0 (no pilot loop), L-R through the 15 kHz filter, L/R matrix; all filters
 * ApplyFIRReal from a zero history.  out: 2*(n-1) floats.  Returns frames. */
int or_wfm_stereo_free(const cf32 *iq, int n, int rate, float *out) {
    if (n < 2) return 0;
    int m = n - 1;
    float *base = (float *)malloc(sizeof(float) * (size_t)m * 5);
    float *lpr = base + m, *hi = base + 2 * (size_t)m, *lo = base + 3 * (size_t)m, *lr = base + 4 * (size_t)m;
    or_fm_discrim(iq, n, base);
    double lp[101], h53[101], h23[101];
    or_lowpass_fir(15000, rate, 101, lp);
    or_lowpass_fir(53000, rate, 101, h53);
    or_lowpass_fir(23000, rate, 101, h23);
    apply_fir_real(base, m, lp, 101, lpr);
    apply_fir_real(base, m, h53, 101, hi);
    apply_fir_real(base, m, h23, 101, lo);
    double phase = 0.0, inc = 2 * OR_PI * 38000 / (double)rate;
    for (int i = 0; i < m; i++) {
        float bpf = hi[i] - lo[i];
        phase += inc;
        lr[i] = bpf * (float)(2 * cos(phase));
    }
    apply_fir_real(lr, m, lp, 101, hi);
    for (int i = 0; i < m; i++) {
        out[2 * i] = 0.5f * (lpr[i] + hi[i]);
        out[2 * i + 1] = 0.5f * (lpr[i] - hi[i]);
    }
    free(base);
    return m;
}

/* recorder/cpu_audio.go:10-75 demodAudioCPU, the one-shot demod of a segment
 * (live /api/demod and event recordings): FreqShift, 101-tap LowpassFIR at
 * max(bw/2, 200) (75 kHz at least for the 192 kS/s WFM demodulators), ApplyFIR,
 * Decimate by round(fs/demodRate) from index 0, the mode's Demod at the actual
 * rate (WFM: the discriminator; WFM_STEREO: the free-running stereo decoder),
 * then above 48 kHz a 63-tap anti-alias LowpassFIR at 21.6 kHz and every
 * round(rate/48000)-th sample (stereo: whole frames only).  Writes the audio
 * to out (capacity out_cap floats); returns the float count or -1. */
int or_demod_audio_segment(int mode, const cf32 *iq, int n, int fs, double offset, double bw, float *out,
                           int out_cap, int *channels_out, int *out_rate, int *demod_rate_out) {
    *channels_out = mode == OR_MODE_WFM_STEREO ? 2 : 1;
    *out_rate = 0;
    if (n <= 0 || fs <= 0) return 0;
    int drate = (mode == OR_MODE_WFM || mode == OR_MODE_WFM_STEREO) ? 192000 : 48000;
    double cutoff = bw / 2;
    if (cutoff < 200) cutoff = 200;
    if (cutoff < 75000 && drate >= 192000) cutoff = 75000;
    double taps[128];
    int nt = or_lowpass_fir(cutoff, fs, 101, taps);
    int d1 = (int)round((double)fs / (double)drate);
    if (d1 < 1) d1 = 1;
    int rate = fs / d1;
    *demod_rate_out = rate;
    int nd = (n + d1 - 1) / d1;
    cf32 *sh = (cf32 *)malloc(sizeof(cf32) * (size_t)n);
    double inc = offset != 0 ? -2 * OR_PI * offset / (double)fs : 0.0, ph = 0.0;
    for (int i = 0; i < n; i++) {
        if (offset == 0) {
            sh[i] = iq[i];
            continue;
        }
        ph += inc;
        double re = cos(ph), im = sin(ph);
        sh[i].re = (float)((double)iq[i].re * re - (double)iq[i].im * im);
        sh[i].im = (float)((double)iq[i].re * im + (double)iq[i].im * re);
    }
    cf32 *dec = (cf32 *)malloc(sizeof(cf32) * (size_t)nd);
    for (int j = 0; j < nd; j++) {
        double ar = 0, ai = 0;
        for (int k = 0; k < nt; k++) {
            int idx = j * d1 - k;
            if (idx < 0) break;
            ar += (double)sh[idx].re * taps[k];
            ai += (double)sh[idx].im * taps[k];
        }
        dec[j].re = (float)ar;
        dec[j].im = (float)ai;
    }
    free(sh);
    float *audio = (float *)malloc(sizeof(float) * (size_t)(2 * nd + 2));
    int na = 0;  /* floats */
    switch (mode) {
    case OR_MODE_NFM:
    case OR_MODE_WFM: na = or_fm_discrim(dec, nd, audio); break;
    case OR_MODE_WFM_STEREO: na = 2 * or_wfm_stereo_free(dec, nd, rate, audio); break;
    case OR_MODE_AM: na = or_am_demod(dec, nd, audio); break;
    case OR_MODE_USB: na = or_ssb_demod(dec, nd, rate, 1, audio); break;
    case OR_MODE_LSB: na = or_ssb_demod(dec, nd, rate, 0, audio); break;
    case OR_MODE_CW: na = or_cw_demod(dec, nd, rate, audio); break;
    default: break;
    }
    free(dec);
    int C = *channels_out, orate = rate, nout = na;
    if (rate > 48000 && na > 0) {
        double aa[64];
        int na_t = or_lowpass_fir(48000.0 / 2.0 * 0.9, rate, 63, aa);
        int d2 = (int)round((double)rate / 48000.0);
        if (d2 < 1) d2 = 1;
        int frames = na / C;
        float *ch = (float *)malloc(sizeof(float) * (size_t)frames * 2);
        float *flt = ch + frames;
        int of = C == 2 ? frames / d2 : (frames + d2 - 1) / d2;
        if (C * of > out_cap) {
            free(ch);
            free(audio);
            return -1;
        }
        for (int c = 0; c < C; c++) {
            for (int i = 0; i < frames; i++) ch[i] = audio[i * C + c];
            apply_fir_real(ch, frames, aa, na_t, flt);
            for (int i = 0; i < of; i++) out[i * C + c] = flt[i * d2];
        }
        free(ch);
        nout = C * of;
        orate = rate / d2;
    } else {
        if (na > out_cap) {
            free(audio);
            return -1;
        }
        memcpy(out, audio, sizeof(float) * (size_t)na);
    }
    free(audio);
    *out_rate = orate;
    return nout;
}

/* ------------------------------------------------------------------------ */
/* Job construction (cmd/sdrd): the rules that turn detected signals into    */
/* extraction jobs, i.e. which (out rate, taps, bandwidth) classes the       */
/* extractor sees.  Go `int` is 64-bit: int64_t throughout.                  */
/* ------------------------------------------------------------------------ */

/* cmd/sdrd/streaming_refactor.go:105-137 nearestExactDecimationRate: the
 * target itself when it divides the rate; else, over d = max(1, floor(sr /
 * target) - 2) .. floor + 2, the rate sr / d (>= minRate, and only when it
 * divides sr exactly) closest to the target, the first of equal distances;
 * the target when none qualifies. */
int64_t or_nearest_exact_decimation_rate(int64_t sample_rate, int64_t target, int64_t min_rate) {
    if (sample_rate <= 0 || target <= 0) return target;
    if (sample_rate % target == 0) return target;
    int64_t td = sample_rate / target;
    int64_t best = 0, best_dist = sample_rate;
    int64_t d0 = td - 2 > 1 ? td - 2 : 1;
    for (int64_t d = d0; d <= td + 2; d++) {
        int64_t rate = sample_rate / d;
        if (rate < min_rate) continue;
        if (sample_rate % rate != 0) continue;
        int64_t dist = target - rate;
        if (dist < 0) dist = -dist;
        if (dist < best_dist) {
            best_dist = dist;
            best = rate;
        }
    }
    return best > 0 ? best : target;
}

/* cmd/sdrd/helpers.go:292-310 snapOutRate: among the divisors d <= 256 of the
 * rate, the one closest to sr / target (float64 distance, first of equals);
 * sr / d, or the target when the inputs are not positive. */
int64_t or_snap_out_rate(int64_t sample_rate, int64_t target) {
    if (sample_rate <= 0 || target <= 0) return target;
    double ideal = (double)sample_rate / (double)target;
    int64_t best_d = 0;
    double best_err = 1.7976931348623157e308;
    for (int64_t d = 1; d <= 256 && d <= sample_rate; d++) {
        if (sample_rate % d != 0) continue;
        double e = fabs((double)d - ideal);
        if (e < best_err) {
            best_err = e;
            best_d = d;
        }
    }
    if (best_d < 1) return target;
    return sample_rate / best_d;
}

/* The WFM test shared by the job builders (streaming_refactor.go:27-28,
 * helpers.go:178,449): centre in the 87.5-108 MHz broadcast band, or a
 * classifier verdict of WFM / WFM_STEREO. */
static int job_is_wfm(double center_hz, int class_wfm) {
    double mhz = center_hz / 1e6;
    return (mhz >= 87.5 && mhz <= 108.0) || class_wfm;
}

/* cmd/sdrd/streaming_refactor.go:16-60 buildStreamingJobs, one signal:
 * bandwidth x bwMult (<= 0 means 1); WFM: out rate 512000 and bandwidth at
 * least 250000; others: nearestExactDecimationRate(sr, 200000, 128000) and
 * bandwidth at least 20000; taps = firTaps (<= 0 means 101); offset = centre
 * - tuner centre.  Returns 0, or -1 where ExactIntegerDecimation rejects the
 * out rate (the reference fails the whole batch). */
int or_streaming_job(int64_t sample_rate, double tuner_center_hz, double sig_center_hz, double sig_bw_hz,
                     int class_wfm, int fir_taps, double bw_mult, double *offset_hz, double *bw, int64_t *out_rate,
                     int *num_taps) {
    if (bw_mult <= 0) bw_mult = 1.0;
    if (fir_taps <= 0) fir_taps = 101;
    double b = sig_bw_hz * bw_mult;
    int64_t rate;
    if (job_is_wfm(sig_center_hz, class_wfm)) {
        rate = 512000;
        if (b < 250000) b = 250000;
    } else {
        rate = or_nearest_exact_decimation_rate(sample_rate, 200000, 128000);
        if (b < 20000) b = 20000;
    }
    if (sample_rate <= 0 || rate <= 0 || sample_rate % rate != 0) return -1;
    *offset_hz = sig_center_hz - tuner_center_hz;
    *bw = b;
    *out_rate = rate;
    *num_taps = fir_taps;
    return 0;
}

/* cmd/sdrd/helpers.go:174-194 extractSignalIQBatch, one signal's ExtractJob
 * for the batch runner: out rate snapOutRate(sr, 512000) for WFM, else
 * snapOutRate(sr, 200000); bandwidth floors 250000 (WFM) / 20000, no
 * multiplier. */
void or_batch_extract_job(int64_t sample_rate, double tuner_center_hz, double sig_center_hz, double sig_bw_hz,
                          int class_wfm, double *offset_hz, double *bw, int64_t *out_rate) {
    int wfm = job_is_wfm(sig_center_hz, class_wfm);
    double b = sig_bw_hz;
    if (wfm) {
        if (b < 250000) b = 250000;
    } else if (b < 20000) {
        b = 20000;
    }
    *offset_hz = sig_center_hz - tuner_center_hz;
    *bw = b;
    *out_rate = or_snap_out_rate(sample_rate, wfm ? 512000 : 200000);
}

/* cmd/sdrd/pipeline_runtime.go:1094-1101: the RDS extraction job's out rate,
 * ring rate / max(1, floor(ring rate / 250000)) (bandwidth 200000). */
int64_t or_rds_job_out_rate(int64_t ring_rate) {
    int64_t d = ring_rate / 250000;
    if (d < 1) d = 1;
    return ring_rate / d;
}

/* recorder/streamer.go:1098-1113 processSnippet's decim1: round(snip rate /
 * demod rate), at least 1; WFM forced to 2 when above 2 and snip rate / 2 >=
 * 200000.  Demod rates (OutputSampleRate in the demod package): WFM 192000, others
 * 48000. */
int or_snippet_decim(int64_t snip_rate, int64_t demod_rate, int wfm) {
    int64_t d = (int64_t)round((double)snip_rate / (double)demod_rate);
    if (d < 1) d = 1;
    if (wfm && d > 2 && snip_rate / 2 >= 200000) d = 2;
    return (int)d;
}

/* ------------------------------------------------------------------------ */
/* The single-signal Engine (internal/demod/gpudemod/gpudemod.go, Linux) and */
/* the legacy GPU batch slot (batch_runner_windows.go:142-182)               */
/* ------------------------------------------------------------------------ */

/* dsp.FreqShift (dsp/freqshift.go:6-23): phase from 0, incremented before
 * use, float64 cos/sin, products rounded once per component; a copy when the
 * offset is 0. */
static void freq_shift_go(const cf32 *iq, int n, int fs, double offset, cf32 *out) {
    if (n <= 0) return;
    if (fs <= 0 || offset == 0) {
        memcpy(out, iq, sizeof(cf32) * (size_t)n);
        return;
    }
    double phase = 0.0;
    double inc = -2 * OR_PI * offset / (double)fs;
    for (int i = 0; i < n; i++) {
        phase += inc;
        double re = cos(phase), im = sin(phase);
        double vr = iq[i].re, vi = iq[i].im;
        out[i].re = (float)(vr * re - vi * im);
        out[i].im = (float)(vr * im + vi * re);
    }
}

/* dsp.Decimate(dsp.ApplyFIR(dsp.FreqShift(iq, fs, offset), taps), decim)
 * (gpudemod.go:336-350; dsp/fir.go:31-95): zero-history FIR with float64
 * accumulation, every decim-th output from index 0 (ceil(n/decim) of them;
 * all n when decim <= 1).  Returns the count. */
int or_shift_filter_decimate(const cf32 *iq, int n, int fs, double offset, const double *taps, int nt, int decim,
                             cf32 *out) {
    if (n <= 0 || nt <= 0) return 0;
    if (decim < 1) decim = 1;
    cf32 *sh = (cf32 *)malloc(sizeof(cf32) * (size_t)n);
    freq_shift_go(iq, n, fs, offset, sh);
    int cnt = 0;
    for (int i = 0; i < n; i += decim) {
        double ar = 0, ai = 0;
        for (int k = 0; k < nt; k++) {
            int idx = i - k;
            if (idx < 0) break;
            ar += (double)sh[idx].re * taps[k];
            ai += (double)sh[idx].im * taps[k];
        }
        out[cnt].re = (float)ar;
        out[cnt].im = (float)ai;
        cnt++;
    }
    free(sh);
    return cnt;
}

/* Engine.ShiftFilterDecimate (gpudemod.go:325-350): cutoff = BW/2 clamped to
 * [200, fs/2 - 1], 101-tap LowpassFIR, decimation round(fs / out_rate) >= 1.
 * Returns the count (-1 for a non-positive out rate); *rate = fs / decim. */
int or_engine_shift_filter_decimate(const cf32 *iq, int n, int fs, double offset, double bw, int out_rate,
                                    cf32 *out, int *rate) {
    *rate = 0;
    if (n <= 0) return 0;
    if (out_rate <= 0) return -1;
    double cutoff = bw / 2;
    if (cutoff < 200) cutoff = 200;
    if (cutoff > (double)fs / 2 - 1) cutoff = (double)fs / 2 - 1;
    double taps[101];
    or_lowpass_fir(cutoff, fs, 101, taps);
    int decim = (int)round((double)fs / (double)out_rate);
    if (decim < 1) decim = 1;
    *rate = fs / decim;
    return or_shift_filter_decimate(iq, n, fs, offset, taps, 101, decim, out);
}

/* Engine state across Demod calls (gpudemod.go:81-100): the FIR taps set on
 * the first call (float32, at most 256) and the BFO phase of the SSB/CW
 * product. */
typedef struct {
    int fs;
    int nfir;
    float fir[256];
    double bfo_phase;
} or_engine;

size_t or_engine_size(void) { return sizeof(or_engine); }
void or_engine_init(or_engine *e, int fs) {
    memset(e, 0, sizeof *e);
    e->fs = fs;
}

/* Engine.Demod (gpudemod.go:352-461) with the CUDA engine ready.  The shift,
 * FIR and decimation stages take the results the reference keeps after its
 * CPU comparison (ValidateFreqShift / ValidateFIR / ValidateDecimate,
 * gpudemod.go:368-427): dsp.FreqShift from phase 0, the FIR with the first
 * call's float32 taps (LowpassFIR(max(BW/2, 200), fs, 101)) accumulated in
 * float64, dsp.Decimate by round(fs / rate), rate 192000 for WFM and 48000
 * otherwise.  The demodulator is the GPU launcher the reference returns
 * unchecked: the discriminator (n-1 outputs; float64 products and atan2 as
 * the CPU path), the AM envelope without mean removal (exports.cu K6), the
 * BFO product re*cos - im*sin with phase bfo_phase + i*inc and inc =
 * 2 pi bfo / fs at the engine's full rate (gpudemod.go:296-318; BFO +700 Hz
 * for USB and CW, -700 Hz for LSB), bfo_phase advanced by inc * count.
 * mode: 0 NFM, 1 WFM, 2 AM, 3 USB, 4 LSB, 5 CW (DemodType).  Returns the
 * audio count, *rate the demod input rate; -1 for an unknown mode. */
int or_engine_demod(or_engine *e, const cf32 *iq, int n, double offset, double bw, int mode, float *audio,
                    int *rate) {
    *rate = 0;
    if (n <= 0) return 0;
    if (mode < 0 || mode > 5) return -1;
    int out_rate = mode == 1 ? 192000 : 48000;
    double cutoff = bw / 2;
    if (cutoff < 200) cutoff = 200;
    if (e->nfir == 0) {
        double t64[101];
        or_lowpass_fir(cutoff, e->fs, 101, t64);
        for (int k = 0; k < 101; k++) e->fir[k] = (float)t64[k];
        e->nfir = 101;
    }
    double taps[256];
    for (int k = 0; k < e->nfir; k++) taps[k] = (double)e->fir[k];
    int decim = (int)round((double)e->fs / (double)out_rate);
    if (decim < 1) decim = 1;
    int m = (n + decim - 1) / decim;
    cf32 *dec = (cf32 *)malloc(sizeof(cf32) * (size_t)m);
    m = or_shift_filter_decimate(iq, n, e->fs, offset, taps, e->nfir, decim, dec);
    *rate = e->fs / decim;
    int cnt = 0;
    if (mode == 0 || mode == 1) {
        if (m >= 2) cnt = or_fm_discrim(dec, m, audio);
    } else if (mode == 2) {
        for (int i = 0; i < m; i++) {
            double x = dec[i].re, y = dec[i].im;
            audio[i] = (float)sqrt(x * x + y * y);
        }
        cnt = m;
    } else {
        double bfo = mode == 4 ? -700.0 : 700.0;
        double inc = 2.0 * OR_PI * bfo / (double)e->fs;
        for (int i = 0; i < m; i++) {
            double ph = e->bfo_phase + inc * (double)i;
            ph -= rint(ph / 6.283185307179586) * 6.283185307179586;
            audio[i] = (float)((double)dec[i].re * cos(ph) - (double)dec[i].im * sin(ph));
        }
        e->bfo_phase += inc * (double)m;
        cnt = m;
    }
    free(dec);
    return cnt;
}

/* One slot of the legacy GPU batch (batch_runner_windows.go:142-182,
 * shiftFilterDecimateSlotParallel): 101-tap LowpassFIR(max(BW/2, 200), fs)
 * as float32, exact integer decimation, the shift K1 with phase
 * phase_start + i*inc (inc = -2 pi offset / fs, no pre-increment), the
 * zero-history FIR K5 and the decimation K3: n / decim outputs,
 * out[j] = filtered[j*decim].  Returns the count, -1 when fs / out_rate is
 * not an integer, -2 when no output remains; *rate = fs / decim; *phase_end
 * = phase_start + inc * n (batch_runner.go:83-88). */
int or_batch_slot(const cf32 *iq, int n, int fs, double offset, double bw, int out_rate, double phase_start,
                  cf32 *out, int *rate, double *phase_end) {
    double cutoff = bw / 2;
    if (cutoff < 200) cutoff = 200;
    double t64[101];
    or_lowpass_fir(cutoff, fs, 101, t64);
    double taps[101];
    for (int k = 0; k < 101; k++) taps[k] = (double)(float)t64[k];
    if (fs <= 0 || out_rate <= 0 || fs % out_rate != 0) return -1;
    int decim = fs / out_rate;
    int nout = n / decim;
    if (nout <= 0) return -2;
    double inc = -2.0 * OR_PI * offset / (double)fs;
    *rate = fs / decim;
    *phase_end = phase_start + inc * (double)n;
    for (int j = 0; j < nout; j++) {
        int i = j * decim;
        double ar = 0, ai = 0;
        for (int k = 0; k < 101 && i - k >= 0; k++) {
            int idx = i - k;
            double ph = phase_start + inc * (double)idx;
            ph -= rint(ph / 6.283185307179586) * 6.283185307179586;
            double c = cos(ph), s = sin(ph);
            double vr = iq[idx].re, vi = iq[idx].im;
            float sr = (float)(vr * c - vi * s), si = (float)(vr * s + vi * c);
            ar += (double)sr * taps[k];
            ai += (double)si * taps[k];
        }
        out[j].re = (float)ar;
        out[j].im = (float)ai;
    }
    return nout;
}

// rds.cu -- RDS symbol and group decoder on the device (internal/rds/rds.go:
// 78-636, rds.Decoder.Decode) for a batch of stations, one CTA per station.
//
// The reference runs the decoder once per RDS window of each broadcast
// station (cmd/sdrd/pipeline_runtime.go:1137).  Per call: Mueller-Muller
// symbol timing with linear interpolation (sps = fs / 1187.5, gain 0.01),
// a Costas loop (alpha 0.132, beta alpha^2/4) with sign decisions, differential
// decoding against the previous call's last decision, then the block / group
// search of tryDecode: every start offset is tried with one-bit error
// correction (a block is corrected only when exactly one flip gives an
// allowed offset word), a flywheel keeps consecutive groups in step (+-3 bits),
// and when the bits yield no group the inverted bits are tried.  Timing,
// loop and differential state carry across calls; the group search stays
// inside one call's bits.
//
// On the device the timing and loop recurrences run serially in one thread
// (they are sequential by definition); the expensive part of the search --
// decoding a 104-bit group at every start offset, each block with up to 26
// trial flips -- runs over all offsets in parallel into a table, and the
// flywheel walk then only looks entries up.  Arithmetic follows the
// reference's operation order with explicit roundings (no contraction), so
// decisions, groups, PI, PS and RT equal the CPU path's.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpudemod.h"

extern "C" void gpud_count_launch(int n);

namespace {

constexpr int kRdsThreads = 256;
constexpr uint16_t kOffA = 0x0FC, kOffB = 0x198, kOffC = 0x168, kOffCp = 0x350, kOffD = 0x1B4;
constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
constexpr double kPi = 3.14159265358979323846;

// Per-station decoder state (the fields of rds.Decoder that feed decoding).
struct RdsState {
    char ps[8];
    char rt[64];
    uint16_t last_pi;
    uint16_t pad0;
    int32_t last_sample_rate;
    double costas_phase, costas_freq, sync_mu;
    float2 sync_prev, sync_prev_dec;
    int32_t sync_has_prev, last_hard_bit, has_last_hard_bit;
    int32_t total_decodes, groups_found_calls, groups_total;
};

struct RdsJobDev {
    const float2 *s;
    int32_t n, fs, station, pad;
    int64_t off;  // scratch offset (samples)
};

struct RdsOut {
    int32_t groups, groups_total, status, pad;
};

// crcSyndrome (rds.go:590-599), the reference's reduction exactly.
__device__ __forceinline__ uint32_t rds_syndrome(uint32_t raw) {
    uint32_t reg = raw;
#pragma unroll
    for (int i = 25; i >= 10; --i)
        if ((reg >> i) & 1u) reg ^= 0x1B9u << (i - 10);
    return reg & 0x3FFu;
}

// decodeBlockExpected (rds.go:538-576) for one allowed offset set: 0 = A,
// 1 = B, 2 = C or C', 3 = D.
__device__ __forceinline__ bool rds_allowed(uint32_t s, int which) {
    switch (which) {
    case 0: return s == kOffA;
    case 1: return s == kOffB;
    case 2: return s == kOffC || s == kOffCp;
    default: return s == kOffD;
    }
}

__device__ __forceinline__ bool rds_valid_offset(uint32_t s) {
    return s == kOffA || s == kOffB || s == kOffC || s == kOffCp || s == kOffD;
}

__device__ bool rds_block(const uint8_t *bits, bool inv, int which, uint16_t *data) {
    uint32_t raw = 0;
    for (int i = 0; i < 26; ++i) raw = (raw << 1) | ((uint32_t)(bits[i] ^ (inv ? 1 : 0)) & 1u);
    const uint32_t s = rds_syndrome(raw);
    if (rds_valid_offset(s) && rds_allowed(s, which)) {
        *data = (uint16_t)(raw >> 10);
        return true;
    }
    int count = 0;
    uint16_t cand = 0;
    for (int i = 0; i < 26; ++i) {
        const uint32_t f = raw ^ (1u << (25 - i));
        const uint32_t sf = rds_syndrome(f);
        if (!rds_valid_offset(sf) || !rds_allowed(sf, which)) continue;
        cand = (uint16_t)(f >> 10);
        if (++count > 1) return false;
    }
    if (count == 1) {
        *data = cand;
        return true;
    }
    return false;
}

__device__ char rds_sanitize(uint32_t b) { return (b < 32 || b > 126) ? ' ' : (char)b; }

// applyGroup (rds.go:477-502)
__device__ void rds_apply(RdsState &d, uint64_t g) {
    const uint16_t g0 = (uint16_t)g, g1 = (uint16_t)(g >> 16), g2 = (uint16_t)(g >> 32), g3 = (uint16_t)(g >> 48);
    if (g0 != 0) d.last_pi = g0;
    const int gtype = (g1 >> 12) & 0xF;
    const bool va = ((g1 >> 11) & 1) == 0;
    if (gtype == 0 && va) {
        const int idx = (g1 & 0x3) * 2;
        d.ps[idx] = rds_sanitize(g3 >> 8);
        d.ps[idx + 1] = rds_sanitize(g3 & 0xFF);
    }
    if (gtype == 2 && va) {
        const int idx = (g1 & 0xF) * 4;
        const uint32_t ch[4] = {(uint32_t)(g2 >> 8), (uint32_t)(g2 & 0xFF), (uint32_t)(g3 >> 8), (uint32_t)(g3 & 0xFF)};
        for (int j = 0; j < 4 && idx + j < 64; ++j) d.rt[idx + j] = rds_sanitize(ch[j]);
    }
}

// tryDecode's flywheel walk (rds.go:365-430) over the table of group decodes.
__device__ int rds_walk(RdsState &d, const uint8_t *ok, const uint64_t *grp, int nbits) {
    int groups = 0;
    auto at = [&](int s) { return s >= 0 && s + 104 <= nbits && ok[s]; };
    for (int i = 0; i + 104 <= nbits;) {
        if (!ok[i]) {
            i++;
            continue;
        }
        groups++;
        rds_apply(d, grp[i]);
        int next = i + 104;
        bool locked = true;
        while (locked && next + 104 <= nbits) {
            if (at(next)) {
                rds_apply(d, grp[next]);
                groups++;
                next += 104;
                continue;
            }
            bool matched = false;
            for (int delta = 1; delta <= 3 && !matched; ++delta) {
                const int left = next - delta;
                if (at(left)) {
                    rds_apply(d, grp[left]);
                    groups++;
                    next = left + 104;
                    matched = true;
                    break;
                }
                const int right = next + delta;
                if (at(right)) {
                    rds_apply(d, grp[right]);
                    groups++;
                    next = right + 104;
                    matched = true;
                    break;
                }
            }
            if (!matched) locked = false;
        }
        int resume = next - 3;
        if (resume <= i) resume = i + 1;
        i = resume;
    }
    return groups;
}

// Every start offset's group decode (decodeGroupAt, rds.go:432-475), in parallel.
__device__ void rds_table(const uint8_t *bits, int nbits, bool inv, uint8_t *ok, uint64_t *grp) {
    for (int i = threadIdx.x; i + 104 <= nbits; i += kRdsThreads) {
        uint16_t g[4];
        bool good = true;
        for (int b = 0; b < 4 && good; ++b) good = rds_block(bits + i + 26 * b, inv, b, &g[b]);
        ok[i] = good ? 1 : 0;
        grp[i] = good ? ((uint64_t)g[0] | ((uint64_t)g[1] << 16) | ((uint64_t)g[2] << 32) | ((uint64_t)g[3] << 48)) : 0;
    }
}

__global__ void __launch_bounds__(kRdsThreads)
k_rds_decode(const RdsJobDev *__restrict__ jobs, RdsState *__restrict__ states, float2 *__restrict__ sym_s,
             uint8_t *__restrict__ bits_s, uint8_t *__restrict__ ok_s, uint64_t *__restrict__ grp_s, int cap,
             RdsOut *__restrict__ out) {
    __shared__ int s_nb, s_go, s_groups;
    const RdsJobDev jb = jobs[blockIdx.x];
    RdsState &d = states[jb.station];
    float2 *sym = sym_s + jb.off;
    uint8_t *bits = bits_s + jb.off;
    uint8_t *ok = ok_s + jb.off;
    uint64_t *grp = grp_s + jb.off;
    RdsOut o{0, 0, 0, 0};
    if (threadIdx.x == 0) {
        s_go = 0;
        s_nb = 0;
        const int n = jb.n, fs = jb.fs;
        if (n >= 104 && fs > 0) {
            d.total_decodes++;
            if (d.last_sample_rate != 0 && d.last_sample_rate != fs) {
                d.costas_phase = d.costas_freq = d.sync_mu = 0.0;
                d.sync_prev = d.sync_prev_dec = make_float2(0.f, 0.f);
                d.sync_has_prev = d.last_hard_bit = d.has_last_hard_bit = 0;
            }
            d.last_sample_rate = fs;
            // Mueller-Muller timing (rds.go:109-160)
            const double sps = (double)fs / 1187.5;
            double mu = d.sync_mu;
            if (mu < 0 || mu >= sps || isnan(mu) || isinf(mu)) mu = sps / 2;
            float2 prev = d.sync_prev, prev_dec = d.sync_prev_dec;
            int have_prev = d.sync_has_prev, ns = 0;
            while (mu < (double)(n - 1)) {
                const int idx = (int)mu;
                const double frac = __dsub_rn(mu, (double)idx);
                if (idx + 1 >= n) break;
                if (ns >= cap) {  // a timing loop that no longer advances: stop, report
                    o.status = 1;
                    break;
                }
                const float2 a = jb.s[idx], b = jb.s[idx + 1];
                const double w0 = __dsub_rn(1.0, frac);
                float2 sm;
                sm.x = (float)__dadd_rn(__dmul_rn((double)a.x, w0), __dmul_rn((double)b.x, frac));
                sm.y = (float)__dadd_rn(__dmul_rn((double)a.y, w0), __dmul_rn((double)b.y, frac));
                const float2 dec = make_float2(sm.x >= 0.f ? 1.0f : -1.0f, 0.0f);
                if (have_prev) {
                    const double er = __dsub_rn(__dmul_rn((double)__fsub_rn(dec.x, prev_dec.x), (double)prev.x),
                                                __dmul_rn((double)__fsub_rn(sm.x, prev.x), (double)prev_dec.x));
                    mu = __dadd_rn(mu, __dadd_rn(sps, __dmul_rn(0.01, er)));
                } else {
                    mu = __dadd_rn(mu, sps);
                    have_prev = 1;
                }
                prev_dec = dec;
                prev = sm;
                sym[ns++] = sm;
            }
            double res = __dsub_rn(mu, (double)n);
            if (o.status) {
                res = sps / 2;
            } else {
                for (int g = 0; g < 64 && res < 0; ++g) res = __dadd_rn(res, sps);
                for (int g = 0; g < 64 && res >= sps; ++g) res = __dsub_rn(res, sps);
            }
            d.sync_mu = res;
            d.sync_prev = prev;
            d.sync_prev_dec = prev_dec;
            d.sync_has_prev = have_prev;
            if (ns >= 104) {
                // Costas loop and sign decisions (rds.go:162-206)
                const double alpha = 0.132, beta = alpha * alpha / 4.0;
                double phase = d.costas_phase, freq = d.costas_freq;
                uint8_t last = 0;
                for (int i = 0; i < ns; ++i) {
                    const float cp = (float)cos(phase), sp = (float)sin(phase);
                    const float2 s = sym[i];
                    const float yr = __fadd_rn(__fmul_rn(s.x, cp), __fmul_rn(s.y, sp));
                    const float yi = __fsub_rn(__fmul_rn(s.y, cp), __fmul_rn(s.x, sp));
                    const double err = yr >= 0.f ? (double)yi : -(double)yi;
                    freq = __dadd_rn(freq, __dmul_rn(beta, err));
                    phase = __dadd_rn(phase, __dadd_rn(freq, __dmul_rn(alpha, err)));
                    int g = 0;
                    for (; g < 64 && phase > kPi; ++g) phase = __dsub_rn(phase, kTwoPi);
                    for (; g < 64 && phase < -kPi; ++g) phase = __dadd_rn(phase, kTwoPi);
                    if (g == 64) phase = remainder(phase, kTwoPi);  // diverged loop: no endless wrap
                    const uint8_t h = yr >= 0.f ? 1 : 0;
                    // differential decoding (rds.go:208-230)
                    if (i == 0) {
                        if (d.has_last_hard_bit) bits[s_nb++] = h ^ (uint8_t)d.last_hard_bit;
                    } else {
                        bits[s_nb++] = h ^ last;
                    }
                    last = h;
                }
                d.costas_phase = phase;
                d.costas_freq = freq;
                d.last_hard_bit = last;
                d.has_last_hard_bit = 1;
                s_go = 1;
            }
        }
    }
    __syncthreads();
    if (s_go) {
        const int nb = s_nb;
        rds_table(bits, nb, false, ok, grp);
        __syncthreads();
        if (threadIdx.x == 0) {
            s_groups = rds_walk(d, ok, grp, nb);
            s_go = s_groups == 0 ? 2 : 1;
        }
        __syncthreads();
        if (s_go == 2) {  // no group in the bits: the inverted bits (rds.go:246-251)
            rds_table(bits, nb, true, ok, grp);
            __syncthreads();
            if (threadIdx.x == 0) s_groups = rds_walk(d, ok, grp, nb);
        }
    }
    if (threadIdx.x == 0) {
        o.groups = s_go ? s_groups : 0;
        if (o.groups > 0) d.groups_found_calls++;
        d.groups_total += o.groups;
        o.groups_total = d.groups_total;
        out[blockIdx.x] = o;
    }
}

}  // namespace

struct gpud_rds_decoder {
    int max_stations = 0, max_samples = 0, cap = 0;
    RdsState *d_state = nullptr;
    RdsJobDev *d_jobs = nullptr;
    RdsOut *d_out = nullptr;
    float2 *d_sym = nullptr;
    uint8_t *d_bits = nullptr, *d_ok = nullptr;
    uint64_t *d_grp = nullptr;
    std::vector<RdsJobDev> jobs;
    std::vector<RdsOut> outs;
    std::vector<RdsState> states;
};

extern "C" {

GPUD_API int GPUD_CALL gpud_rds_decoder_destroy(gpud_rds_decoder *r) {
    if (!r) return 0;
    cudaFree(r->d_state);
    cudaFree(r->d_jobs);
    cudaFree(r->d_out);
    cudaFree(r->d_sym);
    cudaFree(r->d_bits);
    cudaFree(r->d_ok);
    cudaFree(r->d_grp);
    delete r;
    return 0;
}

GPUD_API int GPUD_CALL gpud_rds_decoder_create(int max_stations, int max_samples, gpud_rds_decoder **out) {
    if (!out || max_stations <= 0 || max_samples < 104) return GPUD_E_ARG;
    auto *r = new gpud_rds_decoder();
    r->max_stations = max_stations;
    r->max_samples = max_samples;
    r->cap = max_samples + 8;  // symbols, bits and table entries per station and call
    const size_t slots = (size_t)max_stations * (size_t)r->cap;
    bool ok = cudaMalloc((void **)&r->d_state, sizeof(RdsState) * (size_t)max_stations) == cudaSuccess &&
              cudaMalloc((void **)&r->d_jobs, sizeof(RdsJobDev) * (size_t)max_stations) == cudaSuccess &&
              cudaMalloc((void **)&r->d_out, sizeof(RdsOut) * (size_t)max_stations) == cudaSuccess &&
              cudaMalloc((void **)&r->d_sym, sizeof(float2) * slots) == cudaSuccess &&
              cudaMalloc((void **)&r->d_bits, slots) == cudaSuccess &&
              cudaMalloc((void **)&r->d_ok, slots) == cudaSuccess &&
              cudaMalloc((void **)&r->d_grp, sizeof(uint64_t) * slots) == cudaSuccess &&
              cudaMemset(r->d_state, 0, sizeof(RdsState) * (size_t)max_stations) == cudaSuccess;
    if (!ok) {
        gpud_rds_decoder_destroy(r);
        return GPUD_E_CUDA;
    }
    r->states.resize((size_t)max_stations);
    *out = r;
    return 0;
}

GPUD_API int GPUD_CALL gpud_rds_decoder_reset(gpud_rds_decoder *r, int station) {
    if (!r || station < 0 || station >= r->max_stations) return GPUD_E_ARG;
    return cudaMemset(r->d_state + station, 0, sizeof(RdsState)) == cudaSuccess ? 0 : GPUD_E_CUDA;
}

GPUD_API int GPUD_CALL gpud_rds_decode_run(gpud_rds_decoder *r, const gpud_rds_job *jobs, int count,
                                           gpud_stream_handle stream, gpud_rds_result *results) {
    if (!r || count < 0 || count > r->max_stations || (count > 0 && (!jobs || !results))) return GPUD_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    r->jobs.resize((size_t)count);
    std::vector<char> seen((size_t)r->max_stations, 0);
    for (int j = 0; j < count; ++j) {
        const gpud_rds_job &q = jobs[j];
        if (q.station < 0 || q.station >= r->max_stations || seen[(size_t)q.station]) return GPUD_E_ARG;
        if (q.n < 0 || q.n > r->max_samples || (q.n > 0 && !q.samples)) return GPUD_E_ARG;
        seen[(size_t)q.station] = 1;
        r->jobs[(size_t)j] = RdsJobDev{reinterpret_cast<const float2 *>(q.samples), q.n, q.sample_rate, q.station, 0,
                                       (int64_t)j * r->cap};
    }
    if (count == 0) return 0;
    if (cudaMemcpyAsync(r->d_jobs, r->jobs.data(), sizeof(RdsJobDev) * (size_t)count, cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
        return GPUD_E_CUDA;
    k_rds_decode<<<count, kRdsThreads, 0, s>>>(r->d_jobs, r->d_state, r->d_sym, r->d_bits, r->d_ok, r->d_grp, r->cap,
                                               r->d_out);
    if (cudaGetLastError() != cudaSuccess) return GPUD_E_CUDA;
    gpud_count_launch(1);
    r->outs.resize((size_t)count);
    if (cudaMemcpyAsync(r->outs.data(), r->d_out, sizeof(RdsOut) * (size_t)count, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaMemcpyAsync(r->states.data(), r->d_state, sizeof(RdsState) * (size_t)r->max_stations,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GPUD_E_CUDA;
    for (int j = 0; j < count; ++j) {
        const RdsOut &o = r->outs[(size_t)j];
        const RdsState &st = r->states[(size_t)jobs[j].station];
        gpud_rds_result &res = results[j];
        std::memset(&res, 0, sizeof res);
        res.groups = o.groups;
        res.groups_total = o.groups_total;
        res.status = o.status;
        res.pi = st.last_pi;
        // psString / rtString (rds.go:603-636): zero bytes as spaces, trailing spaces trimmed
        int end = 8;
        for (int i = 0; i < 8; ++i) res.ps[i] = st.ps[i] ? st.ps[i] : ' ';
        while (end > 0 && res.ps[end - 1] == ' ') --end;
        res.ps[end] = 0;
        end = 64;
        for (int i = 0; i < 64; ++i) res.rt[i] = st.rt[i] ? st.rt[i] : ' ';
        while (end > 0 && res.rt[end - 1] == ' ') --end;
        res.rt[end] = 0;
    }
    return 0;
}

}  // extern "C"

// pilot.cu -- long-window stereo pilot detector on the device.
//
// classifier.StereoPilotPresent / estimateWFMPilot (internal/classifier/
// pll.go:75-131, 170-196): float64 FM discriminator of an FM-multiplex
// baseband, magnitude of its spectrum at 201 frequencies 19 kHz +- 1 kHz in
// 10 Hz steps (the reference runs one Goertzel recurrence per frequency), a
// stereo pilot when the largest magnitude exceeds `threshold` times the median
// (4.0 in the reference, SDRD_PILOT_RATIO overrides it there).
//
// Every analysis frequency f is a multiple of 10 Hz, so exp(-j 2 pi f i / fs)
// repeats with period P = fs / gcd(fs, 10) in i.  The discriminator output is
// folded modulo P once (y[m] = sum of d[m + pP]) and the 201 bins are direct
// float64 DFT sums of y over [0, P) with twiddles from a table of the P-th
// roots of unity (exact sincospi arguments): the Goertzel magnitudes without
// the Goertzel recurrence's error growth, one CTA per (job, bin), and the
// max / median decision on the device.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gpudemod.h"

extern "C" void gpud_count_launch(int n);

namespace {

constexpr int kBins = 201;
constexpr int kPilotThreads = 256;
constexpr int64_t kMaxTable = 1 << 20;  // roots-of-unity table entries (16 MiB)

struct PilotJob {
    const float2 *iq;  // first sample of the analysed window
    int32_t nd;        // discriminator samples (window length - 1)
    int32_t fs;
    int32_t period;    // P = fs / gcd(fs, 10)
    int32_t folded;    // min(P, nd)
    int32_t fstep;     // 10 / gcd(fs, 10): table index step per 10 Hz of frequency
    int32_t table;     // 1: twiddles from the table, 0: sincospi per term
    int64_t y_off;     // offset of this job's folded vector
};

// fmDemod (pll.go:170-183): float64 products of the float32 samples, atan2.
__device__ __forceinline__ double pilot_disc(const float2 *iq, int i) {
    const float2 p = iq[i], c = iq[i + 1];
    const double num = (double)p.x * (double)c.y - (double)p.y * (double)c.x;
    const double den = (double)p.x * (double)c.x + (double)p.y * (double)c.y;
    return atan2(num, den);
}

__global__ void __launch_bounds__(kPilotThreads)
k_pilot_fold(const PilotJob *__restrict__ jobs, double *__restrict__ y) {
    const PilotJob jb = jobs[blockIdx.y];
    for (int m = blockIdx.x * kPilotThreads + threadIdx.x; m < jb.folded; m += gridDim.x * kPilotThreads) {
        double acc = 0.0;
        for (int i = m; i < jb.nd; i += jb.period) acc += pilot_disc(jb.iq, i);
        y[jb.y_off + m] = acc;
    }
}

// tab[a] = exp(j 2 pi a / P), a < P
__global__ void k_pilot_table(int P, double2 *__restrict__ tab) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < P; a += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)a / (double)P, &s, &c);
        tab[a] = make_double2(c, s);
    }
}

__global__ void __launch_bounds__(kPilotThreads)
k_pilot_bins(const PilotJob *__restrict__ jobs, const double *__restrict__ y, const double2 *__restrict__ tab,
             double *__restrict__ mags) {
    __shared__ double s_re[kPilotThreads / 32], s_im[kPilotThreads / 32];
    const PilotJob jb = jobs[blockIdx.y];
    const int bin = blockIdx.x;
    const int64_t fq = (int64_t)(1800 + bin) * jb.fstep;  // f / gcd(fs, 10), f = 18000 + 10*bin
    const int P = jb.period;
    const int per = (jb.folded + kPilotThreads - 1) / kPilotThreads;
    const int m0 = min(jb.folded, (int)threadIdx.x * per), m1 = min(jb.folded, m0 + per);
    const double *ym = y + jb.y_off;
    double re = 0.0, im = 0.0;
    if (m0 < m1) {
        int64_t a = (fq * (int64_t)m0) % P;  // index of exp(j 2 pi f m / fs) among the P-th roots
        for (int m = m0; m < m1; ++m) {
            double2 w;
            if (jb.table) {
                w = tab[a];
            } else {
                double s, c;
                sincospi(2.0 * (double)a / (double)P, &s, &c);
                w = make_double2(c, s);
            }
            re = fma(ym[m], w.x, re);
            im = fma(ym[m], w.y, im);
            a += fq;
            if (a >= P) a -= P;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, off);
        im += __shfl_xor_sync(0xffffffffu, im, off);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_re[warp] = re;
        s_im[warp] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0, i = 0.0;
        for (int w = 0; w < kPilotThreads / 32; ++w) {
            r += s_re[w];
            i += s_im[w];
        }
        mags[(int64_t)blockIdx.y * kBins + bin] = sqrt(r * r + i * i);
    }
}

// max (first occurrence, as the reference's strict '>' scan from 0) and the
// median (element 100 of the sorted 201) of each job's magnitudes
__global__ void __launch_bounds__(kPilotThreads)
k_pilot_decide(const double *__restrict__ mags, double threshold, gpud_pilot_result *__restrict__ out) {
    __shared__ double s_m[kBins], s_sorted[kBins];
    const double *m = mags + (int64_t)blockIdx.x * kBins;
    for (int i = threadIdx.x; i < kBins; i += kPilotThreads) s_m[i] = m[i];
    __syncthreads();
    for (int i = threadIdx.x; i < kBins; i += kPilotThreads) {
        int rank = 0;
        for (int j = 0; j < kBins; ++j) rank += (s_m[j] < s_m[i]) || (s_m[j] == s_m[i] && j < i);
        s_sorted[rank] = s_m[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double best = 0.0;
        int bb = -1;
        for (int i = 0; i < kBins; ++i)
            if (s_m[i] > best) {
                best = s_m[i];
                bb = i;
            }
        const double med = s_sorted[kBins / 2];
        gpud_pilot_result r{};
        r.best_bin = bb < 0 ? 100 : bb;
        r.best_hz = 18000.0 + 10.0 * (double)r.best_bin;
        r.median = med;
        r.ratio = med > 0 ? best / med : 0.0;
        r.present = (med > 0 && r.ratio > threshold) ? 1 : 0;
        out[blockIdx.x] = r;
    }
}

}  // namespace

struct gpud_pilot {
    int max_jobs = 0, max_samples = 0;
    double *d_y = nullptr, *d_mags = nullptr;
    double2 *d_tab = nullptr;
    int tab_period = 0;  // period the table currently holds
    PilotJob *d_jobs = nullptr;
    gpud_pilot_result *d_res = nullptr;
    std::vector<PilotJob> jobs;
    std::vector<int> job_of;  // job index -> index into the device list (-1: no decision possible)
};

extern "C" {

GPUD_API int GPUD_CALL gpud_pilot_create(int max_jobs, int max_samples, gpud_pilot **out) {
    if (!out || max_jobs <= 0 || max_samples <= 1) return GPUD_E_ARG;
    auto *p = new gpud_pilot();
    p->max_jobs = max_jobs;
    p->max_samples = max_samples;
    bool ok = cudaMalloc((void **)&p->d_y, sizeof(double) * (size_t)max_jobs * (size_t)max_samples) == cudaSuccess &&
              cudaMalloc((void **)&p->d_mags, sizeof(double) * (size_t)max_jobs * kBins) == cudaSuccess &&
              cudaMalloc((void **)&p->d_tab, sizeof(double2) * (size_t)kMaxTable) == cudaSuccess &&
              cudaMalloc((void **)&p->d_jobs, sizeof(PilotJob) * (size_t)max_jobs) == cudaSuccess &&
              cudaMalloc((void **)&p->d_res, sizeof(gpud_pilot_result) * (size_t)max_jobs) == cudaSuccess;
    if (!ok) {
        gpud_pilot_destroy(p);
        return GPUD_E_CUDA;
    }
    *out = p;
    return 0;
}

GPUD_API int GPUD_CALL gpud_pilot_destroy(gpud_pilot *p) {
    if (!p) return 0;
    cudaFree(p->d_y);
    cudaFree(p->d_mags);
    cudaFree(p->d_tab);
    cudaFree(p->d_jobs);
    cudaFree(p->d_res);
    delete p;
    return 0;
}

GPUD_API int GPUD_CALL gpud_pilot_run(gpud_pilot *p, const gpud_pilot_job *jobs, int count, double threshold,
                                      gpud_stream_handle stream, gpud_pilot_result *results) {
    if (!p || count < 0 || count > p->max_jobs || (count > 0 && (!jobs || !results))) return GPUD_E_ARG;
    if (threshold <= 0) threshold = 4.0;
    cudaStream_t s = (cudaStream_t)stream;
    p->jobs.clear();
    p->job_of.assign((size_t)count, -1);
    std::vector<int> periods;
    for (int j = 0; j < count; ++j) {
        const gpud_pilot_job &q = jobs[j];
        results[j] = gpud_pilot_result{};
        results[j].best_hz = 19000.0;
        results[j].best_bin = 100;
        int n = q.n, start = 0;
        if (!q.iq || n < 0) return GPUD_E_ARG;
        if (q.window) {  // StereoPilotPresent: the last sample_rate/2 samples
            const int mx = q.sample_rate / 2;
            if (mx > 0 && n > mx) {
                start = n - mx;
                n = mx;
            }
        }
        if (n > p->max_samples) return GPUD_E_ARG;
        if (q.sample_rate < 40000 || n < 2) continue;  // the reference returns unlocked
        PilotJob jb{};
        const int g = std::gcd(q.sample_rate, 10);
        jb.iq = reinterpret_cast<const float2 *>(q.iq) + start;
        jb.nd = n - 1;
        jb.fs = q.sample_rate;
        jb.period = q.sample_rate / g;
        jb.folded = std::min(jb.period, jb.nd);
        jb.fstep = 10 / g;
        jb.table = jb.period <= kMaxTable ? 1 : 0;
        jb.y_off = (int64_t)p->jobs.size() * p->max_samples;
        p->job_of[(size_t)j] = (int)p->jobs.size();
        p->jobs.push_back(jb);
        if (jb.table) periods.push_back(jb.period);
    }
    const int nj = (int)p->jobs.size();
    if (nj == 0) return 0;
    // one roots-of-unity table per call: jobs with another period use sincospi
    int tp = 0;
    if (!periods.empty()) {
        std::sort(periods.begin(), periods.end());
        int best = 0, cnt = 0;
        for (size_t i = 0; i < periods.size(); ++i) {
            cnt = (i > 0 && periods[i] == periods[i - 1]) ? cnt + 1 : 1;
            if (cnt > best) {
                best = cnt;
                tp = periods[i];
            }
        }
    }
    for (auto &jb : p->jobs) jb.table = (jb.table && jb.period == tp) ? 1 : 0;
    if (cudaMemcpyAsync(p->d_jobs, p->jobs.data(), sizeof(PilotJob) * (size_t)nj, cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
        return GPUD_E_CUDA;
    if (tp > 0 && tp != p->tab_period) {
        k_pilot_table<<<(tp + 255) / 256 < 1024 ? (tp + 255) / 256 : 1024, 256, 0, s>>>(tp, p->d_tab);
        gpud_count_launch(1);
        p->tab_period = tp;
    }
    int maxf = 0;
    for (auto &jb : p->jobs) maxf = std::max(maxf, jb.folded);
    dim3 gf((unsigned)std::min(1024, (maxf + kPilotThreads - 1) / kPilotThreads), (unsigned)nj);
    k_pilot_fold<<<gf, kPilotThreads, 0, s>>>(p->d_jobs, p->d_y);
    k_pilot_bins<<<dim3(kBins, (unsigned)nj), kPilotThreads, 0, s>>>(p->d_jobs, p->d_y, p->d_tab, p->d_mags);
    k_pilot_decide<<<nj, kPilotThreads, 0, s>>>(p->d_mags, threshold, p->d_res);
    if (cudaGetLastError() != cudaSuccess) return GPUD_E_CUDA;
    gpud_count_launch(3);
    std::vector<gpud_pilot_result> tmp((size_t)nj);
    if (cudaMemcpyAsync(tmp.data(), p->d_res, sizeof(gpud_pilot_result) * (size_t)nj, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GPUD_E_CUDA;
    for (int j = 0; j < count; ++j)
        if (p->job_of[(size_t)j] >= 0) results[j] = tmp[(size_t)p->job_of[(size_t)j]];
    return 0;
}

}  // extern "C"

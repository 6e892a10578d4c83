// bank_extract.cu -- extraction of short-arm channel banks.
//
// Channels that share the decimation D, the tap count T (T <= 4D: at most four
// taps per polyphase arm) and the phase count before the block take their
// outputs on the same input grid n_j = (D - pc - 1) + j*D.  With the NCO moved
// from the samples onto the taps (the modulated-taps identity of the
// reference's NCO-then-FIR chain, streaming_host_core.go:5-64):
//
//     y_c(j) = exp(j phi_c(n_j)) * sum_{k<T} g_c[k] x(n_j - k),   g_c[k] = h_c[k] exp(-j k inc_c),
//
// every channel of the bank filters the same unrotated block x.  One work item
// is 32 outputs x 32 channels: the 32 outputs' input windows are staged once in
// shared memory, 128 taps at a time, beside the 32 channels' modulated taps of
// the same range; lane c of warp w accumulates outputs 4w..4w+3 of channel c
// in registers (the window samples are warp-wide broadcasts, the taps one
// 16-byte load per lane for two taps), across all tap chunks, then rotates by
// exp(j phi_c(n_j)) from the exact Q0.64 phase and stores.  So the block is
// read once per bank and tile instead of once per channel, and no partial
// sums leave the SM.  Outputs whose window reaches into the carried history
// (before the bank's first tile) stay on the warp-per-output kernel.
#include <algorithm>

#include "gpud_internal.cuh"

namespace gpud {

constexpr int kBankThreads = 256;
constexpr int kBankLanes = 32;                 // channels per work item (one per lane)
constexpr int kBankR = 4;                      // most outputs per lane
constexpr int kBankJ = (kBankThreads / 32) * kBankR;  // most outputs per work item
constexpr int kBankKC = 128;                   // taps per staged chunk
constexpr int kBankSmem = (kBankJ + kBankLanes) * kBankKC * 8;  // windows + taps, float2

int bank_lanes() { return kBankLanes; }
int bank_warps() { return kBankThreads / 32; }

// Modulated taps of every bank, g[b.g_off + k*cpad + c] (float2), zero for
// padding columns; the same products as the other modulated forms.
__global__ void __launch_bounds__(256)
k_bank_pack(const BankGroup *__restrict__ groups, const int *__restrict__ members, const SlotBlock *__restrict__ sbt,
            const ChanParams *__restrict__ prm, const float *__restrict__ taps_arena, float2 *__restrict__ gtab) {
    const BankGroup b = groups[blockIdx.y];
    const int total = b.T * b.cpad;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int k = i / b.cpad, c = i - k * b.cpad;
        float2 v = make_float2(0.f, 0.f);
        if (c < b.nmem) {
            const ChanParams &cp = prm[sbt[members[b.mem_off + c]].slot];
            const float h = taps_arena[cp.dtaps_off + k];
            const float2 ph = q64_phasor((uint64_t)0 - (uint64_t)k * cp.inc_q);
            v = make_float2(h * ph.x, h * ph.y);
        }
        gtab[b.g_off + i] = v;
    }
}

// Work item (bank, tile * chunks + chunk): outputs jt0 + 8r*tile .. of
// channels 32*chunk .. +31, r outputs per lane (small banks take r < 4, so
// that they still give every SM work).
__global__ void __launch_bounds__(kBankThreads, 3)
k_extract_bank(const int2 *__restrict__ work, const BankGroup *__restrict__ groups, const int *__restrict__ members,
               const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
               const ChanState *__restrict__ st, const float2 *__restrict__ x, const float2 *__restrict__ gtab,
               float2 *__restrict__ ext) {
    extern __shared__ float4 bsm[];
    float4 *s_x = bsm;                                  // [kBankJ][kBankKC/2]: (x(n_o-k), x(n_o-k-1))
    float4 *s_g = bsm + kBankJ * (kBankKC / 2);         // [kBankKC/2][kBankLanes]: (g_c[k], g_c[k+1])
    float2 *s_x2 = reinterpret_cast<float2 *>(s_x);
    float2 *s_g2 = reinterpret_cast<float2 *>(s_g);
    const int2 w = work[blockIdx.x];
    const BankGroup b = groups[w.x];
    const int nch = b.cpad / kBankLanes;
    const int tile = w.y / nch, chunk = w.y - tile * nch;
    const int R = b.r, J = (kBankThreads / 32) * R;
    const int j0 = b.jt0 + tile * J;
    if (j0 >= b.n_out) return;
    const int D = b.D, T = b.T;
    const int s0 = D - b.pc - 1;
    const int c0 = chunk * kBankLanes;
    const int tid = (int)threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float ar[kBankR], ai[kBankR];
#pragma unroll
    for (int r = 0; r < kBankR; ++r) ar[r] = ai[r] = 0.f;
    for (int kc = 0; kc < T; kc += kBankKC) {
        const int kn = min(kBankKC, T - kc);
        // windows: output o's samples n_o - kc - kk (inside the block: the
        // bank starts at the first output whose window does)
#pragma unroll 4
        for (int i = tid; i < J * kBankKC; i += kBankThreads) {
            const int o = i / kBankKC, kk = i - o * kBankKC;
            const int j = j0 + o;
            float2 v = make_float2(0.f, 0.f);
            if (kk < kn && j < b.n_out) v = __ldg(x + (s0 + j * D - kc - kk));
            s_x2[i] = v;
        }
        // taps of this chunk's channels (padding channels and taps: zero)
#pragma unroll 4
        for (int i = tid; i < kBankKC * kBankLanes; i += kBankThreads) {
            const int kk = i / kBankLanes, c = i - kk * kBankLanes;
            const float2 v = kk < kn ? gtab[b.g_off + (kc + kk) * b.cpad + c0 + c] : make_float2(0.f, 0.f);
            s_g2[((kk >> 1) * kBankLanes + c) * 2 + (kk & 1)] = v;
        }
        __syncthreads();
        const float4 *xw = s_x + (warp * R) * (kBankKC / 2);
        const int nq = (kn + 1) >> 1;
#pragma unroll 4
        for (int q = 0; q < nq; ++q) {
            const float4 g = s_g[q * kBankLanes + lane];
#pragma unroll
            for (int r = 0; r < kBankR; ++r) {
                if (r >= R) break;
                const float4 v = xw[r * (kBankKC / 2) + q];  // broadcast
                ar[r] = fmaf(g.x, v.x, ar[r]);
                ar[r] = fmaf(-g.y, v.y, ar[r]);
                ar[r] = fmaf(g.z, v.z, ar[r]);
                ar[r] = fmaf(-g.w, v.w, ar[r]);
                ai[r] = fmaf(g.x, v.y, ai[r]);
                ai[r] = fmaf(g.y, v.x, ai[r]);
                ai[r] = fmaf(g.z, v.w, ai[r]);
                ai[r] = fmaf(g.w, v.z, ai[r]);
            }
        }
        __syncthreads();  // the staging is rewritten by the next chunk
    }
    const int c = c0 + lane;
    if (c >= b.nmem) return;
    const SlotBlock &sb = sbt[members[b.mem_off + c]];
    const uint64_t u0 = st[sb.slot].nco_q, inc = prm[sb.slot].inc_q;
#pragma unroll
    for (int r = 0; r < kBankR; ++r) {
        const int j = j0 + warp * R + r;
        if (r < R && j < b.n_out) {
            const float2 rot = q64_phasor(u0 + (uint64_t)(int64_t)(s0 + j * D) * inc);
            ext[sb.ext_off + j] = cmulf(make_float2(ar[r], ai[r]), rot);
        }
    }
}

cudaError_t launch_bank_pack(int ngroups, int max_total, cudaStream_t sm, const BankGroup *groups,
                             const int *members, const SlotBlock *sbt, const ChanParams *prm, const float *taps,
                             float2 *gtab) {
    const int gx = std::min(64, (max_total + 255) / 256);
    k_bank_pack<<<dim3(gx > 0 ? gx : 1, ngroups), 256, 0, sm>>>(groups, members, sbt, prm, taps, gtab);
    return cudaGetLastError();
}

cudaError_t launch_extract_bank(int grid, cudaStream_t sm, const int2 *work, const BankGroup *groups,
                                const int *members, const SlotBlock *sbt, const ChanParams *prm, const ChanState *st,
                                const float2 *x, const float2 *gtab, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_bank, kBankSmem);
    if (e != cudaSuccess) return e;
    k_extract_bank<<<grid, kBankThreads, kBankSmem, sm>>>(work, groups, members, sbt, prm, st, x, gtab, ext);
    return cudaGetLastError();
}

}  // namespace gpud

// runner_kernels.cu -- sm_100a kernels of the batched / serving runner.
//
// One IQ block flows through, in stream order:
//   k_extract_dense<L> / k_extract_wide   NCO + polyphase FIR + decimation
//   k_demod, k_am                         FM discriminator (with bridge), SSB/CW, AM
//   k_wfm_fir                             stereo FIR bank: L+R, L-R band, pilot band
//   k_pll                                 19 kHz pilot PLL, L-R product, lock decision
//   k_wfm_out                             L-R 15 kHz LPF and L/R matrix, or mono fallback
//   k_rds                                 57 kHz RDS baseband (exact FreqShift phase)
//   k_post                                per-slot state carry (histories, phases)
// Every kernel takes a work list of (slot-block index, tile) pairs so channels
// with uneven taps / decimation run in the same launch.
#include <climits>
#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

#include "gpud_internal.cuh"

#ifndef GPUD_DENSE_STAGE_U
#define GPUD_DENSE_STAGE_U 4
#endif
#ifndef GPUD_COLUMN_STAGE_U
#define GPUD_COLUMN_STAGE_U 4
#endif

namespace gpud {

// ===========================================================================
// Extraction: NCO shift -> FIR -> decimate  (streaming_host_core.go:5-64)
// ===========================================================================
//
// Output j of a block takes the input sample n_j = (D - pc - 1) + j*D as its
// newest sample (exports.cu:583) and y_j = sum_{k<T} h[k] * s(n_j - k), where
// s(i) = x[i] * exp(j*phi_i) for i >= 0 and the carried shifted history for
// i < 0 (zero before the stream start).
//
// Dense form (L = ceil(T/D) >= 2): the rotated samples of a tile are staged in
// shared memory transposed into the D polyphase components,
//     Z[p][m] = s(s0 + m*D - p),   p < D,
// so that y_j = sum_p sum_u h[p + u*D] * Z[p][j - u].  Warp w owns the phases
// p = w, w+8, ...; each lane owns R = 8 consecutive outputs and keeps a
// register window of R + L - 1 samples per phase (R*L FMAs per R+L-1 shared
// loads).  A row stride padded by one slot every 8 keeps the lane-strided
// window loads free of bank conflicts.  The 8 warps' partial sums are reduced
// through shared memory at the end.
constexpr int kDenseR = 8;
constexpr int kDenseOT = 32 * kDenseR;  // outputs per tile
constexpr int kDenseThreads = 256;

// Row stride in float2: one pad slot per 8 (lane-strided window reads stay
// conflict-free) and odd (the staging stores, which walk down a column with
// consecutive threads on consecutive phases, spread over all banks).
__host__ __device__ inline int dense_row_stride(int L) {
    int M = kDenseOT + L - 1;
    return (M + (M >> 3) + 1) | 1;
}

// Rotation table entries: one per 256-sample staging round.
__host__ __device__ inline int dense_rounds(int P, int L) { return (P * (kDenseOT + L - 1) + kDenseThreads - 1) / kDenseThreads; }

// Shared memory: Z (reused for the cross-warp reduction) | taps | rotation
// table.
__host__ __device__ inline int dense_zbytes(int P, int L) {
    int z = (P * dense_row_stride(L) * 8 + 15) & ~15;
    int red = 8 * (kDenseOT + kDenseOT / 8) * 16;  // float64 reduction of precise channels
    return z > red ? z : red;
}

__host__ __device__ inline int dense_smem_bytes(int P, int L) {
    return dense_zbytes(P, L) + ((P * L + 3) & ~3) * 4 + dense_rounds(P, L) * 8 + 16;
}

// Rotation of tile sample i' = t + 256k: exp(j phi(ibase + t)) * exp(j 256 k inc).
struct RotPair {
    float2 a;
    const float2 *tab;
    __device__ __forceinline__ float2 operator()(int k) const { return cmulf(a, tab[k]); }
};

__device__ __forceinline__ void dense_stage(float2 *Z, int Mp, int D, int total, int nk, int ibase, int n,
                                            const float2 *__restrict__ x, const float2 *__restrict__ hist, int H,
                                            const RotPair &rp) {
    const int t = (int)threadIdx.x;
    int mr = t / D, q = t - (t / D) * D;
    const int dm = kDenseThreads / D, dq = kDenseThreads - dm * D;
    const int nfull = total / kDenseThreads;  // rounds in which every thread has a sample
    const bool interior = ibase >= 0 && ibase + total <= n;
    constexpr int U = GPUD_DENSE_STAGE_U;  // staged loads in flight per thread
    int k = 0;
    if (interior && 32 % D == 0) {
        // D divides 32: the thread's phase row never changes (256 is a
        // multiple of D) and its column advances by dm = 256/D, a multiple of
        // 8, so the padded column c + c/8 advances by the constant 9*dm/8.
        const float2 *xp = x + ibase + t;
        float2 *zp = Z + (D - 1 - q) * Mp + mr + (mr >> 3);
        const int dz = dm + (dm >> 3);
        for (; k + U <= nfull; k += U) {
            float2 xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = __ldg(xp + (k + u) * kDenseThreads);
#pragma unroll
            for (int u = 0; u < U; ++u) zp[(k + u) * dz] = cmulf(xv[u], rp(k + u));
        }
        mr += k * dm;  // hand the position to the remaining rounds
    } else if (interior) {
        const float2 *xp = x + ibase + t;
        for (; k + U <= nfull; k += U) {
            float2 xv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) xv[u] = __ldg(xp + (k + u) * kDenseThreads);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const float2 rot = rp(k + u);
                Z[(D - 1 - q) * Mp + mr + (mr >> 3)] = cmulf(xv[u], rot);
                q += dq;
                mr += dm;
                if (q >= D) {
                    q -= D;
                    ++mr;
                }
            }
        }
    }
    // remaining rounds, and every round of tiles at the block edges
    for (; k < nk; ++k) {
        const int ip = t + k * kDenseThreads;
        if (ip < total) {
            const int i = ibase + ip;
            float2 v;
            if (i >= 0) {
                v = i < n ? cmulf(__ldg(x + i), rp(k)) : make_float2(0.f, 0.f);
            } else {
                const int hi = H + i;
                v = hi >= 0 ? hist[hi] : make_float2(0.f, 0.f);
            }
            Z[(D - 1 - q) * Mp + mr + (mr >> 3)] = v;
        }
        q += dq;
        mr += dm;
        if (q >= D) {
            q -= D;
            ++mr;
        }
    }
}

int dense_smem_bytes_host(int P, int L) { return dense_smem_bytes(P, L); }
int dense_tile() { return kDenseOT; }

// One phase row, L <= 16 taps: lane's R outputs from a window of R+L-1.
template <int L>
__device__ __forceinline__ void group_row(const float2 *zrow, const float *hrow, int lane, float *ar, float *ai) {
    constexpr int R = kDenseR;
    float2 win[R + L - 1];
#pragma unroll
    for (int tt = 0; tt < R + L - 1; ++tt) {
        const int c = lane * R + tt;
        win[tt] = zrow[c + (c >> 3)];
    }
    float h[L];
#pragma unroll
    for (int u = 0; u < L; ++u) h[u] = hrow[u];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int u = 0; u < L; ++u) {
            const float2 z = win[r + L - 1 - u];
            ar[r] = fmaf(h[u], z.x, ar[r]);
            ai[r] = fmaf(h[u], z.y, ai[r]);
        }
    }
}

// One phase row, long arm (Le a multiple of 8 > 16): chunks of 8 taps with a
// window of R+7 samples that slides 8 columns per chunk (8 new loads).
__device__ __forceinline__ void group_row_long(const float2 *zrow, const float *hrow, int Le, int lane, float *ar,
                                               float *ai) {
    constexpr int R = kDenseR;
    constexpr int W = R + 7;
    float2 win[W];
    int base = lane * R + Le - 8;  // chunk c: columns base - 8c + t
#pragma unroll
    for (int t = 0; t < W; ++t) {
        const int c = base + t;
        win[t] = zrow[c + (c >> 3)];
    }
    const int nc = Le >> 3;
    for (int ch = 0; ch < nc; ++ch) {
        const float4 h0 = *reinterpret_cast<const float4 *>(hrow + 8 * ch);
        const float4 h1 = *reinterpret_cast<const float4 *>(hrow + 8 * ch + 4);
        const float h[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int v = 0; v < 8; ++v) {
                const float2 z = win[r + 7 - v];
                ar[r] = fmaf(h[v], z.x, ar[r]);
                ai[r] = fmaf(h[v], z.y, ai[r]);
            }
        }
        if (ch + 1 < nc) {
#pragma unroll
            for (int t = W - 1; t >= 8; --t) win[t] = win[t - 8];
            base -= 8;
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int c = base + t;
                win[t] = zrow[c + (c >> 3)];
            }
        }
    }
}

// Sum of a tile: the rows pp = warp, warp+8, ... < rows accumulate into each
// lane's R outputs, then the 8 warps' partial sums are reduced through shared
// memory (Z reused) and out(o, sum) receives tile output o.  With PREC each
// row is summed in float32 on its own and the rows are added in float64
// (channels whose demodulator magnifies white output error: the float32
// rounding then no longer grows with the running sum of the whole tile).
constexpr int kRedStride = kDenseOT + kDenseOT / 8;
constexpr int kRedBytes = 8 * kRedStride * 16;

template <bool PREC, class Row, class Out>
__device__ __forceinline__ void tile_sum(int rows, const Row &row, float2 *Z, const Out &out) {
    constexpr int R = kDenseR;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if constexpr (!PREC) {
        float ar[R], ai[R];
#pragma unroll
        for (int r = 0; r < R; ++r) ar[r] = ai[r] = 0.f;
        for (int pp = warp; pp < rows; pp += 8) row(pp, lane, ar, ai);
        __syncthreads();
        float2 *red = Z + warp * kRedStride;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int o = lane * R + r;
            red[o + (o >> 3)] = make_float2(ar[r], ai[r]);
        }
        __syncthreads();
        for (int o = threadIdx.x; o < kDenseOT; o += kDenseThreads) {
            float2 sum = make_float2(0.f, 0.f);
#pragma unroll
            for (int wv = 0; wv < 8; ++wv) {
                const float2 v = Z[wv * kRedStride + o + (o >> 3)];
                sum.x += v.x;
                sum.y += v.y;
            }
            out(o, sum);
        }
    } else {
        double dr[R], di[R];
#pragma unroll
        for (int r = 0; r < R; ++r) dr[r] = di[r] = 0.0;
        for (int pp = warp; pp < rows; pp += 8) {
            float ar[R], ai[R];
#pragma unroll
            for (int r = 0; r < R; ++r) ar[r] = ai[r] = 0.f;
            row(pp, lane, ar, ai);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                dr[r] += (double)ar[r];
                di[r] += (double)ai[r];
            }
        }
        __syncthreads();
        double2 *Z64 = reinterpret_cast<double2 *>(Z);
        double2 *red = Z64 + warp * kRedStride;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int o = lane * R + r;
            red[o + (o >> 3)] = make_double2(dr[r], di[r]);
        }
        __syncthreads();
        for (int o = threadIdx.x; o < kDenseOT; o += kDenseThreads) {
            double2 sum = make_double2(0.0, 0.0);
#pragma unroll
            for (int wv = 0; wv < 8; ++wv) {
                const double2 v = Z64[wv * kRedStride + o + (o >> 3)];
                sum.x += v.x;
                sum.y += v.y;
            }
            out(o, sum);
        }
    }
}

// One 256-output tile of the dense form (work item w), arm length L.
template <int L>
__device__ __forceinline__ void dense_tile(const int2 w, const SlotBlock &sb, const ChanParams &cp,
                                           const ChanState *__restrict__ st, const float2 *__restrict__ x, int n,
                                           const float2 *__restrict__ hist_arena,
                                           const float *__restrict__ taps_arena, float2 *__restrict__ ext,
                                           float4 *smem4) {
    const int j0 = w.y * kDenseOT;
    const int D = cp.decim;
    const int P = cp.nphase;
    const int M = kDenseOT + L - 1;
    const int Mp = dense_row_stride(L);
    float2 *Z = reinterpret_cast<float2 *>(smem4);
    float *tsm = reinterpret_cast<float *>(reinterpret_cast<char *>(smem4) + dense_zbytes(P, L));
    void *wtab = tsm + ((P * L + 3) & ~3);

    const int s0 = D - sb.pc - 1;
    const int m_base = j0 - (L - 1);
    const uint64_t u0 = st[sb.slot].nco_q;
    const uint64_t inc = cp.inc_q;
    const float2 *hist = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
    const int H = sb.hist_len;
    // Staging.  Tile sample i' = 0..M*D-1 is block sample i = ibase + i' and
    // lands in Z[p][m] with m = i'/D, p = D-1 - i'%D.  Thread t takes
    // i' = t + 256*k: consecutive threads hit consecutive phases (odd row
    // stride: no bank conflicts), and (m, p) advance by a constant step with
    // one carry.  The rotation of sample i' is exp(j*phi(ibase + t)) *
    // exp(j*256*k*inc), both exact from the Q0.64 phase (the second from a
    // per-tile table).
    const int total = P * M;  // P == D in the dense form
    const int ibase = s0 + m_base * D - (D - 1);
    const int nk = dense_rounds(P, L);
    const float *tg = taps_arena + cp.taps_off;
    for (int i = threadIdx.x; i < P * L; i += kDenseThreads) tsm[i] = tg[i];
    const int t = (int)threadIdx.x;
    {
        float2 *w32 = reinterpret_cast<float2 *>(wtab);
        for (int k = threadIdx.x; k < nk; k += kDenseThreads)
            w32[k] = q64_phasor((uint64_t)k * (uint64_t)kDenseThreads * inc);
        const RotPair rp{q64_phasor(u0 + (uint64_t)(int64_t)(ibase + t) * inc), w32};
        __syncthreads();
        dense_stage(Z, Mp, D, total, nk, ibase, n, x, hist, H, rp);
    }
    __syncthreads();

    auto row = [&](int p, int lane, float *ar, float *ai) { group_row<L>(Z + p * Mp, tsm + p * L, lane, ar, ai); };
    float2 *dst = ext + sb.ext_off + j0;
    const int nv = sb.n_out - j0;
    if (cp.precise_sum)
        tile_sum<true>(P, row, Z, [&](int o, double2 v) {
            if (o < nv) dst[o] = make_float2((float)v.x, (float)v.y);
        });
    else
        tile_sum<false>(P, row, Z, [&](int o, float2 v) {
            if (o < nv) dst[o] = v;
        });
}

template <int L>
__global__ void __launch_bounds__(kDenseThreads, 2)
k_extract_dense(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
                const ChanState *__restrict__ st, const float2 *__restrict__ x, int n,
                const float2 *__restrict__ hist_arena, const float *__restrict__ taps_arena,
                float2 *__restrict__ ext) {
    extern __shared__ float4 smem4[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    if (w.y * kDenseOT >= sb.n_out) return;
    dense_tile<L>(w, sb, prm[sb.slot], st, x, n, hist_arena, taps_arena, ext, smem4);
}

// Several dense classes in one launch (each too small to fill the GPU alone):
// every CTA takes its tile's arm length from the channel.
__global__ void __launch_bounds__(kDenseThreads, 2)
k_extract_dense_any(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt,
                    const ChanParams *__restrict__ prm, const ChanState *__restrict__ st,
                    const float2 *__restrict__ x, int n, const float2 *__restrict__ hist_arena,
                    const float *__restrict__ taps_arena, float2 *__restrict__ ext) {
    extern __shared__ float4 smem4[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    if (w.y * kDenseOT >= sb.n_out) return;
    const ChanParams &cp = prm[sb.slot];
    switch (cp.plen) {  // uniform per CTA
#define GPUD_ANY(LL) \
    case LL: dense_tile<LL>(w, sb, cp, st, x, n, hist_arena, taps_arena, ext, smem4); break;
        GPUD_ANY(2) GPUD_ANY(3) GPUD_ANY(4) GPUD_ANY(5) GPUD_ANY(6) GPUD_ANY(7) GPUD_ANY(8) GPUD_ANY(9)
        GPUD_ANY(10) GPUD_ANY(11) GPUD_ANY(12) GPUD_ANY(13) GPUD_ANY(14) GPUD_ANY(15) GPUD_ANY(16)
#undef GPUD_ANY
    default: break;
    }
}

// ---------------------------------------------------------------------------
// Dense form, persistent pipelined variant (k_extract_dense_pipe<L, NG>).
//
// One CTA per SM walks a contiguous run of the class's tiles (consecutive
// tiles of a channel stay together).  Warp 16 is the producer: it loads the
// next tile's descriptors ahead of time and, as soon as the previous tile has
// been staged, brings the next tile's polyphase taps and (for tiles inside
// the block) its raw input span into shared memory with bulk copies whose
// completion is counted on an mbarrier.  The 16 consumer warps form NG groups
// that take the tiles in turn, each with its own Z: a group rotates and
// transposes its tile from the raw span into Z (tiles that reach into the
// history or past the block end stage from global memory as k_extract_dense
// does), releases the raw span, then runs the FIR rows and the cross-warp
// reduction while the other group stages the next tile.  The global-load
// latency of the one-tile-per-CTA kernel (descriptor chain, then staging
// loads) thereby overlaps arithmetic.  Every mbarrier wait is bounded: a wait
// that gives up stores a code in the runner's fault word and the CTA returns
// (the host reports GPUD_E_DEVICE_STATUS).
//
// Barrier use: full[g] completes once per tile of group g (the producer's
// arrival plus the bulk-copy bytes), `empty` once per staged tile (tiles are
// staged strictly in order, each after the previous one's release), named
// barrier 1 + g synchronises group g.
// ---------------------------------------------------------------------------
constexpr int kPipeCW = 16;                     // consumer warps
constexpr int kPipeThreads = 32 * kPipeCW + 32;  // + the producer warp
constexpr int kPipeMaxRounds = 64;              // staging rounds per tile (two table entries per producer lane)

struct PipeDesc {
    const float2 *hist;
    uint64_t u0, inc;
    int j0, n_out, ext_off, ibase, total, nk, D, P, H, precise, tma, off;
};
static_assert(32 + sizeof(PipeDesc) <= 128, "the descriptor sits between the mbarriers and the rotation table");

struct PipeLayout {
    int o_w, o_taps, tstride, o_z, zstride, o_r, bytes;
};

// Shared memory of a launch whose channels have at most pmax phases, ng
// consumer groups: mbarriers (full[2], empty) | descriptor | rotation table |
// taps x4 | Z (and reduction) per group | raw span.
__host__ __device__ inline PipeLayout pipe_layout(int pmax, int L, int ng) {
    PipeLayout lo;
    lo.o_w = 128;
    lo.o_taps = lo.o_w + kPipeMaxRounds * 8;
    lo.tstride = (pmax * L + 3) & ~3;  // floats; bulk-copy sizes are multiples of 16 bytes
    lo.o_z = lo.o_taps + 4 * lo.tstride * 4;
    const int z = pmax * dense_row_stride(L) * 8;
    const int red = (kPipeCW / ng) * kRedStride * 16;
    lo.zstride = ((z > red ? z : red) + 15) & ~15;
    lo.o_r = lo.o_z + ng * lo.zstride;
    lo.bytes = lo.o_r + (((pmax * (kDenseOT + L - 1) + 2) * 8 + 15) & ~15);
    return lo;
}

__device__ __forceinline__ void named_sync(int id, int count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Named barrier that also ORs a predicate over the participating threads.
__device__ __forceinline__ bool named_sync_or(int id, int count, bool pred) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((unsigned)pred), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

// Rows, cross-warp reduction (Z reused) and output of one tile for a consumer
// group of GW warps synchronised on named barrier `bar`.
template <bool PREC, int GW, class Row, class Out>
__device__ __forceinline__ void pipe_tile_sum(int rows, int gw, int lane, int gt, int bar, const Row &row, float2 *Z,
                                              const Out &out) {
    constexpr int R = kDenseR;
    constexpr int GNT = 32 * GW;
    if constexpr (!PREC) {
        float ar[R], ai[R];
#pragma unroll
        for (int r = 0; r < R; ++r) ar[r] = ai[r] = 0.f;
        for (int pp = gw; pp < rows; pp += GW) row(pp, lane, ar, ai);
        named_sync(bar, GNT);
        float2 *red = Z + gw * kRedStride;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int o = lane * R + r;
            red[o + (o >> 3)] = make_float2(ar[r], ai[r]);
        }
        named_sync(bar, GNT);
        for (int o = gt; o < kDenseOT; o += GNT) {
            float2 sum = make_float2(0.f, 0.f);
#pragma unroll
            for (int wv = 0; wv < GW; ++wv) {
                const float2 v = Z[wv * kRedStride + o + (o >> 3)];
                sum.x += v.x;
                sum.y += v.y;
            }
            out(o, sum);
        }
    } else {
        double dr[R], di[R];
#pragma unroll
        for (int r = 0; r < R; ++r) dr[r] = di[r] = 0.0;
        for (int pp = gw; pp < rows; pp += GW) {
            float ar[R], ai[R];
#pragma unroll
            for (int r = 0; r < R; ++r) ar[r] = ai[r] = 0.f;
            row(pp, lane, ar, ai);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                dr[r] += (double)ar[r];
                di[r] += (double)ai[r];
            }
        }
        named_sync(bar, GNT);
        double2 *Z64 = reinterpret_cast<double2 *>(Z);
        double2 *red = Z64 + gw * kRedStride;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int o = lane * R + r;
            red[o + (o >> 3)] = make_double2(dr[r], di[r]);
        }
        named_sync(bar, GNT);
        for (int o = gt; o < kDenseOT; o += GNT) {
            double2 sum = make_double2(0.0, 0.0);
#pragma unroll
            for (int wv = 0; wv < GW; ++wv) {
                const double2 v = Z64[wv * kRedStride + o + (o >> 3)];
                sum.x += v.x;
                sum.y += v.y;
            }
            out(o, sum);
        }
    }
}

template <int L, int NG>
__global__ void __launch_bounds__(kPipeThreads, 1)
k_extract_dense_pipe(const int2 *__restrict__ work, int ntiles, int pmax, const SlotBlock *__restrict__ sbt,
                     const ChanParams *__restrict__ prm, const ChanState *__restrict__ st,
                     const float2 *__restrict__ x, int n, const float2 *__restrict__ hist_arena,
                     const float *__restrict__ taps_arena, float2 *__restrict__ ext, unsigned *fault) {
    constexpr int GW = kPipeCW / NG;  // warps per consumer group
    constexpr int GNT = 32 * GW;      // threads per consumer group
    extern __shared__ __align__(128) unsigned char psm[];
    const PipeLayout lo = pipe_layout(pmax, L, NG);
    uint64_t *full = reinterpret_cast<uint64_t *>(psm);  // full[0], full[1]
    uint64_t *empty = full + 2;
    PipeDesc *dsc = reinterpret_cast<PipeDesc *>(psm + 32);
    float2 *wt = reinterpret_cast<float2 *>(psm + lo.o_w);
    float *tsm = reinterpret_cast<float *>(psm + lo.o_taps);
    float2 *Rw = reinterpret_cast<float2 *>(psm + lo.o_r);
    const int b0 = (int)((long long)ntiles * blockIdx.x / gridDim.x);
    const int b1 = (int)((long long)ntiles * (blockIdx.x + 1) / gridDim.x);
    const int nt = b1 - b0;
    if (threadIdx.x == 0) {
        mbar_init(full, 1);
        mbar_init(full + 1, 1);
        mbar_init(empty, 1);
        mbar_init_fence();
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int M = kDenseOT + L - 1;
    const int Mp = dense_row_stride(L);

    if (warp == kPipeCW) {
        // ---- producer ----
        for (int it = 0; it < nt; ++it) {
            const int2 w = work[b0 + it];
            const SlotBlock &sb = sbt[w.x];
            const ChanParams &cp = prm[sb.slot];
            PipeDesc d;
            d.D = cp.decim;
            d.P = cp.nphase;
            d.j0 = w.y * kDenseOT;
            d.n_out = sb.n_out;
            d.ext_off = sb.ext_off;
            d.u0 = st[sb.slot].nco_q;
            d.inc = cp.inc_q;
            d.ibase = (d.D - sb.pc - 1) + (d.j0 - (L - 1)) * d.D - (d.D - 1);
            d.total = d.P * M;
            d.nk = (d.total + GNT - 1) / GNT;
            d.hist = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
            d.H = sb.hist_len;
            d.precise = cp.precise_sum;
            const int a0 = d.ibase & ~1;
            const int cnt = (d.ibase - a0 + d.total + 1) & ~1;
            d.tma = d.ibase >= 0 && (long long)a0 + cnt <= (long long)n;
            d.off = d.tma ? d.ibase - a0 : 0;
            // rotation of staging round k: exp(j k GNT inc), exact from the Q0.64 phase
            const float2 w0 = q64_phasor((uint64_t)lane * (uint64_t)GNT * d.inc);
            const float2 w1 = q64_phasor((uint64_t)(lane + 32) * (uint64_t)GNT * d.inc);
            const float *tsrc = taps_arena + cp.taps_off;
            // the previous tile has been staged: the raw span, the table and
            // the descriptor are free; taps buffer it & 3 was last read by
            // tile it - 4, finished before tile it - 2 of its group was staged
            if (it > 0 && !mbar_wait_bounded(empty, (unsigned)(it - 1) & 1u)) {
                if (lane == 0) device_fault(fault, 1u);
                return;
            }
            if (lane < d.nk) wt[lane] = w0;
            if (lane + 32 < d.nk) wt[lane + 32] = w1;
            if (lane == 0) *dsc = d;
            __syncwarp();
            if (lane == 0) {
                uint64_t *fb = full + (NG == 2 ? (it & 1) : 0);
                const unsigned tb = (unsigned)(((d.P * L + 3) & ~3) * 4);
                const unsigned rb = d.tma ? (unsigned)cnt * 8u : 0u;
                mbar_arrive_expect_tx(fb, tb + rb);
                bulk_to_smem(tsm + (it & 3) * lo.tstride, tsrc, tb, fb);
                if (d.tma) bulk_to_smem(Rw, x + a0, rb, fb);
            }
        }
        return;
    }

    // ---- consumers: group g takes tiles g, g + NG, ... ----
    const int g = warp / GW, gw = warp - g * GW;
    const int gt = (int)threadIdx.x - g * GNT;
    float2 *Z = reinterpret_cast<float2 *>(psm + lo.o_z + g * lo.zstride);
    uint64_t *fb = full + g;
    for (int it = g, kl = 0; it < nt; it += NG, ++kl) {
        const bool ok = mbar_wait_bounded(fb, (unsigned)kl & 1u);
        // the group has read its previous tile's reduction; all agree whether
        // to go on
        if (named_sync_or(1 + g, GNT, !ok)) {
            if (gt == 0) device_fault(fault, 2u);
            return;
        }
        const PipeDesc d = *dsc;
        const int D = d.D;
        const float2 a = q64_phasor(d.u0 + (uint64_t)(int64_t)(d.ibase + gt) * d.inc);
        int mr = gt / D, q = gt - (gt / D) * D;
        const int dm = GNT / D, dq = GNT - dm * D;
        if (d.tma) {
            const float2 *sp = Rw + d.off + gt;
            const int nfull = d.total / GNT;
            int k = 0;
            if ((GNT / 8) % D == 0) {
                // the thread's phase row is fixed and its padded column
                // advances by the constant dm + dm/8 (dm a multiple of 8)
                float2 *zp = Z + (D - 1 - q) * Mp + mr + (mr >> 3);
                const int dz = dm + (dm >> 3);
                for (; k + 4 <= nfull; k += 4) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) zp[(k + u) * dz] = cmulf(sp[(k + u) * GNT], cmulf(a, wt[k + u]));
                }
                for (; k < nfull; ++k) zp[k * dz] = cmulf(sp[k * GNT], cmulf(a, wt[k]));
                mr += k * dm;
            }
            for (; k < d.nk; ++k) {
                if (gt + k * GNT < d.total)
                    Z[(D - 1 - q) * Mp + mr + (mr >> 3)] = cmulf(sp[k * GNT], cmulf(a, wt[k]));
                q += dq;
                mr += dm;
                if (q >= D) {
                    q -= D;
                    ++mr;
                }
            }
        } else {
            // tile at a block edge: history before sample 0, zeros past n;
            // four loads in flight per thread
            constexpr int U = 4;
            for (int k0 = 0; k0 < d.nk; k0 += U) {
                float2 v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int ip = gt + (k0 + u) * GNT, i = d.ibase + ip;
                    v[u] = make_float2(0.f, 0.f);
                    if (k0 + u < d.nk && ip < d.total) {
                        if (i >= 0) {
                            if (i < n) v[u] = __ldg(x + i);
                        } else if (d.H + i >= 0) {
                            v[u] = d.hist[d.H + i];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = k0 + u, ip = gt + k * GNT;
                    if (k < d.nk && ip < d.total) {
                        // block samples are rotated here; history samples were stored rotated
                        const float2 z = d.ibase + ip >= 0 ? cmulf(v[u], cmulf(a, wt[k])) : v[u];
                        Z[(D - 1 - q) * Mp + mr + (mr >> 3)] = z;
                    }
                    q += dq;
                    mr += dm;
                    if (q >= D) {
                        q -= D;
                        ++mr;
                    }
                }
            }
        }
        named_sync(1 + g, GNT);
        if (gt == 0) mbar_arrive(empty);  // the raw span, the table and the descriptor may be refilled

        const float *hb = tsm + (it & 3) * lo.tstride;
        auto row = [&](int p, int ln, float *ar, float *ai) { group_row<L>(Z + p * Mp, hb + p * L, ln, ar, ai); };
        float2 *dst = ext + d.ext_off + d.j0;
        const int nv = d.n_out - d.j0;
        if (d.precise)
            pipe_tile_sum<true, GW>(d.P, gw, lane, gt, 1 + g, row, Z, [&](int o, double2 v) {
                if (o < nv) dst[o] = make_float2((float)v.x, (float)v.y);
            });
        else
            pipe_tile_sum<false, GW>(d.P, gw, lane, gt, 1 + g, row, Z, [&](int o, float2 v) {
                if (o < nv) dst[o] = v;
            });
    }
}

// Wide form (short polyphase arms, or tiles too large for shared memory): one
// warp per kWideOPW outputs, lanes stride the taps, warp-shuffle reduction.
// The NCO rotation is folded into the taps: for a sample of this block,
//     h[k] * x[n-k] * exp(j phi(n-k)) = exp(j phi(n)) * (h[k] exp(-j k inc)) * x[n-k],
// so each CTA builds the modulated taps hc[k] = h[k] exp(-j k inc) once (exact
// Q0.64 phases) and each output takes one rotation exp(j phi(n)) at the end;
// history samples (already shifted) take the real taps directly.
constexpr int kWideOPW = 4;                  // outputs per warp
constexpr int kWideOT = 8 * kWideOPW;        // outputs per 256-thread tile

int wide_smem_bytes_host(int T) { return T * 12; }

__global__ void __launch_bounds__(256)
k_extract_wide(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
               const ChanState *__restrict__ st, const float2 *__restrict__ x, int n,
               const float2 *__restrict__ hist_arena, const float *__restrict__ taps_arena,
               float2 *__restrict__ ext) {
    extern __shared__ float4 smemw4[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const int j0 = w.y * kWideOT;
    // a banked channel: only the outputs before its bank's first one
    const int n_end = sb.wide_end > 0 ? min(sb.wide_end, sb.n_out) : sb.n_out;
    if (j0 >= n_end) return;
    const ChanParams &cp = prm[sb.slot];
    const int T = cp.ntaps, D = cp.decim;
    const uint64_t u0 = st[sb.slot].nco_q;
    const uint64_t inc = cp.inc_q;
    float2 *hc = reinterpret_cast<float2 *>(smemw4);
    float *hr = reinterpret_cast<float *>(hc + T);
    for (int k = threadIdx.x; k < T; k += 256) {
        const float h = taps_arena[cp.dtaps_off + k];
        const float2 ph = q64_phasor((uint64_t)0 - (uint64_t)k * inc);
        hr[k] = h;
        hc[k] = make_float2(h * ph.x, h * ph.y);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = D - sb.pc - 1;
    const float2 *hist = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
    const int H = sb.hist_len;
    const int jw = j0 + warp * kWideOPW;
    if (jw >= n_end) return;
    const int no = min(kWideOPW, n_end - jw);
    float ar[kWideOPW], ai[kWideOPW], br[kWideOPW], bi[kWideOPW];
#pragma unroll
    for (int o = 0; o < kWideOPW; ++o) ar[o] = ai[o] = br[o] = bi[o] = 0.f;
    const int nj0 = s0 + jw * D;
    for (int k = lane; k < T; k += 32) {
        const float2 c = hc[k];
#pragma unroll
        for (int o = 0; o < kWideOPW; ++o) {
            if (o >= no) break;
            const int i = nj0 + o * D - k;
            if (i >= 0) {
                const float2 v = __ldg(x + i);
                ar[o] = fmaf(c.x, v.x, fmaf(-c.y, v.y, ar[o]));
                ai[o] = fmaf(c.x, v.y, fmaf(c.y, v.x, ai[o]));
            } else if (H + i >= 0) {
                const float2 v = hist[H + i];
                const float h = hr[k];
                br[o] = fmaf(h, v.x, br[o]);
                bi[o] = fmaf(h, v.y, bi[o]);
            }
        }
    }
#pragma unroll
    for (int o = 0; o < kWideOPW; ++o) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            ar[o] += __shfl_xor_sync(0xffffffffu, ar[o], off);
            ai[o] += __shfl_xor_sync(0xffffffffu, ai[o], off);
            br[o] += __shfl_xor_sync(0xffffffffu, br[o], off);
            bi[o] += __shfl_xor_sync(0xffffffffu, bi[o], off);
        }
    }
    if (lane < no) {
        // lane o writes output o (register arrays indexed by a compile-time loop)
#pragma unroll
        for (int o = 0; o < kWideOPW; ++o) {
            if (o == lane) {
                const int nj = nj0 + o * D;
                const float2 rot = q64_phasor(u0 + (uint64_t)(int64_t)nj * inc);
                const float2 y = cmulf(make_float2(ar[o], ai[o]), rot);
                ext[sb.ext_off + jw + o] = make_float2(y.x + br[o], y.y + bi[o]);
            }
        }
    }
}

// ===========================================================================
// Phase-grouped polyphase form: channels whose D phases of a 256-output tile
// do not fit in shared memory (large D), channels with one tap per phase
// (T <= D), and long arms (L > 16).  A work item is (tile, phase group g):
// the CTA stages the rotated samples of phases p_lo .. p_lo+Pc-1 only,
//     Z[pp][m] = s(s0 + (m_base + m)*D - (p_lo + pp)),
// -- for each column m a contiguous run of Pc samples -- and computes the
// group's share of the 256 outputs with the same warp/lane layout as the dense
// form.  One CTA takes all groups of its tile in turn, restaging shared memory
// per group, and each thread adds its output's group shares in group order in
// a register (deterministic: the grouping depends on the channel only), so no
// partial sums leave the SM.
// The rotation of sample cb(m) + r is A[m] * B[r], A[m] = exp(j phi(cb(m))),
// B[r] = exp(j r inc), both exact from the Q0.64 phase.
// ===========================================================================
__host__ __device__ inline int group_Le(int L) { return L > 16 ? (L + 7) & ~7 : L; }

__host__ __device__ inline int group_smem_bytes(int Pc, int L) {
    const int Le = group_Le(L);
    const int M = kDenseOT + Le - 1;
    int z = (Pc * dense_row_stride(Le) * 8 + 15) & ~15;  // the taps after Z are read as float4
    const int red = 8 * (kDenseOT + kDenseOT / 8) * 16;
    if (z < red) z = red;
    return z + ((Pc * Le + 3) & ~3) * 4 + (M + Pc) * 8 + 16;
}

int group_smem_bytes_host(int Pc, int L) { return group_smem_bytes(Pc, L); }

struct GroupTile {
    int j0, g, p_lo, Pc, Le, M, Mp;
};

// Sample x(cb0 + m*D + r) of column m lands in Z[Pc-1-r][m].  Warp w takes
// the columns m = w, w+8, ...; its lanes walk the column's contiguous run
// (coalesced loads; the stores go down one column of Z, odd row stride: no
// bank conflicts), four columns in flight.  fetch(i) returns the tile's
// value of block sample i.
template <class Fetch>
__device__ __forceinline__ void stage_columns(int Pc, int M, int Mp, int D, int cb0, float2 *Z, const Fetch &fetch) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int U = GPUD_COLUMN_STAGE_U;  // columns in flight per lane
    for (int m0 = warp; m0 < M; m0 += 8 * U) {
        for (int r = lane; r < Pc; r += 32) {
            float2 v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int m = m0 + 8 * u;
                v[u] = m < M ? fetch(cb0 + m * D + r, m, r) : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int m = m0 + 8 * u;
                if (m < M) Z[(Pc - 1 - r) * Mp + m + (m >> 3)] = v[u];
            }
        }
    }
}

__device__ __forceinline__ void group_stage_samples(const GroupTile &gt, int D, int cb0, int n, int H,
                                                    const float2 *__restrict__ x, const float2 *__restrict__ hist,
                                                    float2 *Z, const float2 *A, const float2 *B) {
    const bool interior = cb0 >= 0 && cb0 + (gt.M - 1) * D + gt.Pc <= n;
    if (interior) {
        stage_columns(gt.Pc, gt.M, gt.Mp, D, cb0, Z, [&](int i, int m, int r) {
            return cmulf(__ldg(x + i), cmulf(A[m], B[r]));
        });
    } else {
        stage_columns(gt.Pc, gt.M, gt.Mp, D, cb0, Z, [&](int i, int m, int r) {
            if (i >= n) return make_float2(0.f, 0.f);
            if (i >= 0) return cmulf(__ldg(x + i), cmulf(A[m], B[r]));
            const int hi = H + i;  // carried history: shifted already
            return hi >= 0 ? hist[hi] : make_float2(0.f, 0.f);
        });
    }
}

// Stage Z (row stride Mp, column c stored at c + c/8), the taps of the
// group's phases (padded with zeros to Le per phase) and the rotation tables
// (tabs: M + Pc float2 entries).
__device__ __forceinline__ void group_stage(const GroupTile &gt, const SlotBlock &sb, const ChanParams &cp,
                                            uint64_t u0, const float2 *__restrict__ x, int n,
                                            const float2 *__restrict__ hist, const float *__restrict__ tg,
                                            float2 *Z, float *tsm, void *tabs) {
    const int D = cp.decim, L = cp.plen;
    const uint64_t inc = cp.inc_q;
    const int s0 = D - sb.pc - 1;
    const int m_base = gt.j0 - (gt.Le - 1);
    const int Pc = gt.Pc;
    // cb(m): first sample of column m's run
    const int cb0 = s0 + m_base * D - gt.p_lo - Pc + 1;
    for (int i = threadIdx.x; i < Pc * gt.Le; i += kDenseThreads) {
        const int pp = i / gt.Le, u = i - pp * gt.Le;
        tsm[i] = u < L ? tg[(gt.p_lo + pp) * L + u] : 0.f;
    }
    {
        float2 *A = reinterpret_cast<float2 *>(tabs), *B = A + gt.M;
        for (int m = threadIdx.x; m < gt.M; m += kDenseThreads)
            A[m] = q64_phasor(u0 + (uint64_t)(int64_t)(cb0 + m * D) * inc);
        for (int r = threadIdx.x; r < Pc; r += kDenseThreads) B[r] = q64_phasor((uint64_t)r * inc);
        __syncthreads();
        group_stage_samples(gt, D, cb0, n, sb.hist_len, x, hist, Z, A, B);
    }
    __syncthreads();
}

static_assert(kDenseOT == kDenseThreads, "the phase-group kernels keep one output per thread");

__global__ void __launch_bounds__(kDenseThreads, 2)
k_extract_group(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
                const ChanState *__restrict__ st, const float2 *__restrict__ x, int n,
                const float2 *__restrict__ hist_arena, const float *__restrict__ taps_arena,
                float2 *__restrict__ ext) {
    extern __shared__ float4 smemg4[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    GroupTile gt;
    gt.j0 = w.y * kDenseOT;
    if (gt.j0 >= sb.n_out) return;
    const int L = cp.plen;
    gt.Le = group_Le(L);
    gt.M = kDenseOT + gt.Le - 1;
    gt.Mp = dense_row_stride(gt.Le);
    int zb = (sb.pg * gt.Mp * 8 + 15) & ~15;
    const int red_b = kRedBytes;
    if (zb < red_b) zb = red_b;
    float2 *Z = reinterpret_cast<float2 *>(smemg4);
    float *tsm = reinterpret_cast<float *>(reinterpret_cast<char *>(smemg4) + zb);
    void *tabs = tsm + ((sb.pg * gt.Le + 3) & ~3);
    const float2 *hist = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
    const uint64_t u0 = st[sb.slot].nco_q;

    auto row = [&](int pp, int lane, float *ar, float *ai) {
        const float2 *zrow = Z + pp * gt.Mp;
        const float *hrow = tsm + pp * gt.Le;
        switch (L) {
#define GPUD_ROW(LL) \
    case LL: group_row<LL>(zrow, hrow, lane, ar, ai); break;
            GPUD_ROW(1) GPUD_ROW(2) GPUD_ROW(3) GPUD_ROW(4) GPUD_ROW(5) GPUD_ROW(6) GPUD_ROW(7) GPUD_ROW(8)
            GPUD_ROW(9) GPUD_ROW(10) GPUD_ROW(11) GPUD_ROW(12) GPUD_ROW(13) GPUD_ROW(14) GPUD_ROW(15) GPUD_ROW(16)
#undef GPUD_ROW
        default: group_row_long(zrow, hrow, gt.Le, lane, ar, ai); break;
        }
    };
    const int nv = sb.n_out - gt.j0;
    const int o = (int)threadIdx.x;  // this thread's output of the tile
    double2 acc64 = make_double2(0.0, 0.0);
    float2 acc = make_float2(0.f, 0.f);
    for (int g = 0; g < sb.ng; ++g) {
        gt.g = g;
        gt.p_lo = g * sb.pg;
        gt.Pc = min(sb.pg, cp.nphase - gt.p_lo);
        if (g) __syncthreads();  // the last group's reduction has read Z
        group_stage(gt, sb, cp, u0, x, n, hist, taps_arena + cp.taps_off, Z, tsm, tabs);
        if (cp.precise_sum) {
            tile_sum<true>(gt.Pc, row, Z, [&](int, double2 v) {
                acc64.x += v.x;
                acc64.y += v.y;
            });
        } else {
            tile_sum<false>(gt.Pc, row, Z, [&](int, float2 v) {
                acc.x += v.x;
                acc.y += v.y;
            });
        }
    }
    if (o < nv)
        ext[sb.ext_off + gt.j0 + o] = cp.precise_sum ? make_float2((float)acc64.x, (float)acc64.y) : acc;
}

// Short arms (L <= 4) in phase groups with the NCO folded into the taps: with
// few taps per staged sample, rotating every sample costs more than the
// multiply-adds it feeds.  The tile stages raw samples (history samples, kept
// shifted, are turned back by exp(-j phi(i))), each CTA builds the modulated
// taps hc[p + uD] = h[p + uD] exp(-j (p + uD) inc) of its phases, and every
// output takes one rotation exp(j phi(n_j)) at the end:
//     y_j = exp(j phi(n_j)) * sum_k hc[k] x(n_j - k).

__host__ __device__ inline int mod_smem_bytes(int Pc, int L) {
    int z = (Pc * dense_row_stride(L) * 8 + 15) & ~15;
    if (z < kRedBytes) z = kRedBytes;
    return z + Pc * L * 8 + 16;
}

int mod_smem_bytes_host(int Pc, int L) { return mod_smem_bytes(Pc, L); }

template <int L>
__device__ __forceinline__ void mod_row(const float2 *zrow, const float2 *hrow, int lane, float *ar, float *ai) {
    constexpr int R = kDenseR;
    float2 win[R + L - 1];
#pragma unroll
    for (int tt = 0; tt < R + L - 1; ++tt) {
        const int c = lane * R + tt;
        win[tt] = zrow[c + (c >> 3)];
    }
    float2 h[L];
#pragma unroll
    for (int u = 0; u < L; ++u) h[u] = hrow[u];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
        for (int u = 0; u < L; ++u) {
            const float2 z = win[r + L - 1 - u];
            ar[r] = fmaf(h[u].x, z.x, fmaf(-h[u].y, z.y, ar[r]));
            ai[r] = fmaf(h[u].x, z.y, fmaf(h[u].y, z.x, ai[r]));
        }
    }
}

__global__ void __launch_bounds__(kDenseThreads, 3)
k_extract_mod(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
              const ChanState *__restrict__ st, const float2 *__restrict__ x, int n,
              const float2 *__restrict__ hist_arena, const float *__restrict__ taps_arena,
              float2 *__restrict__ ext) {
    extern __shared__ float4 smemm4[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    const int j0 = w.y * kDenseOT;
    if (j0 >= sb.n_out) return;
    const int L = cp.plen, D = cp.decim;
    const int M = kDenseOT + L - 1;
    const int Mp = dense_row_stride(L);
    int zb = (sb.pg * Mp * 8 + 15) & ~15;
    if (zb < kRedBytes) zb = kRedBytes;
    float2 *Z = reinterpret_cast<float2 *>(smemm4);
    float2 *hc = reinterpret_cast<float2 *>(reinterpret_cast<char *>(smemm4) + zb);
    const uint64_t u0 = st[sb.slot].nco_q;
    const uint64_t inc = cp.inc_q;
    const float *tg = taps_arena + cp.taps_off;
    const int s0 = D - sb.pc - 1;
    const float2 *hist = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
    const int H = sb.hist_len;
    auto row = [&](int pp, int lane, float *ar, float *ai) {
        const float2 *zrow = Z + pp * Mp;
        const float2 *hrow = hc + pp * L;
        switch (L) {
        case 1: mod_row<1>(zrow, hrow, lane, ar, ai); break;
        case 2: mod_row<2>(zrow, hrow, lane, ar, ai); break;
        case 3: mod_row<3>(zrow, hrow, lane, ar, ai); break;
        default: mod_row<4>(zrow, hrow, lane, ar, ai); break;
        }
    };
    const int nv = sb.n_out - j0;
    const int o = (int)threadIdx.x;  // this thread's output of the tile
    // its rotation exp(j phi(n_j)), taken by every group's share
    const float2 ph = q64_phasor(u0 + (uint64_t)(int64_t)(s0 + (j0 + o) * D) * inc);
    double2 acc64 = make_double2(0.0, 0.0);
    float2 acc = make_float2(0.f, 0.f);
    for (int g = 0; g < sb.ng; ++g) {
        const int p_lo = g * sb.pg;
        const int Pc = min(sb.pg, cp.nphase - p_lo);
        if (g) __syncthreads();  // the last group's reduction has read Z and its rows hc
        for (int i = threadIdx.x; i < Pc * L; i += kDenseThreads) {
            const int pp = i / L, u = i - pp * L;
            const int k = p_lo + pp + u * D;
            const float h = tg[(p_lo + pp) * L + u];
            const float2 t = q64_phasor((uint64_t)0 - (uint64_t)k * inc);
            hc[i] = make_float2(h * t.x, h * t.y);
        }
        // raw samples: Z[pp][m] = x(cb0 + m*D + r), pp = Pc-1-r
        const int cb0 = s0 + (j0 - (L - 1)) * D - p_lo - Pc + 1;
        const bool interior = cb0 >= 0 && cb0 + (M - 1) * D + Pc <= n;
        if (interior) {
            stage_columns(Pc, M, Mp, D, cb0, Z, [&](int i, int, int) { return __ldg(x + i); });
        } else {
            stage_columns(Pc, M, Mp, D, cb0, Z, [&](int i, int, int) {
                if (i >= n) return make_float2(0.f, 0.f);
                if (i >= 0) return __ldg(x + i);
                const int hi = H + i;
                // a carried sample is shifted already: undo its rotation
                return hi >= 0 ? cmulf(hist[hi], q64_phasor((uint64_t)0 - (u0 + (uint64_t)(int64_t)i * inc)))
                               : make_float2(0.f, 0.f);
            });
        }
        __syncthreads();
        if (cp.precise_sum) {
            tile_sum<true>(Pc, row, Z, [&](int, double2 v) {
                acc64.x += v.x * (double)ph.x - v.y * (double)ph.y;
                acc64.y += v.x * (double)ph.y + v.y * (double)ph.x;
            });
        } else {
            tile_sum<false>(Pc, row, Z, [&](int, float2 v) {
                const float2 y = cmulf(v, ph);
                acc.x += y.x;
                acc.y += y.y;
            });
        }
    }
    if (o < nv) ext[sb.ext_off + j0 + o] = cp.precise_sum ? make_float2((float)acc64.x, (float)acc64.y) : acc;
}

// ===========================================================================
// Pre-demod decimation (recorder/streamer.go:1098-1146 with
// dsp/decimating_fir.go:56-95): 101-tap float64 low-pass, one output each
// time the decimator's phase counter is 0 -- stream samples d1_phase + j*d1
// of this block -- over the newest 101 extraction outputs (earlier blocks'
// from the carried 100-sample history), float64 accumulate in the
// reference's order, complex64 output.
// ===========================================================================
constexpr int kDecOT = 256;

__global__ void __launch_bounds__(kDecOT)
k_decim2(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
         const double *__restrict__ d1taps, const float2 *__restrict__ d1hist, float2 *__restrict__ ext) {
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const int j = w.y * kDecOT + (int)threadIdx.x;
    if (j >= sb.n_dem) return;
    const ChanParams &cp = prm[sb.slot];
    const double *h = d1taps + (int64_t)sb.slot * kD1Taps;
    const float2 *hist = d1hist + (int64_t)sb.slot * kWfmHist;  // oldest first
    const float2 *x = ext + sb.ext_off;
    const int i = sb.d1_phase + j * cp.d1;
    double ar = 0.0, ai = 0.0;
    for (int k = 0; k < kD1Taps; ++k) {
        const int q = i - k;
        const float2 v = q >= 0 ? x[q] : hist[kWfmHist + q];
        ar = __dadd_rn(ar, __dmul_rn((double)v.x, h[k]));
        ai = __dadd_rn(ai, __dmul_rn((double)v.y, h[k]));
    }
    ext[sb.dem_off + j] = make_float2((float)ar, (float)ai);
}

// ===========================================================================
// Demodulators (internal/demod/*.go; bridge per recorder/streamer.go:1287-1302)
// ===========================================================================
constexpr int kDemodOT = 1024;

__global__ void __launch_bounds__(256)
k_demod(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
        const ChanState *__restrict__ st, const float2 *__restrict__ ext, float *__restrict__ comp,
        float *__restrict__ audio) {
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    const int q0 = w.y * kDemodOT;
    const float2 *iq = ext + sb.dem_off;
    const int mode = cp.mode;
    if (mode == 1 || mode == 2 || mode == 3) {  // NFM / WFM / WFM_STEREO: fmDiscrimInto (fm.go:179-196)
        const float2 last = st[sb.slot].last_iq;
        float *dst = (mode == 1) ? (audio + sb.audio_off) : (comp + sb.comp_off);
        for (int q = q0 + threadIdx.x; q < q0 + kDemodOT && q < sb.n_disc; q += blockDim.x) {
            float2 p, c;
            if (sb.bridge) {
                p = q == 0 ? last : iq[q - 1];
                c = iq[q];
            } else {
                p = iq[q];
                c = iq[q + 1];
            }
            double num = (double)p.x * (double)c.y - (double)p.y * (double)c.x;
            double den = (double)p.x * (double)c.x + (double)p.y * (double)c.y;
            dst[q] = (float)atan2(num, den);
        }
    } else if (mode == 5 || mode == 6 || mode == 7) {  // ssb.go:19-39, cw.go:11-26
        float *dst = audio + sb.audio_off;
        for (int q = q0 + threadIdx.x; q < q0 + kDemodOT && q < sb.n_dem; q += blockDim.x) {
            double ph = (double)(q + 1) * cp.ssb_inc;
            double s, c;
            sincos(ph, &s, &c);
            float2 v = iq[q];
            dst[q] = (mode == 7) ? (float)((double)v.x * c) : (float)((double)v.x * c - (double)v.y * s);
        }
    }
}

// AM.Demod (am.go:11-27): envelope minus the per-call mean.  One CTA per slot.
__global__ void __launch_bounds__(256)
k_am(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const float2 *__restrict__ ext,
     float *__restrict__ audio) {
    __shared__ double red[256];
    const SlotBlock sb = sbt[work[blockIdx.x].x];
    const float2 *iq = ext + sb.dem_off;
    double acc = 0.0;
    for (int q = threadIdx.x; q < sb.n_dem; q += 256) acc += hypot((double)iq[q].x, (double)iq[q].y);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const float mean = (float)(red[0] / (double)sb.n_dem);
    float *dst = audio + sb.audio_off;
    for (int q = threadIdx.x; q < sb.n_dem; q += 256) {
        float mag = (float)hypot((double)iq[q].x, (double)iq[q].y);
        dst[q] = mag - mean;
    }
}

// ===========================================================================
// WFM multiplex (recorder/streamer.go:1525-1644)
// ===========================================================================
//
// Rate-class tables: the stereo filters as float taps padded to 104
//   x = LPF 15 kHz (L+R and L-R lowpass), y = LPF 53 kHz - LPF 23 kHz (L-R
//   band), z = LPF 21 kHz - LPF 17 kHz (pilot band); the band-pass pairs are
//   differenced in float64 before rounding, one filter each instead of two;
// and the RDS lowpass (7.5 kHz, fm.go:155) in float64.
constexpr int kWfmTapsPad = 104;
struct WfmTaps {
    float4 t[kWfmTapsPad];
    double rds[kWfmTaps];
};

// Composite-rate work arrays (all float, same offsets comp_off):
//   work + 0*W comp (discriminator output), 1*W lpr, 2*W bpf, 3*W pilot, 4*W lr
constexpr int kFirOT = 1024;   // composite samples per tile
constexpr int kAudioDlStride = kWfmHist + 4;  // 100 samples + valid count
constexpr int kFirThreads = 128;  // 8 outputs each

__host__ __device__ constexpr int padi(int e) { return e + (e >> 3); }

// Loads composite samples [q0-104, q0+kFirOT) into shared memory; indices
// below 0 come from the 100-sample delay line `dl` (oldest first, newest at
// 99) with `valid` trailing entries, zero before that.
__device__ __forceinline__ void stage_window(float *win, const float *__restrict__ src, int q0, int nvalid,
                                             const float *__restrict__ dl, int valid) {
    for (int i = threadIdx.x; i < kFirOT + kWfmTapsPad; i += blockDim.x) {
        int q = q0 - kWfmTapsPad + i;
        float v = 0.f;
        if (q >= 0) {
            if (q < nvalid) v = src[q];
        } else if (q >= -valid) {
            v = dl[kWfmHist + q];
        }
        win[padi(i)] = v;
    }
}

__global__ void __launch_bounds__(kFirThreads)
k_wfm_fir(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
          const WfmTaps *__restrict__ taps, float *__restrict__ wk, int W, const float *__restrict__ comp_dl) {
    __shared__ float win[padi(kFirOT + kWfmTapsPad) + 8];
    __shared__ float4 tp[kWfmTapsPad];
    __shared__ float s_out[3 * (kFirOT + kFirOT / 32)];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    const int q0 = w.y * kFirOT;
    if (q0 >= sb.n_disc) return;
    const WfmTaps &tb = taps[cp.rds_tab];
    for (int i = threadIdx.x; i < kWfmTapsPad; i += kFirThreads) tp[i] = tb.t[i];
    const float *comp = wk + sb.comp_off;
    stage_window(win, comp, q0, sb.n_disc, comp_dl + cp.wfm_idx * kWfmHist, sb.comp_hist_len);
    __syncthreads();
    const int t = threadIdx.x;
    // window index of composite sample q0 + 8t + r - k is 8t + r - k + 104
    const int base = 8 * t + kWfmTapsPad;
    float a[8], b[8], c[8], ring[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) a[r] = b[r] = c[r] = 0.f;
#pragma unroll
    for (int j = 1; j < 8; ++j) ring[j] = win[padi(base + j)];
    for (int kb = 0; kb < kWfmTapsPad; kb += 8) {
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const int k = kb + kk;
            ring[(8 - kk) & 7] = win[padi(base - k)];
            const float4 h = tp[k];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const float v = ring[(r - kk + 8) & 7];
                a[r] = fmaf(h.x, v, a[r]);
                b[r] = fmaf(h.y, v, b[r]);
                c[r] = fmaf(h.z, v, c[r]);
            }
        }
    }
    // outputs through shared memory (index i + i/32: conflict-free both
    // ways), then coalesced stores of the three arrays
    constexpr int kS = kFirOT + kFirOT / 32;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = 8 * t + r, j = i + (i >> 5);
        s_out[j] = a[r];
        s_out[kS + j] = b[r];
        s_out[2 * kS + j] = c[r];
    }
    __syncthreads();
    float *lpr = wk + 1 * W + sb.comp_off, *bpf = wk + 2 * W + sb.comp_off, *pil = wk + 3 * W + sb.comp_off;
    const int nq = min(kFirOT, sb.n_disc - q0);
    for (int i = t; i < nq; i += kFirThreads) {
        const int j = i + (i >> 5);
        lpr[q0 + i] = s_out[j];
        bpf[q0 + i] = s_out[kS + j];
        pil[q0 + i] = s_out[2 * kS + j];
    }
}

struct PllK {
    double alpha, beta;
    float lpa;
    double dfmin, dfmax;  // frequency clamp as deviations from the block-start frequency
    uint64_t q0, qf;      // block-start phase and frequency in Q0.64 turns
};

// One loop step (recorder/streamer.go:1588-1613) in deviation form: the phase
// is phase0 + t*freq0 + dphi, the frequency freq0 + df (dphi, df float64); the
// ramp phase0 + t*freq0 is exact in Q0.64 turns, so the sin/cos argument needs
// no float64 range reduction.  The I/Q lowpass states are float32.  The serial
// loop and the Newton solver both use this step, so they iterate the same map.
struct PllEval {
    double dphi1, df1;
    float I1, Q1;
    float e;
    float ja, jb, jc, jd;   // phase row: d/dphase, d/dfreq, d/dI, d/dQ
    float ka, kb, kc, kd;   // freq row
    float iphi, qphi;       // I/Q rows' d/dphase (diagonals are 1 - lpa)
};

// q: the ramp phase phase0 + t*freq0 of step t in Q0.64 turns (callers carry
// it by adding k.qf per step: the same integer as k.q0 + t*k.qf).
__device__ __forceinline__ void pll_angle(uint64_t q, double dphi, float &s, float &c) {
    const float h = (float)(int32_t)(q >> 32) * 4.656612873077393e-10f + (float)(dphi * (1.0 / GPUD_PI));
    __sincosf(h * 3.14159265358979f, &s, &c);  // |angle| <= pi + |dphi|
}

template <bool kJac>
__device__ __forceinline__ void pll_step(uint64_t q, double dphi, double df, float I, float Q, float p, const PllK &k,
                                         PllEval &o) {
    float sn, cs;
    pll_angle(q, dphi, sn, cs);
    o.I1 = fmaf(k.lpa, fmaf(p, cs, -I), I);
    o.Q1 = fmaf(k.lpa, fmaf(p, -sn, -Q), Q);
    const float e = atan2f(o.Q1, o.I1);
    o.e = e;
    double d = df + k.beta * (double)e;
    bool clamped = false;
    if (d < k.dfmin) {
        d = k.dfmin;
        clamped = true;
    } else if (d > k.dfmax) {
        d = k.dfmax;
        clamped = true;
    }
    o.df1 = d;
    o.dphi1 = dphi + d + k.alpha * (double)e;
    if (kJac) {
        // the Jacobian sets the convergence rate only, not the fixed point:
        // an approximate reciprocal is enough
        const float r2 = fmaf(o.I1, o.I1, o.Q1 * o.Q1);
        const float inv = r2 > 0.f ? __fdividef(1.f, r2) : 0.f;
        const float gI = -o.Q1 * inv, gQ = o.I1 * inv;
        const float dIphi = -k.lpa * p * sn;  // d/dphase of lpa*p*cos(phase)
        const float dQphi = -k.lpa * p * cs;  // d/dphase of -lpa*p*sin(phase)
        const float ePhi = fmaf(gI, dIphi, gQ * dQphi);
        const float om = 1.f - k.lpa;
        const float eI = gI * om, eQ = gQ * om;
        const float g = clamped ? 0.f : (float)k.beta, h = clamped ? 0.f : 1.f;
        const float ga = g + (float)k.alpha;
        o.ka = g * ePhi;
        o.kb = h;
        o.kc = g * eI;
        o.kd = g * eQ;
        o.ja = 1.f + ga * ePhi;
        o.jb = h;
        o.jc = ga * eI;
        o.jd = ga * eQ;
        o.iphi = dIphi;
        o.qphi = dQphi;
    }
}

__device__ __forceinline__ PllK pll_consts(const ChanParams &cp, const ChanState &s) {
    PllK k;
    k.alpha = cp.pll_alpha;
    k.beta = cp.pll_beta;
    k.lpa = (float)cp.pll_lpa;
    k.dfmin = cp.pll_fmin - s.pll_freq;
    k.dfmax = cp.pll_fmax - s.pll_freq;
    k.q0 = rad_to_q64(s.pll_phase);
    k.qf = rad_to_q64(s.pll_freq);
    return k;
}

// Loop phase after t steps, wrapped to [0, 2pi) (the serial loop's range).
__device__ __forceinline__ double pll_phase_at(const PllK &k, int t, double dphi) {
    const uint64_t q = k.q0 + (uint64_t)t * k.qf;
    double ph = (double)q * (2.0 * GPUD_PI / 18446744073709551616.0) + dphi;
    ph -= (2.0 * GPUD_PI) * floor(ph * (1.0 / (2.0 * GPUD_PI)));
    return ph;
}

// 2*sin(2*phase) of the loop phase, float32 (lr = bpf * that); q is the ramp
// phase of the same step in Q0.64 turns.
__device__ __forceinline__ float pll_two_sin2(uint64_t q, double dphi) {
    const uint64_t q2 = 2 * q;
    const float h = (float)(int32_t)(q2 >> 32) * 4.656612873077393e-10f + (float)(dphi * (2.0 / GPUD_PI));
    return 2.0f * sinpif(h);
}

// End of one stereoDecodeStateful call: store the loop state, update errAvg
// (EMA per call), the coherence / frequency / errAvg lock test and the
// hysteresis counters (streamer.go:1614-1635, 1363-1380).
__device__ void pll_finish(ChanState &s, const ChanParams &cp, int n, double ph, double fr, double I, double Q,
                           double es, double pp) {
    const double twopi = 2.0 * GPUD_PI;
    s.pll_phase = ph;
    s.pll_freq = fr;
    s.pll_i = I;
    s.pll_q = Q;
    const double block_err = es / (double)n;
    if (cp.flags & kChBatchStereo) {
        // wfmStereoDecodeBatch (wfm_batch_stereo.go:137-142): one call, no
        // hysteresis; locked by the pilot-band share of the composite's power
        const double ratio = s.comp_power > 0.0 ? pp / s.comp_power : 0.0;
        const double fhz = fr * (double)cp.out_rate / twopi;
        const int locked = ratio > 0.003 && fabs(fhz - 19000.0) < 250.0 && block_err < 0.35;
        s.locked = locked;
        s.enabled = locked;
        s.coherence = (float)ratio;
        s.pilot_hz = (float)fhz;
        s.last_err_avg = (float)block_err;
        return;
    }
    const double ea = 0.9 * s.err_avg + 0.1 * block_err;
    s.err_avg = ea;
    double coherence = 0.0;
    if (pp > 1e-12) coherence = (I * I + Q * Q) * (double)n / pp;
    const double fhz = fr * (double)cp.out_rate / twopi;
    const int locked = coherence > 0.15 && fabs(fhz - 19000.0) < 250.0 && ea < 0.35;
    s.locked = locked;
    s.coherence = (float)coherence;
    s.pilot_hz = (float)fhz;
    s.last_err_avg = (float)ea;
    if (locked) {
        s.on_count += 1;
        s.off_count = 0;
        if (s.on_count >= 4) s.enabled = 1;
    } else {
        s.on_count = 0;
        s.off_count += 1;
        if (s.off_count >= 10) s.enabled = 0;
    }
}

// Pilot PLL, serial per channel (recorder/streamer.go:1560-1619).  Phase,
// frequency and the I/Q lowpass states are float64 (the frequency integrator
// moves by ~1e-10 rad/sample, below float32 resolution); the loop's sin/cos and
// atan2 are float32.  One CTA per channel: lane 0 of warp 0 runs the recurrence
// from shared memory; warp 1 prefetches the next chunk of the pilot band and
// finishes the previous chunk off the critical path (lr = bpf * float32(2 sin
// 2phase), pilot power).  Per-call lock decision and hysteresis at the end
// (streamer.go:1363-1380, 1615-1635).
constexpr int kPllChunk = 2048;

__global__ void __launch_bounds__(64)
k_pll(const int *__restrict__ list, int count, const SlotBlock *__restrict__ sbt,
      const ChanParams *__restrict__ prm, ChanState *__restrict__ st, float *__restrict__ wk, int W) {
    __shared__ float s_pil[2][kPllChunk];
    __shared__ float s_th[2][kPllChunk];
    __shared__ double s_red[32];
    const int idx = blockIdx.x;
    if (idx >= count) return;
    const SlotBlock sb = sbt[list[idx]];
    const int n = sb.n_disc;
    if (n <= 0) return;
    const ChanParams &cp = prm[sb.slot];
    ChanState &s = st[sb.slot];
    const float *pil = wk + 3 * W + sb.comp_off;
    const float *bpf = wk + 2 * W + sb.comp_off;
    float *lr = wk + 4 * W + sb.comp_off;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nc = (n + kPllChunk - 1) / kPllChunk;
    double pp = 0.0;  // pilot power, accumulated by warp 1
    // prologue: chunk 0 into buffer 0
    if (warp == 1) {
        for (int q = lane; q < min(n, kPllChunk); q += 32) s_pil[0][q] = pil[q];
    }
    __syncthreads();
    const PllK k = pll_consts(cp, s);
    double dphi = 0.0, df = 0.0, es = 0.0;
    float I = (float)s.pll_i, Q = (float)s.pll_q;
    for (int c = 0; c <= nc; ++c) {
        if (warp == 0) {
            if (lane == 0 && c < nc) {
                const float *sp = s_pil[c & 1];
                float *th = s_th[c & 1];
                const int base = c * kPllChunk;
                const int len = min(kPllChunk, n - base);
                uint64_t qr = k.q0 + (uint64_t)base * k.qf;
                for (int q = 0; q < len; ++q) {
                    PllEval o;
                    pll_step<false>(qr, dphi, df, I, Q, sp[q], k, o);
                    qr += k.qf;
                    dphi = o.dphi1;
                    df = o.df1;
                    I = o.I1;
                    Q = o.Q1;
                    es += fabs((double)o.e);
                    th[q] = pll_two_sin2(qr, dphi);
                }
            }
        } else {
            // finish chunk c-1, then prefetch chunk c+1 into the buffer it frees
            if (c >= 1) {
                const int base = (c - 1) * kPllChunk;
                const int len = min(kPllChunk, n - base);
                const float *th = s_th[(c - 1) & 1];
                const float *sp = s_pil[(c - 1) & 1];
                for (int q = lane; q < len; q += 32) {
                    const double p = (double)sp[q];
                    pp += p * p;
                    lr[base + q] = bpf[base + q] * th[q];
                }
            }
            __syncwarp();
            if (c + 1 < nc) {
                const int base = (c + 1) * kPllChunk;
                const int len = min(kPllChunk, n - base);
                float *dst = s_pil[(c + 1) & 1];
                for (int q = lane; q < len; q += 32) dst[q] = pil[base + q];
            }
        }
        __syncthreads();
    }
    if (warp == 1) {
        for (int off = 16; off > 0; off >>= 1) pp += __shfl_xor_sync(0xffffffffu, pp, off);
        if (lane == 0) s_red[0] = pp;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    pll_finish(s, cp, n, pll_phase_at(k, n, dphi), s.pll_freq + df, (double)I, (double)Q, es, s_red[0]);
    s.pll_path = 2;
}


// ===========================================================================
// Pilot PLL, parallel in time: multiple-shooting Newton.
// ===========================================================================
// The block's loop trajectory x_t = (phase, freq, I, Q), t = 0..n, obeys
// x_{t+1} = F(x_t, p_t) with the serial kernel's exact step F.  The block is
// cut into one segment of S consecutive steps per thread; the unknowns are the
// segment start states s_g.  Each iteration every thread integrates its
// segment with F from s_g (the exact nonlinear loop, no linearisation inside
// the segment), giving the end state E_g(s_g) and the segment Jacobian
// M_g = J_{t1-1} ... J_{t0}.  Newton's update of the start states,
//     d_{g+1} = M_g d_g + (E_g(s_g) - s_{g+1}),   d_0 = 0,   s_g <- s_g + d_g,
// is a linear recurrence over segments, solved by an associative scan over
// affine maps (4x4 matrix + vector, float32; states and residuals float64 /
// float32 as in F): warp shuffles, then shared memory across warps, then
// distributed shared memory across the cluster's CTAs.  The fixed point is the
// serial trajectory.  From the free-running guess s_g = (phase_0 + t0 freq_0,
// freq_0, I_0, Q_0) a locked loop converges in 3-5 iterations; acquisition
// from zero I/Q and noise-driven loops (no pilot) take tens to a hundred, since
// a segment whose start is exact is exact after one more iteration.  A block
// not converged after max_iters iterations keeps its consistent prefix and one
// thread runs the serial loop over the rest.  No trajectory is stored: a last
// pass integrates each segment from its converged start and writes the
// outputs.
#ifndef GPUD_PLL_CLUSTER
#define GPUD_PLL_CLUSTER 8  // CTAs per channel at most: segment length max(16, n / (256 * this))
#endif
#ifndef GPUD_PLL_JAC_SWEEPS
#define GPUD_PLL_JAC_SWEEPS 2  // sweeps that evaluate the segment Jacobians before chord steps may start
#endif
constexpr int kNewtonThreads = 256;
constexpr int kNewtonMaxCluster = GPUD_PLL_CLUSTER;
constexpr int kNewtonMinSeg = 16;

// Steps per segment (per thread) for a block of n loop steps.
__host__ __device__ inline int pll_segment_len(int n) {
    const int cap = kNewtonMaxCluster * kNewtonThreads;
    const int s = (n + cap - 1) / cap;
    return s > kNewtonMinSeg ? s : kNewtonMinSeg;
}

// CTAs per cluster that give every channel of a launch (at most max_n steps)
// one thread per segment.
int pll_cluster_for(int max_n) {
    const int seg = (max_n + pll_segment_len(max_n) - 1) / pll_segment_len(max_n);
    int c = (seg + kNewtonThreads - 1) / kNewtonThreads;
    int p = 1;
    while (p < c) p *= 2;
    return p < 1 ? 1 : (p > kNewtonMaxCluster ? kNewtonMaxCluster : p);
}
// Convergence: the last correction of every segment start is below what the
// outputs resolve (the float32 sin/cos/atan2 and lowpass states leave a floor
// near 1e-10 rad and 1e-9 in I/Q).
constexpr float kTolPhase = 1e-8f, kTolFreq = 1e-12f, kTolIQ = 1e-7f;
constexpr int kNW = kNewtonThreads / 32;

struct Aff {
    float a[16];  // row-major, state order (phase, freq, I, Q)
    float b[4];
};

// M <- J M, with J's sparsity (phase/freq rows dense, I/Q rows phase + diagonal).
__device__ __forceinline__ void mat_push(float (&m)[16], const PllEval &o, float om) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float p0 = m[j], f0 = m[4 + j], i0 = m[8 + j], q0 = m[12 + j];
        m[j] = fmaf(o.ja, p0, fmaf(o.jb, f0, fmaf(o.jc, i0, o.jd * q0)));
        m[4 + j] = fmaf(o.ka, p0, fmaf(o.kb, f0, fmaf(o.kc, i0, o.kd * q0)));
        m[8 + j] = fmaf(o.iphi, p0, om * i0);
        m[12 + j] = fmaf(o.qphi, p0, om * q0);
    }
}

// hi o lo (lo applied first)
__device__ __forceinline__ void aff_compose(Aff &out, const Aff &hi, const Aff &lo) {
    Aff r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            r.a[4 * i + j] = fmaf(hi.a[4 * i], lo.a[j],
                                  fmaf(hi.a[4 * i + 1], lo.a[4 + j],
                                       fmaf(hi.a[4 * i + 2], lo.a[8 + j], hi.a[4 * i + 3] * lo.a[12 + j])));
        }
        r.b[i] = fmaf(hi.a[4 * i], lo.b[0],
                      fmaf(hi.a[4 * i + 1], lo.b[1], fmaf(hi.a[4 * i + 2], lo.b[2], fmaf(hi.a[4 * i + 3], lo.b[3], hi.b[i]))));
    }
    out = r;
}

__device__ __forceinline__ void aff_shfl_up(Aff &dst, const Aff &src, int d) {
#pragma unroll
    for (int i = 0; i < 16; ++i) dst.a[i] = __shfl_up_sync(0xffffffffu, src.a[i], d);
#pragma unroll
    for (int i = 0; i < 4; ++i) dst.b[i] = __shfl_up_sync(0xffffffffu, src.b[i], d);
}

__device__ __forceinline__ void aff_identity(Aff &m) {
#pragma unroll
    for (int i = 0; i < 16; ++i) m.a[i] = (i % 5 == 0) ? 1.f : 0.f;
#pragma unroll
    for (int i = 0; i < 4; ++i) m.b[i] = 0.f;
}

__device__ __forceinline__ void aff_load(Aff &m, const float *src) {
#pragma unroll
    for (int i = 0; i < 16; ++i) m.a[i] = src[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) m.b[i] = src[16 + i];
}

__device__ __forceinline__ void aff_store(float *dst, const Aff &m) {
#pragma unroll
    for (int i = 0; i < 16; ++i) dst[i] = m.a[i];
#pragma unroll
    for (int i = 0; i < 4; ++i) dst[16 + i] = m.b[i];
}

__device__ __forceinline__ void aff_apply(float out[4], const Aff &m, const float x[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
        out[i] = fmaf(m.a[4 * i], x[0], fmaf(m.a[4 * i + 1], x[1], fmaf(m.a[4 * i + 2], x[2], fmaf(m.a[4 * i + 3], x[3], m.b[i]))));
}

// Segment start state, deviation form (see pll_step).
struct SegState {
    double dphi, df;
    float I, Q;
};

// One channel-block per cluster of `gridDim.x / count` CTAs; the block's steps
// are split into one contiguous segment per thread of the cluster.  With
// segments of at most kPllStageS steps (blocks of up to 32768 composite
// samples) each CTA first stages its span of the pilot band in shared memory,
// transposed (step i of thread j's segment at [i][j], conflict-free), so every
// Newton sweep reads it from there; the output sweep writes 2 sin(2 phase)
// back into the same cells and the CTA then writes the L-R products with
// coalesced stores.
constexpr int kPllStageS = 16;

__global__ void __launch_bounds__(kNewtonThreads, 3)
k_pll_newton(const int *__restrict__ list, int count, const SlotBlock *__restrict__ sbt,
             const ChanParams *__restrict__ prm, ChanState *__restrict__ st, float *__restrict__ wk, int W,
             int max_iters) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    __shared__ float s_tot[kNW][20];     // warp totals
    __shared__ float s_wex[kNW][20];     // exclusive warp prefix (A, b) within the CTA
    __shared__ float s_cta[2][20];       // CTA total, double-buffered across iterations
    __shared__ float s_max[kNW][4];
    __shared__ float s_cmax[2][4];       // CTA max |d|, double-buffered
    __shared__ float s_dcta[4];          // d at this CTA's first segment
    __shared__ SegState s_first[kNW];    // each warp's first segment start (lane 0)
    __shared__ float s_jac[16][kNewtonThreads];  // each segment's Jacobian, kept for chord steps
    __shared__ float s_seg[kPllStageS][kNewtonThreads + 1];  // staged pilot band / 2 sin(2 phase)
    __shared__ double s_sum[kNW][2];
    __shared__ double s_csum[2];
    const int csize = (int)cl.num_blocks();
    const int crank = (int)cl.block_rank();
    const int idx = blockIdx.x / csize;
    if (idx >= count) return;  // uniform per cluster
    const SlotBlock sb = sbt[list[idx]];
    const int n = sb.n_disc;
    if (n <= 0) return;  // uniform per cluster
    const ChanParams &cp = prm[sb.slot];
    ChanState &s = st[sb.slot];
    const float *pil = wk + 3 * W + sb.comp_off;
    const float *bpf = wk + 2 * W + sb.comp_off;
    float *lr = wk + 4 * W + sb.comp_off;
    const PllK k = pll_consts(cp, s);
    const float om = 1.f - k.lpa;
    const float I0 = (float)s.pll_i, Q0 = (float)s.pll_q;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // The segment length depends on the channel's own block length only, so a
    // channel's trajectory (and every rounding in it) is the same whatever
    // other channels share the launch; the cluster supplies at least
    // ceil(n / S) threads.
    const int S = pll_segment_len(n);
    const int g = crank * kNewtonThreads + (int)threadIdx.x;
    const int t0 = min(n, g * S), t1 = min(n, t0 + S);
    const bool has_next = t1 < n;  // the next thread's segment is not empty
    const bool staged = S <= kPllStageS;  // uniform
    const int cbase = min(n, crank * kNewtonThreads * S);
    const int cend = min(n, cbase + kNewtonThreads * S);
    if (staged) {
        for (int t = cbase + (int)threadIdx.x; t < cend; t += kNewtonThreads) {
            const int r = t - cbase;
            s_seg[r % S][r / S] = __ldg(pil + t);
        }
        __syncthreads();
    }
    auto pilot = [&](int t) -> float { return staged ? s_seg[t - t0][threadIdx.x] : __ldg(pil + t); };
    SegState x0{0.0, 0.0, I0, Q0};  // this segment's start: the free-running guess
    bool converged = false, bad = true;
    float prev_m0 = 1e30f;  // last iteration's largest phase correction (uniform in the cluster)
    int iters = 0;
    for (int it = 0; it < max_iters && !converged; ++it) {
        iters = it + 1;
        const int pb = it & 1;
        // ---- the next segment's start state ------------------------------
        SegState nx{0.0, 0.0, I0, Q0};
        {
            const double a = __shfl_down_sync(0xffffffffu, x0.dphi, 1);
            const double b = __shfl_down_sync(0xffffffffu, x0.df, 1);
            const float c = __shfl_down_sync(0xffffffffu, x0.I, 1);
            const float d = __shfl_down_sync(0xffffffffu, x0.Q, 1);
            if (it > 0 && has_next) {
                if (lane < 31)
                    nx = SegState{a, b, c, d};
                else if (warp < kNW - 1)
                    nx = s_first[warp + 1];
                else
                    nx = *cl.map_shared_rank(&s_first[0], crank + 1);
            }
        }
        // ---- integrate the segment: end state and Jacobian ----------------
        // Close to the solution (the last corrections below 1e-2 rad) the
        // segment Jacobians barely move: they are kept from the last full
        // evaluation (chord steps), which converge as fast as Newton there.
        const bool jac = it < GPUD_PLL_JAC_SWEEPS || prev_m0 > 1e-2f;
        Aff m;
        aff_identity(m);
        SegState x = x0;
        if (t0 < t1) {
            uint64_t qr = k.q0 + (uint64_t)t0 * k.qf;
            if (jac) {
                for (int t = t0; t < t1; ++t) {
                    PllEval o;
                    pll_step<true>(qr, x.dphi, x.df, x.I, x.Q, pilot(t), k, o);
                    qr += k.qf;
                    mat_push(m.a, o, om);
                    x = SegState{o.dphi1, o.df1, o.I1, o.Q1};
                }
#pragma unroll
                for (int i = 0; i < 16; ++i) s_jac[i][threadIdx.x] = m.a[i];
            } else {
                for (int t = t0; t < t1; ++t) {
                    PllEval o;
                    pll_step<false>(qr, x.dphi, x.df, x.I, x.Q, pilot(t), k, o);
                    qr += k.qf;
                    x = SegState{o.dphi1, o.df1, o.I1, o.Q1};
                }
#pragma unroll
                for (int i = 0; i < 16; ++i) m.a[i] = s_jac[i][threadIdx.x];
            }
            if (has_next) {
                m.b[0] = (float)(x.dphi - nx.dphi);
                m.b[1] = (float)(x.df - nx.df);
                m.b[2] = x.I - nx.I;
                m.b[3] = x.Q - nx.Q;
            }
        }
        // ---- scan: d at each segment start -------------------------------
        Aff inc = m;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            Aff o;
            aff_shfl_up(o, inc, d);
            if (lane >= d) aff_compose(inc, inc, o);
        }
        Aff exl;  // lanes before this one
        aff_shfl_up(exl, inc, 1);
        if (lane == 0) aff_identity(exl);
        if (lane == 31) aff_store(s_tot[warp], inc);
        __syncthreads();
        if (warp == 0) {
            Aff wv;
            if (lane < kNW) aff_load(wv, s_tot[lane]);
            else aff_identity(wv);
            // only lanes 0..kNW-1 carry warp totals: log2(kNW) rounds
#pragma unroll
            for (int d = 1; d < kNW; d <<= 1) {
                Aff o;
                aff_shfl_up(o, wv, d);
                if (lane >= d) aff_compose(wv, wv, o);
            }
            Aff ex;
            aff_shfl_up(ex, wv, 1);
            if (lane == 0) aff_identity(ex);
            if (lane < kNW) aff_store(s_wex[lane], ex);
            if (lane == kNW - 1) aff_store(s_cta[pb], wv);
        }
        cl.sync();  // CTA totals of the whole cluster are visible
        // d at this CTA's first segment: the CTA totals before it, composed by
        // a scan across warp 0's lanes (lane r holds CTA r's total) and
        // applied to a zero correction
        if (warp == 0) {
            Aff tv;
            if (lane < crank) aff_load(tv, cl.map_shared_rank(&s_cta[pb][0], lane));
            else aff_identity(tv);
#pragma unroll
            for (int d = 1; d < kNewtonMaxCluster; d <<= 1) {
                Aff o;
                aff_shfl_up(o, tv, d);
                if (lane >= d) aff_compose(tv, tv, o);
            }
            const int src = crank > 0 ? crank - 1 : 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float v = __shfl_sync(0xffffffffu, tv.b[i], src);
                if (lane == 0) s_dcta[i] = crank > 0 ? v : 0.f;
            }
        }
        __syncthreads();
        const float dcta[4] = {s_dcta[0], s_dcta[1], s_dcta[2], s_dcta[3]};
        float dl[4];
        {
            Aff wx;
            aff_load(wx, s_wex[warp]);
            float dw[4];
            aff_apply(dw, wx, dcta);
            aff_apply(dl, exl, dw);
        }
        // ---- update the start state --------------------------------------
        float mx[4] = {0.f, 0.f, 0.f, 0.f};
        bad = false;
        if (t0 < t1) {
            bad = fabsf(dl[0]) > kTolPhase || fabsf(dl[1]) > kTolFreq || fabsf(dl[2]) > kTolIQ ||
                  fabsf(dl[3]) > kTolIQ;
            x0.dphi += (double)dl[0];
            x0.df += (double)dl[1];
            x0.I += dl[2];
            x0.Q += dl[3];
            mx[0] = fabsf(dl[0]);
            mx[1] = fabsf(dl[1]);
            mx[2] = fabsf(dl[2]);
            mx[3] = fabsf(dl[3]);
        }
        if (lane == 0) s_first[warp] = x0;
        // ---- convergence, agreed by every CTA of the cluster ---------------
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int i = 0; i < 4; ++i) mx[i] = fmaxf(mx[i], __shfl_xor_sync(0xffffffffu, mx[i], off));
        if (lane == 0)
#pragma unroll
            for (int i = 0; i < 4; ++i) s_max[warp][i] = mx[i];
        __syncthreads();
        if (threadIdx.x < 4) {
            float v = 0.f;
            for (int w2 = 0; w2 < kNW; ++w2) v = fmaxf(v, s_max[w2][threadIdx.x]);
            s_cmax[pb][threadIdx.x] = v;
        }
        cl.sync();  // also publishes s_first for the next iteration's reads
        float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f;
        for (int r = 0; r < csize; ++r) {
            const float *rm = cl.map_shared_rank(&s_cmax[pb][0], r);
            m0 = fmaxf(m0, rm[0]);
            m1 = fmaxf(m1, rm[1]);
            m2 = fmaxf(m2, rm[2]);
            m3 = fmaxf(m3, rm[3]);
        }
        converged = (m0 <= kTolPhase && m1 <= kTolFreq && m2 <= kTolIQ && m3 <= kTolIQ);
        // Accepted one iteration early when the next correction is predicted
        // below the tolerance: corrections shrinking at least linearly at rate
        // m0 / prev_m0 leave a next one of m0^2 / prev_m0 (Newton's quadratic
        // rate leaves less), with the other components already near their floor.
        if (!converged && it >= 1 && m0 <= 1e-5f && m0 * m0 <= kTolPhase * prev_m0 && m1 <= 1e-10f &&
            m2 <= 1e-6f && m3 <= 1e-6f)
            converged = true;
        prev_m0 = m0;
    }
    // ---- not converged: the longest consistent prefix is kept ------------
    // Segments before the first one whose start still moved by more than the
    // tolerance form a consistent trajectory from the block start, and that
    // segment's updated start is its exact start; one thread continues the
    // serial loop from there to the block end.
    __shared__ int s_bad[kNW];
    __shared__ int s_cbad;
    int gstar = INT_MAX;
    if (!converged) {
        int v = bad ? g : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, off));
        if (lane == 0) s_bad[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            int c = INT_MAX;
            for (int w2 = 0; w2 < kNW; ++w2) c = min(c, s_bad[w2]);
            s_cbad = c;
        }
        cl.sync();
        for (int r = 0; r < csize; ++r) gstar = min(gstar, *cl.map_shared_rank(&s_cbad, r));
        if (gstar == INT_MAX) gstar = 0;  // cannot happen (not converged means one start moved)
    }
    // ---- outputs: each converged segment again from its start --------------
    double es = 0.0, pp = 0.0;
    SegState x = x0;
    if (t0 < t1) {
        const bool out = g < gstar;
        uint64_t qr = k.q0 + (uint64_t)t0 * k.qf;
        for (int t = t0; t < t1; ++t) {
            const float pt = pilot(t);
            pp += (double)pt * (double)pt;
            if (out) {
                PllEval o;
                pll_step<false>(qr, x.dphi, x.df, x.I, x.Q, pt, k, o);
                qr += k.qf;
                x = SegState{o.dphi1, o.df1, o.I1, o.Q1};
                es += fabs((double)o.e);
                const float th = pll_two_sin2(qr, x.dphi);
                if (staged)
                    s_seg[t - t0][threadIdx.x] = th;  // this thread's own cell, already read
                else
                    lr[t] = bpf[t] * th;
            }
        }
    }
    if (staged) {
        // the L-R products of this CTA's output segments, coalesced
        __syncthreads();
        for (int t = cbase + (int)threadIdx.x; t < cend; t += kNewtonThreads) {
            const int r = t - cbase;
            if (crank * kNewtonThreads + r / S < gstar) lr[t] = bpf[t] * s_seg[r % S][r / S];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        es += __shfl_xor_sync(0xffffffffu, es, off);
        pp += __shfl_xor_sync(0xffffffffu, pp, off);
    }
    if (lane == 0) {
        s_sum[warp][0] = es;
        s_sum[warp][1] = pp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int w2 = 0; w2 < kNW; ++w2) {
            a += s_sum[w2][0];
            b += s_sum[w2][1];
        }
        s_csum[0] = a;
        s_csum[1] = b;
    }
    cl.sync();
    // the owner finishes the block: the thread holding the last segment, or
    // the thread at the first inconsistent segment start
    const int owner = converged ? (n - 1) / S : gstar;
    double es_all = 0.0, pp_all = 0.0;
    if (g == owner) {
        for (int r = 0; r < csize; ++r) {
            const double *rs = cl.map_shared_rank(&s_csum[0], r);
            es_all += rs[0];
            pp_all += rs[1];
        }
    }
    cl.sync();  // no shared memory of another CTA is read after this
    if (converged) {
        if (g != owner) return;
        pll_finish(s, cp, n, pll_phase_at(k, n, x.dphi), s.pll_freq + x.df, (double)x.I, (double)x.Q, es_all,
                   pp_all);
        s.pll_path = 1;
        s.pll_iters = iters;
        return;
    }
    // Serial loop from the exact start of segment gstar to the block end, by
    // the owner's whole warp: the lanes load the pilot band and the L-R band of
    // the next 32 steps (coalesced, one chunk ahead), all of them evaluate the
    // same recurrence (uniform values, so the loop never waits on a load), and
    // lane i keeps step i's L-R product for one coalesced store per chunk.
    if ((g >> 5) != (owner >> 5)) return;
    const int ol = owner & 31;
    SegState xs{__shfl_sync(0xffffffffu, x.dphi, ol), __shfl_sync(0xffffffffu, x.df, ol),
                __shfl_sync(0xffffffffu, x.I, ol), __shfl_sync(0xffffffffu, x.Q, ol)};
    const int ts = __shfl_sync(0xffffffffu, t0, ol);
    double es_w = __shfl_sync(0xffffffffu, es_all, ol);
    uint64_t qr = k.q0 + (uint64_t)ts * k.qf;
    float pcur = ts + lane < n ? __ldg(pil + ts + lane) : 0.f;
    float bcur = ts + lane < n ? bpf[ts + lane] : 0.f;
    for (int c0 = ts; c0 < n; c0 += 32) {
        const int cn = c0 + 32;
        const float pnext = cn + lane < n ? __ldg(pil + cn + lane) : 0.f;
        const float bnext = cn + lane < n ? bpf[cn + lane] : 0.f;
        const int cnt = min(32, n - c0);  // uniform in the warp
        float mine = 0.f;
#pragma unroll 4
        for (int i = 0; i < cnt; ++i) {
            const float pt = __shfl_sync(0xffffffffu, pcur, i);
            PllEval o;
            pll_step<false>(qr, xs.dphi, xs.df, xs.I, xs.Q, pt, k, o);
            qr += k.qf;
            xs = SegState{o.dphi1, o.df1, o.I1, o.Q1};
            es_w += fabs((double)o.e);
            const float th = pll_two_sin2(qr, xs.dphi);
            if (lane == i) mine = bcur * th;
        }
        if (lane < cnt) lr[c0 + lane] = mine;
        pcur = pnext;
        bcur = bnext;
    }
    if (lane != ol) return;
    pll_finish(s, cp, n, pll_phase_at(k, n, xs.dphi), s.pll_freq + xs.df, (double)xs.I, (double)xs.Q, es_w, pp_all);
    s.pll_path = 2;
    s.pll_iters = iters;
}

// Sum of the block's composite squared for batch-stereo channels (the
// denominator of their lock test), one CTA per channel, fixed reduction order.
__global__ void __launch_bounds__(256)
k_comp_power(const int *__restrict__ list, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
             ChanState *__restrict__ st, const float *__restrict__ wk) {
    __shared__ double red[256];
    const SlotBlock sb = sbt[list[blockIdx.x]];
    const ChanParams &cp = prm[sb.slot];
    if (!(cp.flags & kChBatchStereo)) return;
    const float *m = wk + sb.comp_off;
    double acc = 0.0;
    for (int q = threadIdx.x; q < sb.n_disc; q += 256) acc += (double)m[q] * (double)m[q];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) st[sb.slot].comp_power = red[0];
}

// WFMStereo.Demod's L-R product with a free-running carrier (demod/fm.go:
// 106-112): lr[q] = bpf[q] * float32(2 cos x_{q+1}), x_k = fl(x_{k-1} + inc),
// inc = 2 pi 38000 / rate, the reference's sequential float64 phase evaluated
// exactly from its binade table.
__global__ void __launch_bounds__(256)
k_free_stereo(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
              const BinadeTable *__restrict__ tabs38, float *__restrict__ wk, int W) {
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    const BinadeTable &tab = tabs38[cp.rds_tab];
    const float *bpf = wk + 2 * W + sb.comp_off;
    float *lr = wk + 4 * W + sb.comp_off;
    const int q0 = w.y * 1024;
    for (int q = q0 + threadIdx.x; q < q0 + 1024 && q < sb.n_disc; q += 256)
        lr[q] = bpf[q] * (float)(2.0 * cos(binade_value(tab, (int64_t)q + 1)));
}

// L-R lowpass and L/R matrix when stereo is enabled; otherwise the 15 kHz mono
// fallback filter (its own delay line, advanced only on fallback blocks) duplicated
// to both channels.  WFM (mono) mode always takes the mono filter, one channel.
__global__ void __launch_bounds__(kFirThreads)
k_wfm_out(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
          const ChanState *__restrict__ st, const WfmTaps *__restrict__ taps, const float *__restrict__ wk, int W,
          const float *__restrict__ lr_dl, const float *__restrict__ audio_dl, float *__restrict__ audio) {
    __shared__ float win[padi(kFirOT + kWfmTapsPad) + 8];
    __shared__ float tp[kWfmTapsPad];
    __shared__ float s_out[kFirOT + kFirOT / 32];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const ChanParams &cp = prm[sb.slot];
    const int q0 = w.y * kFirOT;
    if (q0 >= sb.n_disc) return;
    const bool stereo = (cp.mode == 3) && (st[sb.slot].enabled || (cp.flags & kChFreeStereo));
    if (cp.mode == 3 && !stereo && (cp.flags & kChBatchStereo)) {
        // batch decoder not locked: the discriminator output itself on both
        // channels (wfm_batch_stereo.go:43-49)
        const float *m = wk + sb.comp_off;
        float *dst = audio + sb.audio_off;
        for (int q = q0 + threadIdx.x; q < q0 + kFirOT && q < sb.n_disc; q += kFirThreads)
            dst[2 * q] = dst[2 * q + 1] = m[q];
        return;
    }
    const WfmTaps &tb = taps[cp.rds_tab];
    for (int i = threadIdx.x; i < kWfmTapsPad; i += kFirThreads) tp[i] = tb.t[i].x;
    if (stereo) {
        stage_window(win, wk + 4 * W + sb.comp_off, q0, sb.n_disc, lr_dl + cp.wfm_idx * kWfmHist,
                     sb.comp_hist_len);
    } else {
        // The fallback filter's delay line holds composite samples of earlier
        // fallback blocks only; its valid count sits after the 100 samples.
        const float *adl = audio_dl + cp.wfm_idx * kAudioDlStride;
        stage_window(win, wk + sb.comp_off, q0, sb.n_disc, adl, __float_as_int(adl[kWfmHist]));
    }
    __syncthreads();
    const int t = threadIdx.x;
    const int base = 8 * t + kWfmTapsPad;
    float a[8], ring[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) a[r] = 0.f;
#pragma unroll
    for (int j = 1; j < 8; ++j) ring[j] = win[padi(base + j)];
    for (int kb = 0; kb < kWfmTapsPad; kb += 8) {
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
            const int k = kb + kk;
            ring[(8 - kk) & 7] = win[padi(base - k)];
            const float h = tp[k];
#pragma unroll
            for (int r = 0; r < 8; ++r) a[r] = fmaf(h, ring[(r - kk + 8) & 7], a[r]);
        }
    }
    // the tile's filter outputs through shared memory (index i + i/32: the
    // stores of a register row and the reads of consecutive outputs are both
    // conflict-free), then coalesced reads of L+R and stores of (L, R) pairs
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = 8 * t + r;
        s_out[i + (i >> 5)] = a[r];
    }
    __syncthreads();
    float *dst = audio + sb.audio_off;
    const int nq = min(kFirOT, sb.n_disc - q0);
    if (cp.mode == 2) {
        for (int i = t; i < nq; i += kFirThreads) dst[q0 + i] = s_out[i + (i >> 5)];
    } else if (stereo) {
        const float *lpr = wk + 1 * W + sb.comp_off;
        float2 *d2 = reinterpret_cast<float2 *>(dst);
        for (int i = t; i < nq; i += kFirThreads) {
            const float v = s_out[i + (i >> 5)], l = lpr[q0 + i];
            d2[q0 + i] = make_float2(0.5f * (l + v), 0.5f * (l - v));
        }
    } else {
        float2 *d2 = reinterpret_cast<float2 *>(dst);
        for (int i = t; i < nq; i += kFirThreads) {
            const float v = s_out[i + (i >> 5)];
            d2[q0 + i] = make_float2(v, v);
        }
    }
}

// RDS baseband (fm.go:143-163 / 234-271) over the continuous discriminator
// stream: cplx[g] = disc[g] * exp(j x_{g+1}) with x the exact sequential
// float64 FreqShift phase, a 101-tap lowpass accumulated in float64 in the
// reference's order (separate multiply and add, as Go's amd64 code does), and
// every Dr-th stream sample kept.
constexpr int kRdsOT = 128;     // RDS outputs per CTA (one per thread)
constexpr int kRdsThreads = 128;

// Index of the binade entry covering stream index k.
__device__ __forceinline__ int binade_find(const BinadeTable &t, int64_t k) {
    int lo = 0, hi = t.count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (t.e[mid].k_start <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// RDS baseband (demod/fm.go:143-163, 234-271): the composite shifted by the
// reference's float64 FreqShift phase (exact values from the binade table),
// 101-tap float64 low-pass evaluated at the kept outputs only.  Staging: each
// thread takes a contiguous run of composite samples, evaluates sin/cos of
// the exact phase once at the run start (and at any binade start inside it)
// and advances by the exact in-binade step with a float64 rotation
// (relative error < 1e-14 over a run, far below the float32 the shifted
// samples are stored in).
__global__ void __launch_bounds__(kRdsThreads)
k_rds(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
      const ChanState *__restrict__ st, const WfmTaps *__restrict__ taps, const BinadeTable *__restrict__ tabs,
      const float *__restrict__ wk, const float2 *__restrict__ rds_dl, float2 *__restrict__ rds_out) {
    extern __shared__ float2 cpl[];
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const int r0 = w.y * kRdsOT;
    if (r0 >= sb.n_rds) return;
    const ChanParams &cp = prm[sb.slot];
    const int dr = cp.rds_dr;
    const int r1 = min(r0 + kRdsOT, sb.n_rds);
    const int qlo = sb.rds_first + r0 * dr - (kWfmTaps - 1);
    const int qhi = sb.rds_first + (r1 - 1) * dr;
    const int span = qhi - qlo + 1;
    const ChanState &s = st[sb.slot];
    const int64_t c0 = s.rds_count;
    const BinadeTable &tab = tabs[cp.rds_tab];
    const float *comp = wk + sb.comp_off;
    const float2 *dl = rds_dl + cp.wfm_idx * kWfmHist;
    const int per = (span + kRdsThreads - 1) / kRdsThreads;
    const int i0 = min(span, (int)threadIdx.x * per), i1 = min(span, i0 + per);
    int ent = -1;
    int64_t next_k = 0;
    double cs = 0.0, sn = 0.0, wc = 1.0, ws = 0.0;
    for (int i = i0; i < i1; ++i) {
        const int q = qlo + i;
        float2 v = make_float2(0.f, 0.f);
        if (q >= 0) {
            const int64_t k = c0 + q + 1;  // phase index: incremented before use (freqshift.go:13-15)
            if (ent < 0 || k >= next_k) {
                ent = binade_find(tab, k);
                const BinadeEntry &be = tab.e[ent];
                next_k = ent + 1 < tab.count ? tab.e[ent + 1].k_start : INT64_MAX;
                sincos(be.x_start + (double)(k - be.k_start) * be.q, &sn, &cs);
                sincos(be.q, &ws, &wc);
            } else {
                const double c1 = cs * wc - sn * ws;
                sn = sn * wc + cs * ws;
                cs = c1;
            }
            const double b = (double)comp[q];
            v = make_float2((float)(b * cs), (float)(b * sn));
        } else if (q >= -s.rds_hist_len) {
            v = dl[kWfmHist + q];
        }
        cpl[i + (i >> 4)] = v;
    }
    __syncthreads();
    // outputs dr samples apart read through one pad slot every 16: the lanes'
    // addresses fall in distinct banks
    const WfmTaps &tb = taps[cp.rds_tab];
    for (int r = r0 + threadIdx.x; r < r1; r += kRdsThreads) {
        const int qr = sb.rds_first + r * dr;
        const int li = qr - qlo;
        double ar = 0.0, ai = 0.0;
        for (int k = 0; k < kWfmTaps; ++k) {
            const int c = li - k;
            const float2 v = cpl[c + (c >> 4)];
            ar = __dadd_rn(ar, __dmul_rn((double)v.x, tb.rds[k]));
            ai = __dadd_rn(ai, __dmul_rn((double)v.y, tb.rds[k]));
        }
        rds_out[sb.rds_off + r] = make_float2((float)ar, (float)ai);
    }
}

// ===========================================================================
// Per-slot state carry, one CTA per slot, after every other kernel.
// ===========================================================================
__device__ void shift_delay_line(float *dl, const float *__restrict__ src, int n) {
    // dl: 100 floats oldest-first; append src[0..n) and keep the last 100.
    __shared__ float tmp[kWfmHist];
    for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) {
        int g = n + i - kWfmHist;  // index into (dl ++ src) shifted so dl occupies [-100, 0)
        tmp[i] = g >= 0 ? src[g] : dl[kWfmHist + g];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) dl[i] = tmp[i];
    __syncthreads();
}

// Front half: everything the next block's extraction, demod, stereo FIR bank
// and RDS read (extraction history and NCO phase, discriminator bridge,
// composite delay line, RDS stream history).  Runs right after those stages,
// so the next block's front half can overlap this block's PLL.
__global__ void __launch_bounds__(128)
k_post_front(const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm, ChanState *__restrict__ st,
             const float2 *__restrict__ ext, const float *__restrict__ wk, float *__restrict__ comp_dl,
             float2 *__restrict__ rds_dl, const BinadeTable *__restrict__ tabs, float2 *__restrict__ d1hist,
             DevResult *__restrict__ res) {
    const SlotBlock sb = sbt[blockIdx.x];
    const ChanParams &cp = prm[sb.slot];
    ChanState &s = st[sb.slot];
    if (cp.d1 > 1 && sb.n_out > 0) {
        // pre-demod decimator history: the last 100 extraction outputs
        __shared__ float2 dtmp[kWfmHist];
        float2 *dh = d1hist + (int64_t)sb.slot * kWfmHist;
        for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) {
            const int g = sb.n_out + i - kWfmHist;
            dtmp[i] = g >= 0 ? ext[sb.ext_off + g] : dh[kWfmHist + g];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) dh[i] = dtmp[i];
        __syncthreads();
    }
    if (cp.wfm_idx >= 0 && sb.n_disc > 0) {
        const float *comp = wk + sb.comp_off;
        // RDS shifted history: the last 100 values of cplx over the stream
        if (cp.flags & 2) {
            __shared__ float2 rtmp[kWfmHist];
            const BinadeTable &tab = tabs[cp.rds_tab];
            float2 *dl = rds_dl + cp.wfm_idx * kWfmHist;
            const int64_t c0 = s.rds_count;
            for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) {
                int q = sb.n_disc + i - kWfmHist;
                float2 v = make_float2(0.f, 0.f);
                if (q >= 0) {
                    double ph = binade_value(tab, c0 + q + 1);
                    double sn, cs;
                    sincos(ph, &sn, &cs);
                    double b = (double)comp[q];
                    v = make_float2((float)(b * cs), (float)(b * sn));
                } else {
                    v = dl[kWfmHist + q];
                }
                rtmp[i] = v;
            }
            __syncthreads();
            for (int i = threadIdx.x; i < kWfmHist; i += blockDim.x) dl[i] = rtmp[i];
            __syncthreads();
        }
        shift_delay_line(comp_dl + cp.wfm_idx * kWfmHist, comp, sb.n_disc);
    }
    if (threadIdx.x == 0) {
        if (sb.n_dem > 0) {
            s.last_iq = ext[sb.dem_off + sb.n_dem - 1];
            s.has_last = 1;
        }
        if (cp.wfm_idx >= 0 && sb.n_disc > 0) {
            s.rds_count += sb.n_disc;
            s.rds_hist_len = (int)min((int64_t)kWfmHist, s.rds_count);
        }
    }
}

// Extraction state of a block, carried as soon as the block's extraction
// kernels are done (the next block's extraction waits only for this): the
// last min(T-1, H+n) samples of (history ++ shifted block) into the other
// history buffer, and the NCO phase advanced by the block.
__global__ void __launch_bounds__(128)
k_post_extract(const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm, ChanState *__restrict__ st,
               const float2 *__restrict__ x, int n, float2 *__restrict__ hist_arena, DevResult *__restrict__ res) {
    const SlotBlock sb = sbt[blockIdx.x];
    const ChanParams &cp = prm[sb.slot];
    ChanState &s = st[sb.slot];
    const uint64_t u0 = s.nco_q;
    const int keep = cp.ntaps - 1;
    const int H = sb.hist_len;
    const int newH = min(keep, H + n);
    const float2 *hold = hist_arena + cp.hist_off + sb.hist_sel * cp.hcap;
    float2 *hnew = hist_arena + cp.hist_off + (1 - sb.hist_sel) * cp.hcap;
    for (int q = threadIdx.x; q < newH; q += blockDim.x) {
        int g = H + n - newH + q;
        hnew[q] = g < H ? hold[g] : cmulf(__ldg(x + (g - H)), q64_phasor(u0 + (uint64_t)(g - H) * cp.inc_q));
    }
    __syncthreads();  // every thread has read the block-start phase
    if (threadIdx.x == 0) {
        s.nco_q = u0 + (uint64_t)n * cp.inc_q;
        res[sb.res_idx].nco_phase = q64_to_rad(s.nco_q);
    }
}

// Back half: the L-R and mono-fallback delay lines and the block's lock
// flags, margins and PLL solver info, after the PLL and the stereo output.
__global__ void __launch_bounds__(128)
k_post_back(const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm, ChanState *__restrict__ st,
            const float *__restrict__ wk, int W, float *__restrict__ lr_dl, float *__restrict__ audio_dl,
            DevResult *__restrict__ res) {
    const SlotBlock sb = sbt[blockIdx.x];
    const ChanParams &cp = prm[sb.slot];
    ChanState &s = st[sb.slot];
    if (cp.wfm_idx >= 0 && sb.n_disc > 0) {
        const float *comp = wk + sb.comp_off;
        const bool fallback = (cp.mode == 2) || !s.enabled;
        if (fallback) {
            float *adl = audio_dl + cp.wfm_idx * kAudioDlStride;
            int valid = __float_as_int(adl[kWfmHist]);
            shift_delay_line(adl, comp, sb.n_disc);
            if (threadIdx.x == 0) adl[kWfmHist] = __int_as_float(min(kWfmHist, valid + sb.n_disc));
            __syncthreads();
        }
        if (cp.mode == 3) shift_delay_line(lr_dl + cp.wfm_idx * kWfmHist, wk + 4 * W + sb.comp_off, sb.n_disc);
    }
    if (threadIdx.x == 0) {
        DevResult &o = res[sb.res_idx];
        o.flags = (cp.mode == 3 && sb.n_disc > 0) ? ((s.locked ? 1 : 0) | (s.enabled ? 2 : 0))
                                                  : (s.enabled ? 2 : 0);
        o.coherence = s.coherence;
        o.pilot_hz = s.pilot_hz;
        o.err_avg = s.last_err_avg;
        o.status = (cp.mode == 3 && sb.n_disc > 0) ? s.pll_path : 0;
        o.pll_iters = s.pll_iters;
    }
}

// ===========================================================================
// 48 kHz audio back end (recorder/streamer.go:1408-1470, 569-575)
// ===========================================================================
// Resampling: output o of the block sits at the resampler's phase position
// t0 + o*M: it is produced after consuming c = floor((t0+o*M)/L) inputs, at
// arm (t0+o*M) - c*L, over the last K consumed samples (earlier blocks'
// samples from the carried delay line) -- the closed form of
// Resampler.Process (dsp/resample.go:105-153); the host mirrors the phase
// counter, including that method's exits, so every output is independent and
// k_audio48_rs computes one per thread over the whole grid.  The float64 dot
// products keep the reference's separate multiply and add.
// k_audio48_out, one CTA per channel: de-emphasis y = a*y + (1-a)*x (float64),
// a first-order recurrence -- each thread takes a contiguous run of outputs,
// the runs' affine maps are scanned across the CTA and each run is replayed
// from its start -- then the WFM gain 0.35 and s16le: int16(clip(s * 32767)),
// truncating; it also carries the delay lines and the de-emphasis state.
constexpr int kAudThreads = 256;
constexpr int kAudOT = 256;  // resampled frames per CTA in k_audio48_rs

constexpr int kAudWin = 2048;     // staged input frames per channel and CTA (256 outputs at M/L <= 7.8)
constexpr int kAudBank = 4096;    // staged bank coefficients (doubles)

__global__ void __launch_bounds__(kAudThreads)
k_audio48_rs(const int2 *__restrict__ work, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
             const RsBank *__restrict__ banks, const AudState *__restrict__ aud, const float *__restrict__ audio,
             float *__restrict__ rs_out) {
    extern __shared__ double s_aud[];  // bank (L*K doubles) | inputs 2 x kAudWin floats
    const int2 w = work[blockIdx.x];
    const SlotBlock sb = sbt[w.x];
    const int oa = w.y * kAudOT, ob = min(sb.rs_nout, oa + kAudOT);  // this CTA's outputs
    if (oa >= ob) return;
    const ChanParams &cp = prm[sb.slot];
    const AudState &as = aud[sb.slot];
    const RsBank &bk = banks[cp.rs_bank];
    const int C = cp.aud_ch, L = bk.L, M = bk.M, K = bk.K;
    const float *in = audio + sb.audio_off;
    if (L == M) {
        for (int o = oa + (int)threadIdx.x; o < ob; o += kAudThreads)
            for (int c = 0; c < C; ++c) rs_out[sb.pcm_off + o * C + c] = in[o * C + c];
        return;
    }
    // consumed-input window of the tile: [lo, hi]
    const int64_t lo = ((int64_t)sb.rs_t0 + (int64_t)oa * M) / L - K;
    const int64_t hi = ((int64_t)sb.rs_t0 + (int64_t)(ob - 1) * M) / L - 1;
    const int win = (int)(hi - lo + 1);
    const bool staged = win <= kAudWin && L * K <= kAudBank;
    double *s_bank = s_aud;
    float *s_in = reinterpret_cast<float *>(s_aud + kAudBank);
    if (staged) {
        // eight loads in flight per thread: the staging, not the 33-tap dot
        // products, sets this kernel's time
        constexpr int U = 8;
        const int nb = L * K;
        for (int i0 = threadIdx.x; i0 < nb; i0 += U * kAudThreads) {
            double v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * kAudThreads;
                v[u] = i < nb ? bk.arm[i] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * kAudThreads;
                if (i < nb) s_bank[i] = v[u];
            }
        }
        for (int c = 0; c < C; ++c) {
            for (int i0 = threadIdx.x; i0 < win; i0 += U * kAudThreads) {
                float v[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * kAudThreads;
                    const int64_t g = lo + i;
                    v[u] = i < win ? (g >= 0 ? in[g * C + c] : as.dl[c][-1 - g]) : 0.f;
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int i = i0 + u * kAudThreads;
                    if (i < win) s_in[c * kAudWin + i] = v[u];
                }
            }
        }
        __syncthreads();
    }
    for (int o = oa + (int)threadIdx.x; o < ob; o += kAudThreads) {
        const int64_t T = (int64_t)sb.rs_t0 + (int64_t)o * M;
        const int64_t cc = T / L;  // T >= 0
        const int ph = (int)(T - cc * L);
        double acc0 = 0.0, acc1 = 0.0;
        if (staged) {
            const double *arm = s_bank + ph * K;
            const float *x0 = s_in + (cc - 1 - lo), *x1 = s_in + kAudWin + (cc - 1 - lo);
            for (int k = 0; k < K; ++k) {
                const double h = arm[k];
                acc0 = __dadd_rn(acc0, __dmul_rn((double)x0[-k], h));
                if (C == 2) acc1 = __dadd_rn(acc1, __dmul_rn((double)x1[-k], h));
            }
        } else {
            const double *arm = bk.arm + ph * K;
            for (int k = 0; k < K; ++k) {
                const int64_t i = cc - 1 - k;
                const double h = arm[k];
                const float v0 = i >= 0 ? in[i * C] : as.dl[0][-1 - i];
                acc0 = __dadd_rn(acc0, __dmul_rn((double)v0, h));
                if (C == 2) {
                    const float v1 = i >= 0 ? in[i * 2 + 1] : as.dl[1][-1 - i];
                    acc1 = __dadd_rn(acc1, __dmul_rn((double)v1, h));
                }
            }
        }
        float *dst = rs_out + sb.pcm_off + o * C;
        dst[0] = (float)acc0;
        if (C == 2) dst[1] = (float)acc1;
    }
}

constexpr int kAudOutThreads = 1024;  // one CTA per channel: short serial runs
constexpr int kAudOutStage = 16384;   // resampled samples of a channel staged in shared memory (64 KB)

__global__ void __launch_bounds__(kAudOutThreads)
k_audio48_out(const int *__restrict__ list, const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
              const RsBank *__restrict__ banks, AudState *__restrict__ aud, const float *__restrict__ audio,
              const float *__restrict__ rs_out, int16_t *__restrict__ pcm) {
    constexpr int kWarps = kAudOutThreads / 32;
    __shared__ double s_wa[kWarps], s_wb[2][kWarps];  // warp totals, then exclusive warp prefixes
    extern __shared__ float s_rs[];  // the channel's resampled block (when it fits), then its output samples
    const SlotBlock sb = sbt[list[blockIdx.x]];
    const ChanParams &cp = prm[sb.slot];
    AudState &as = aud[sb.slot];
    const int C = cp.aud_ch;
    const int n = sb.rs_frames, nout = sb.rs_nout;
    if (n <= 0) return;
    const RsBank &bk = banks[cp.rs_bank];
    // each thread takes a run of consecutive frames: the block is staged with
    // coalesced loads and the PCM written back coalesced
    const bool staged = nout * C <= kAudOutStage;
    if (staged) {
        const float *src = rs_out + sb.pcm_off;
        for (int i = threadIdx.x; i < nout * C; i += kAudOutThreads) s_rs[i] = src[i];
        __syncthreads();
    }
    const float *r = staged ? s_rs : rs_out + sb.pcm_off;
    const int per = (nout + kAudOutThreads - 1) / kAudOutThreads;
    const int o0 = min(nout, (int)threadIdx.x * per), o1 = min(nout, o0 + per);
    const bool wfm = cp.mode == 2 || cp.mode == 3;
    const double a = cp.deemph_a;
    const bool de = wfm && a > 0.0;
    double y0 = as.y[0], y1 = as.y[1];
    if (de) {
        // this run's map y_end = A*y_start + B, per channel
        double A = 1.0, B0 = 0.0, B1 = 0.0;
        for (int o = o0; o < o1; ++o) {
            A = __dmul_rn(A, a);
            B0 = __dadd_rn(__dmul_rn(a, B0), __dmul_rn(1.0 - a, (double)r[o * C]));
            if (C == 2) B1 = __dadd_rn(__dmul_rn(a, B1), __dmul_rn(1.0 - a, (double)r[o * 2 + 1]));
        }
        // inclusive scan of the maps across the warp (a later run applied
        // after an earlier one), then across the warps' totals
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double pa = __shfl_up_sync(0xffffffffu, A, d);
            const double pb0 = __shfl_up_sync(0xffffffffu, B0, d);
            const double pb1 = __shfl_up_sync(0xffffffffu, B1, d);
            if (lane >= d) {
                B0 = A * pb0 + B0;
                B1 = A * pb1 + B1;
                A = A * pa;
            }
        }
        if (lane == 31) {
            s_wa[warp] = A;
            s_wb[0][warp] = B0;
            s_wb[1][warp] = B1;
        }
        __syncthreads();
        if (warp == 0) {
            double wa = lane < kWarps ? s_wa[lane] : 1.0;
            double wb0 = lane < kWarps ? s_wb[0][lane] : 0.0, wb1 = lane < kWarps ? s_wb[1][lane] : 0.0;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const double pa = __shfl_up_sync(0xffffffffu, wa, d);
                const double pb0 = __shfl_up_sync(0xffffffffu, wb0, d);
                const double pb1 = __shfl_up_sync(0xffffffffu, wb1, d);
                if (lane >= d) {
                    wb0 = wa * pb0 + wb0;
                    wb1 = wa * pb1 + wb1;
                    wa = wa * pa;
                }
            }
            // exclusive: the warps before this one
            const double ea = __shfl_up_sync(0xffffffffu, wa, 1);
            const double eb0 = __shfl_up_sync(0xffffffffu, wb0, 1);
            const double eb1 = __shfl_up_sync(0xffffffffu, wb1, 1);
            if (lane < kWarps) {
                s_wa[lane] = lane ? ea : 1.0;
                s_wb[0][lane] = lane ? eb0 : 0.0;
                s_wb[1][lane] = lane ? eb1 : 0.0;
            }
        }
        __syncthreads();
        // this run's start: the warps before it, then the lanes before it
        const double la = __shfl_up_sync(0xffffffffu, A, 1);
        const double lb0 = __shfl_up_sync(0xffffffffu, B0, 1);
        const double lb1 = __shfl_up_sync(0xffffffffu, B1, 1);
        const double ws0 = s_wa[warp] * as.y[0] + s_wb[0][warp];
        const double ws1 = s_wa[warp] * as.y[1] + s_wb[1][warp];
        y0 = lane ? la * ws0 + lb0 : ws0;
        y1 = lane ? la * ws1 + lb1 : ws1;
    }
    for (int o = o0; o < o1; ++o) {
        for (int c = 0; c < C; ++c) {
            float s = r[o * C + c];
            if (de) {
                double &y = c == 0 ? y0 : y1;
                y = __dadd_rn(__dmul_rn(a, y), __dmul_rn(1.0 - a, (double)s));
                s = (float)y;
            }
            if (wfm) s = s * 0.35f;
            if (staged) {
                s_rs[o * C + c] = s;  // this thread's own cell, already read
            } else if (cp.flags & kChPcmF32) {
                reinterpret_cast<float *>(pcm + sb.pcm_off)[o * C + c] = s;
            } else {
                float v = s * 32767.0f;
                v = fminf(fmaxf(v, -32768.0f), 32767.0f);
                pcm[sb.pcm_off + o * C + c] = (int16_t)v;
            }
        }
    }
    if (staged) {
        __syncthreads();
        if (cp.flags & kChPcmF32) {
            float *dst = reinterpret_cast<float *>(pcm + sb.pcm_off);
            for (int i = threadIdx.x; i < nout * C; i += kAudOutThreads) dst[i] = s_rs[i];
        } else {
            for (int i = threadIdx.x; i < nout * C; i += kAudOutThreads) {
                float v = s_rs[i] * 32767.0f;
                v = fminf(fmaxf(v, -32768.0f), 32767.0f);
                pcm[sb.pcm_off + i] = (int16_t)v;
            }
        }
    }
    __syncthreads();  // every read of the old state is done
    // carried state: the last K consumed samples, newest first; the last y
    const int c = threadIdx.x / kRsTaps, k = threadIdx.x % kRsTaps;
    const bool mine = bk.L != bk.M && threadIdx.x < 2 * kRsTaps && c < C;
    float v = 0.f;
    if (mine) {
        const int i = n - 1 - k;
        v = i >= 0 ? audio[sb.audio_off + i * C + c] : as.dl[c][-1 - i];
    }
    __syncthreads();  // the shifted entries are read before any is overwritten
    if (mine) as.dl[c][k] = v;
    if (de && nout > 0 && o1 == nout && o0 < o1) {
        as.y[0] = y0;
        as.y[1] = y1;
    }
}

// ===========================================================================
// launch helpers (host)
// ===========================================================================
template <int L>
static cudaError_t launch_dense_L(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                  const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                  const float2 *hist, const float *taps, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_dense<L>, 220 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_dense<L><<<grid, kDenseThreads, smem, sm>>>(work, sbt, prm, st, x, n, hist, taps, ext);
    return cudaGetLastError();
}

cudaError_t launch_extract_dense_any(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                     const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                     const float2 *hist, const float *taps, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_dense_any, 220 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_dense_any<<<grid, kDenseThreads, smem, sm>>>(work, sbt, prm, st, x, n, hist, taps, ext);
    return cudaGetLastError();
}

cudaError_t launch_extract_dense(int L, int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                 const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                 const float2 *hist, const float *taps, float2 *ext) {
    switch (L) {
#define GPUD_CASE(LL) \
    case LL: return launch_dense_L<LL>(grid, smem, sm, work, sbt, prm, st, x, n, hist, taps, ext);
        GPUD_CASE(2) GPUD_CASE(3) GPUD_CASE(4) GPUD_CASE(5) GPUD_CASE(6) GPUD_CASE(7) GPUD_CASE(8)
        GPUD_CASE(9) GPUD_CASE(10) GPUD_CASE(11) GPUD_CASE(12) GPUD_CASE(13) GPUD_CASE(14)
        GPUD_CASE(15) GPUD_CASE(16)
#undef GPUD_CASE
    default: return cudaErrorInvalidValue;
    }
}

template <int L, int NG>
static cudaError_t launch_dense_pipe_LG(int ntiles, int grid, int pmax, cudaStream_t sm, const int2 *work,
                                        const SlotBlock *sbt, const ChanParams *prm, const ChanState *st,
                                        const float2 *x, int n, const float2 *hist, const float *taps, float2 *ext,
                                        unsigned *fault) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_dense_pipe<L, NG>, 220 * 1024);
    if (e != cudaSuccess) return e;
    const int smem = pipe_layout(pmax, L, NG).bytes;
    k_extract_dense_pipe<L, NG><<<grid, kPipeThreads, smem, sm>>>(work, ntiles, pmax, sbt, prm, st, x, n, hist,
                                                                  taps, ext, fault);
    return cudaGetLastError();
}

// Consumer groups of the pipelined dense form for a class whose channels have
// at most P phases (two when both groups' Z fit beside the raw span), or 0
// when it does not fit in cap bytes or needs more rotation-table rounds than
// the producer warp fills.
int dense_pipe_groups_host(int P, int L, int cap) {
    const int total = P * (kDenseOT + L - 1);
    if (total <= kPipeMaxRounds * 32 * (kPipeCW / 2) && pipe_layout(P, L, 2).bytes <= cap) return 2;
    if (total <= kPipeMaxRounds * 32 * kPipeCW && pipe_layout(P, L, 1).bytes <= cap) return 1;
    return 0;
}

cudaError_t launch_extract_dense_pipe(int L, int ng, int ntiles, int grid, int pmax, cudaStream_t sm,
                                      const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                                      const ChanState *st, const float2 *x, int n, const float2 *hist,
                                      const float *taps, float2 *ext, unsigned *fault) {
    if (((uintptr_t)x & 15) != 0 || (ng != 1 && ng != 2)) return cudaErrorInvalidValue;
    switch (L * 4 + ng) {
#define GPUD_CASE(LL)                                                                                              \
    case LL * 4 + 1:                                                                                               \
        return launch_dense_pipe_LG<LL, 1>(ntiles, grid, pmax, sm, work, sbt, prm, st, x, n, hist, taps, ext,     \
                                           fault);                                                                 \
    case LL * 4 + 2:                                                                                               \
        return launch_dense_pipe_LG<LL, 2>(ntiles, grid, pmax, sm, work, sbt, prm, st, x, n, hist, taps, ext,     \
                                           fault);
        GPUD_CASE(2) GPUD_CASE(3) GPUD_CASE(4) GPUD_CASE(5) GPUD_CASE(6) GPUD_CASE(7) GPUD_CASE(8)
        GPUD_CASE(9) GPUD_CASE(10) GPUD_CASE(11) GPUD_CASE(12) GPUD_CASE(13) GPUD_CASE(14)
        GPUD_CASE(15) GPUD_CASE(16)
#undef GPUD_CASE
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_extract_wide(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                const float2 *hist, const float *taps, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_wide, 64 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_wide<<<grid, 256, smem, sm>>>(work, sbt, prm, st, x, n, hist, taps, ext);
    return cudaGetLastError();
}

cudaError_t launch_extract_group(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                                 const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                                 const float2 *hist, const float *taps, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_group, 220 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_group<<<grid, kDenseThreads, smem, sm>>>(work, sbt, prm, st, x, n, hist, taps, ext);
    return cudaGetLastError();
}

cudaError_t launch_extract_mod(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                               const ChanParams *prm, const ChanState *st, const float2 *x, int n,
                               const float2 *hist, const float *taps, float2 *ext) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_mod, 220 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_mod<<<grid, kDenseThreads, smem, sm>>>(work, sbt, prm, st, x, n, hist, taps, ext);
    return cudaGetLastError();
}

cudaError_t launch_comp_power(int count, cudaStream_t sm, const int *list, const SlotBlock *sbt,
                              const ChanParams *prm, ChanState *st, const float *wk) {
    k_comp_power<<<count, 256, 0, sm>>>(list, sbt, prm, st, wk);
    return cudaGetLastError();
}

cudaError_t launch_free_stereo(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                               const ChanParams *prm, const BinadeTable *tabs38, float *wk, int W) {
    k_free_stereo<<<grid, 256, 0, sm>>>(work, sbt, prm, tabs38, wk, W);
    return cudaGetLastError();
}

// Second decimation of the one-shot segment demod (recorder/cpu_audio.go:
// 35-72): ApplyFIRReal with the 63-tap anti-alias filter per audio channel
// (float64 taps and sum, separate multiply and add) at frames i*d2.
__global__ void __launch_bounds__(256)
k_seg_aa(const float *__restrict__ in, int C, const double *__restrict__ taps, int nt, int d2, int of,
         float *__restrict__ out) {
    const int idx = blockIdx.x * blockDim.x + (int)threadIdx.x;
    if (idx >= of * C) return;
    const int i = idx / C, c = idx - i * C;
    const int64_t src = (int64_t)i * d2;
    double acc = 0.0;
    for (int k = 0; k < nt; ++k) {
        const int64_t j = src - k;
        if (j < 0) break;
        acc = __dadd_rn(acc, __dmul_rn((double)in[j * C + c], taps[k]));
    }
    out[idx] = (float)acc;
}

cudaError_t launch_seg_aa(cudaStream_t sm, const float *in, int C, const double *taps, int nt, int d2, int of,
                          float *out) {
    const int total = of * C;
    if (total > 0) k_seg_aa<<<(total + 255) / 256, 256, 0, sm>>>(in, C, taps, nt, d2, of, out);
    return cudaGetLastError();
}

cudaError_t launch_demod(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                         const ChanState *st, const float2 *ext, float *comp, float *audio) {
    k_demod<<<grid, 256, 0, sm>>>(work, sbt, prm, st, ext, comp, audio);
    return cudaGetLastError();
}

cudaError_t launch_am(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const float2 *ext,
                      float *audio) {
    k_am<<<grid, 256, 0, sm>>>(work, sbt, ext, audio);
    return cudaGetLastError();
}

cudaError_t launch_wfm_fir(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const WfmTaps *taps, float *wk, int W, const float *comp_dl) {
    k_wfm_fir<<<grid, kFirThreads, 0, sm>>>(work, sbt, prm, taps, wk, W, comp_dl);
    return cudaGetLastError();
}

cudaError_t launch_pll(int count, cudaStream_t sm, const int *list, const SlotBlock *sbt, const ChanParams *prm,
                       ChanState *st, float *wk, int W) {
    k_pll<<<count, 64, 0, sm>>>(list, count, sbt, prm, st, wk, W);
    return cudaGetLastError();
}

cudaError_t launch_pll_newton(int count, int cluster, cudaStream_t sm, const int *list, const SlotBlock *sbt,
                              const ChanParams *prm, ChanState *st, float *wk, int W, int max_iters) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * cluster), 1, 1);
    cfg.blockDim = dim3(kNewtonThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = sm;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_pll_newton, list, count, sbt, prm, st, wk, W, max_iters);
}

int pll_newton_threads() { return kNewtonThreads; }

cudaError_t launch_wfm_out(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                           const ChanState *st, const WfmTaps *taps, const float *wk, int W, const float *lr_dl,
                           const float *audio_dl, float *audio) {
    k_wfm_out<<<grid, kFirThreads, 0, sm>>>(work, sbt, prm, st, taps, wk, W, lr_dl, audio_dl, audio);
    return cudaGetLastError();
}

cudaError_t launch_rds(int grid, int smem, cudaStream_t sm, const int2 *work, const SlotBlock *sbt,
                       const ChanParams *prm, const ChanState *st, const WfmTaps *taps, const BinadeTable *tabs,
                       const float *wk, const float2 *rds_dl, float2 *rds_out) {
    k_rds<<<grid, kRdsThreads, smem, sm>>>(work, sbt, prm, st, taps, tabs, wk, rds_dl, rds_out);
    return cudaGetLastError();
}

cudaError_t launch_decim2(int grid, cudaStream_t sm, const int2 *work, const SlotBlock *sbt, const ChanParams *prm,
                          const double *d1taps, const float2 *d1hist, float2 *ext) {
    k_decim2<<<grid, kDecOT, 0, sm>>>(work, sbt, prm, d1taps, d1hist, ext);
    return cudaGetLastError();
}

int decim2_tile() { return kDecOT; }

cudaError_t launch_post_front(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                              const float2 *ext, const float *wk, float *comp_dl, float2 *rds_dl,
                              const BinadeTable *tabs, float2 *d1hist, DevResult *res) {
    k_post_front<<<grid, 128, 0, sm>>>(sbt, prm, st, ext, wk, comp_dl, rds_dl, tabs, d1hist, res);
    return cudaGetLastError();
}

cudaError_t launch_audio48(int grid_rs, int count, cudaStream_t sm, const int2 *work, const int *list,
                           const SlotBlock *sbt, const ChanParams *prm, const RsBank *banks, AudState *aud,
                           const float *audio, float *rs_buf, int16_t *pcm) {
    const int smem = kAudBank * 8 + 2 * kAudWin * 4;
    static std::atomic<uint64_t> optin{0};  // 64 KiB of dynamic shared memory needs the opt-in
    cudaError_t e = smem_optin_once(optin, (const void *)k_audio48_rs, smem);
    if (e != cudaSuccess) return e;
    if (grid_rs > 0) k_audio48_rs<<<grid_rs, kAudThreads, smem, sm>>>(work, sbt, prm, banks, aud, audio, rs_buf);
    static std::atomic<uint64_t> optin_out{0};
    e = smem_optin_once(optin_out, (const void *)k_audio48_out, kAudOutStage * 4);
    if (e != cudaSuccess) return e;
    k_audio48_out<<<count, kAudOutThreads, kAudOutStage * 4, sm>>>(list, sbt, prm, banks, aud, audio, rs_buf, pcm);
    return cudaGetLastError();
}

int audio48_tile() { return kAudOT; }

cudaError_t launch_post_extract(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                                const float2 *x, int n, float2 *hist, DevResult *res) {
    k_post_extract<<<grid, 128, 0, sm>>>(sbt, prm, st, x, n, hist, res);
    return cudaGetLastError();
}

cudaError_t launch_post_back(int grid, cudaStream_t sm, const SlotBlock *sbt, const ChanParams *prm, ChanState *st,
                             const float *wk, int W, float *lr_dl, float *audio_dl, DevResult *res) {
    k_post_back<<<grid, 128, 0, sm>>>(sbt, prm, st, wk, W, lr_dl, audio_dl, res);
    return cudaGetLastError();
}

int rds_smem_bytes(int dr) {
    const int span = kRdsOT * dr + kWfmTaps + 8;
    return (span + span / 16 + 1) * 8;
}
int rds_tile() { return kRdsOT; }

}  // namespace gpud

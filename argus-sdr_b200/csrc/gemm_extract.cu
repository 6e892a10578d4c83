// gemm_extract.cu -- extraction of channel groups on the tcgen05 tensor cores.
//
// Channels that share the decimation D, the tap count T and the phase count
// before the block (pc) take their outputs on the same input grid
// n_j = (D - pc - 1) + j*D.  With the NCO rotation moved from the samples to
// the taps (the modulated-taps identity of the reference's NCO-then-FIR chain,
// streaming_host_core.go:5-64):
//
//     y_c(j) = exp(j phi_c(n_j)) * sum_k g_c[k] x(n_j - k),   g_c[k] = h_c[k] exp(-j k inc_c),
//
// every channel of the group filters the SAME unrotated block x, so a tile of
// 128 outputs for all C channels is one complex GEMM.  In polyphase form
// (k = u*D + D-1-p') the input operand of arm u is the block cut into rows of
// D samples, X2[m][p'] = x(-pc + m*D + p'), shifted by u rows:
//
//     Y[j][c] = sum_u sum_p' X2[j-u][p'] * g_c[u*D + D-1-p'].
//
// As a real GEMM, K interleaves (re, im) of each sample, N = 2C columns
// (y_r, y_i of each channel), and the taps matrix holds the 2x2 blocks
// [[gr, gi], [-gi, gr]].  The block rows are staged once per tile in shared
// memory in a K-major layout whose rows are 16 bytes apart (stride between
// 8-row groups 128 bytes, 16-byte K chunks in planes), so the operand of arm
// u is the same staging with its start address moved by u rows -- no Hankel
// expansion.  tcgen05.mma (kind::tf32, M = 128, N = 2C padded to 16) reads
// both operands from shared memory and accumulates in TMEM; float32 accuracy
// comes from three TF32 passes (x_hi*g_hi + x_hi*g_lo + x_lo*g_hi, x_hi and
// x_lo the TF32 roundings of x and of x - x_hi).  The arms accumulate into
// several TMEM accumulators (the x_hi*g_hi pass of arm u into u % (na-1), the
// small correction passes into the last), so no large accumulator takes more
// than ceil(L/(na-1)) arms of sequential tensor-core roundings -- the arms'
// partial sums are far larger than a narrow channel's output -- and the
// epilogue adds the accumulators in float32 after reading them with
// tcgen05.ld, applies each channel's output rotation exp(j phi_c(n_j)) from
// the exact Q0.64 phase and stores the extracted IQ.  The taps of each arm
// arrive by one bulk copy into a stage freed by tcgen05.commit: one stage per
// CTA when two CTAs then fit on an SM (one CTA's MMAs overlap the other's
// staging and epilogue), else a ring of two or three.
//
// The first 256 outputs of each channel (which reach into the carried
// history) stay on the dense polyphase kernel; the group kernel covers
// outputs 256.. in 128-output tiles.  Taps are packed on the device
// (k_gemm_pack) from the channel's float32 direct-form taps and its NCO
// increment whenever a group's layout or a member's taps or increment
// changed (the host keys each frame's packed buffer on them).
#include "gpud_internal.cuh"

namespace gpud {

constexpr int kGemmM = 128;        // outputs per tile (TMEM lanes)
constexpr int kGemmThreads = 256;  // 8 warps: staging, epilogue (two column halves)
constexpr int kGemmMaxChannels = 128;  // N <= 256

// Output constants of one channel of the tile: output j takes the rotation of
// phase base + j*step (Q0.64) and lands at ext[ext_off + j].
struct GemmOut {
    uint64_t base, step;
    int32_t ext_off, pad;
};

// Shared memory of one tile: mbarriers + TMEM address | per-channel output
// constants | X2 hi planes | X2 lo planes | ns taps stages (hi planes, lo
// planes).  A plane holds one 16-byte
// chunk (two complex samples) of every staged row; its pitch in rows is
// = 1 (mod 8), so the staging stores of consecutive samples spread over the
// banks.
struct GemmLayout {
    int rp, planes, a_plane, o_a, o_alo, o_b, b_stage, bytes;
};

__host__ __device__ inline GemmLayout gemm_layout(int D, int L, int N, int ns) {
    GemmLayout g;
    const int rows = kGemmM + L - 1;
    g.rp = ((rows + 7) / 8) * 8 + 1;
    g.planes = D / 2;
    g.a_plane = g.rp * 16;
    g.o_a = 128 + kGemmMaxChannels * (int)sizeof(GemmOut);
    g.o_alo = g.o_a + g.planes * g.a_plane;
    g.o_b = g.o_alo + g.planes * g.a_plane;
    g.b_stage = 2 * g.planes * N * 16;
    g.bytes = g.o_b + ns * g.b_stage;
    return g;
}

int gemm_smem_bytes_host(int D, int L, int N, int ns) { return gemm_layout(D, L, N, ns).bytes; }
int gemm_tile() { return kGemmM; }
size_t gemm_pack_bytes_host(int D, int L, int N) { return (size_t)L * gemm_layout(D, L, N, 1).b_stage; }

__device__ __forceinline__ float tf32_round(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

// K-major shared-memory matrix descriptor, no swizzle: rows 16 bytes apart
// inside an 8-row core matrix, 8-row groups `sbo` bytes apart, the two
// 16-byte K chunks of one MMA `lbo` bytes apart.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::tf32: F32 accumulator, TF32 A and B, both
// K-major, M = 128, N = n.
__device__ __forceinline__ uint32_t umma_idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kGemmM >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// Arrive on bar once every tcgen05 operation this thread issued has completed.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Packed taps of every group, arm u (grid.x) of group blockIdx.y: the planes
// of the arm's K range for all N rows, hi then lo, in the staging layout of
// the tile kernel (one bulk copy per arm).
__global__ void __launch_bounds__(256)
k_gemm_pack(const GemmGroup *__restrict__ groups, const int *__restrict__ members, const SlotBlock *__restrict__ sbt,
            const ChanParams *__restrict__ prm, const float *__restrict__ taps_arena, float *__restrict__ gb) {
    const GemmGroup g = groups[blockIdx.y];
    const int u = blockIdx.x;
    if (u >= g.L) return;
    const int D = g.D, N = g.ncol, planes = D / 2, half = N / 2;
    float *blk = gb + (size_t)g.b_off / 4 + (size_t)u * (2 * planes * N * 4);
    for (int i = blockIdx.z * blockDim.x + threadIdx.x; i < D * half; i += gridDim.z * blockDim.x) {
        const int pp = i / half, c = i - pp * half;  // sample p' of the row, channel c
        const int k = u * D + D - 1 - pp;              // tap index
        double gr = 0.0, gi = 0.0;
        if (c < g.nmem && k < g.T) {
            const SlotBlock &sb = sbt[members[g.mem_off + c]];
            const ChanParams &cp = prm[sb.slot];
            const double h = (double)taps_arena[cp.dtaps_off + k];
            // exp(-j k inc) from the exact Q0.64 phase
            const double turns = (double)(int64_t)((uint64_t)0 - (uint64_t)k * cp.inc_q) * 0x1p-64;
            double sn, cs;
            sincospi(2.0 * turns, &sn, &cs);
            gr = h * cs;
            gi = h * sn;
        }
        // column 2c (y_r): (re, im) of the sample take (gr, -gi); column 2c+1 (y_i): (gi, gr)
        const double v[2][2] = {{gr, -gi}, {gi, gr}};
        const int q = pp >> 1, off = (pp & 1) * 2;
        float *hp = blk + (size_t)q * N * 4;
        float *lp = blk + (size_t)(planes + q) * N * 4;
#pragma unroll
        for (int col = 0; col < 2; ++col)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const float hi = tf32_round((float)v[col][e]);
                const float lo = tf32_round((float)(v[col][e] - (double)hi));
                hp[(2 * c + col) * 4 + off + e] = hi;
                lp[(2 * c + col) * 4 + off + e] = lo;
            }
    }
}

// One 128-output tile of one group (work item (group, tile)).
__global__ void __launch_bounds__(kGemmThreads, 1)
k_extract_gemm(const int2 *__restrict__ work, const GemmGroup *__restrict__ groups, const int *__restrict__ members,
               const SlotBlock *__restrict__ sbt, const ChanParams *__restrict__ prm,
               const ChanState *__restrict__ st, const float2 *__restrict__ x, int n, const float *__restrict__ gb,
               float2 *__restrict__ ext, unsigned *fault) {
    extern __shared__ __align__(1024) unsigned char gsm[];
    const int2 w = work[blockIdx.x];
    const GemmGroup g = groups[w.x];
    const int D = g.D, L = g.L, N = g.ncol, NS = g.ns, NA = g.na;
    const GemmLayout lo = gemm_layout(D, L, N, NS);
    uint64_t *fullb = reinterpret_cast<uint64_t *>(gsm);  // [3]: taps stage filled
    uint64_t *freeb = fullb + 3;                          // [3]: taps stage consumed by the MMAs
    uint64_t *accb = fullb + 6;                           // every MMA of the tile done
    uint64_t *rawb = fullb + 7;                           // raw block span landed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(gsm + 64);
    GemmOut *outc = reinterpret_cast<GemmOut *>(gsm + 128);
    const int tid = (int)threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int j0 = g.jt0 + w.y * kGemmM;
    const int used = NA * N;  // accumulator a in columns [a*N, (a+1)*N)
    const uint32_t ncols = used <= 32 ? 32u : used <= 64 ? 64u : used <= 128 ? 128u : used <= 256 ? 256u : 512u;
    const char *gblk = reinterpret_cast<const char *>(gb) + g.b_off;

    if (tid == 0) {
        for (int i = 0; i < 3; ++i) {
            mbar_init(fullb + i, 1);
            mbar_init(freeb + i, 1);
        }
        mbar_init(accb, 1);
        mbar_init(rawb, 1);
        mbar_init_fence();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // The tile's raw block span comes in by one bulk copy into the last taps
    // stage (filled with its arm only after the staging below) when it fits
    // there and lies inside the block; the taps of the other first arms by
    // one bulk copy per stage.
    const int rows = kGemmM + L - 1;
    const int i0 = -g.pc + (j0 - L + 1) * D;
    const int total = rows * D;
    const int a0 = i0 & ~1;
    const int cnt = (i0 - a0 + total + 1) & ~1;
    const bool raw = (long long)a0 + cnt <= (long long)n && cnt * 8 <= lo.b_stage;
    const int nb0 = raw ? NS - 1 : NS;  // stages loaded before the staging
    char *rawp = reinterpret_cast<char *>(gsm + lo.o_b + (NS - 1) * lo.b_stage);
    if (tid == 0) {
        if (raw) {
            mbar_arrive_expect_tx(rawb, (unsigned)cnt * 8u);
            bulk_to_smem(rawp, x + a0, (unsigned)cnt * 8u, rawb);
        }
        for (int u = 0; u < nb0 && u < L; ++u) {
            mbar_arrive_expect_tx(fullb + u, (unsigned)lo.b_stage);
            bulk_to_smem(gsm + lo.o_b + u * lo.b_stage, gblk + (size_t)u * lo.b_stage, (unsigned)lo.b_stage,
                         fullb + u);
        }
    }
    // per-channel output constants (read by the epilogue)
    if (tid < g.nmem) {
        const SlotBlock &sb = sbt[members[g.mem_off + tid]];
        const uint64_t inc = prm[sb.slot].inc_q;
        GemmOut o;
        o.base = st[sb.slot].nco_q + (uint64_t)(int64_t)(D - g.pc - 1) * inc;
        o.step = (uint64_t)D * inc;
        o.ext_off = sb.ext_off;
        o.pad = 0;
        outc[tid] = o;
    }
    // block rows j0-L+1 .. j0+127 of X2, split into TF32 hi and lo planes;
    // from the raw span in shared memory, or (tiles past the block end)
    // eight global loads in flight per thread
    bool raw_ok = true;
    if (raw) raw_ok = __syncthreads_and(mbar_wait_bounded(rawb, 0u));
    if (raw && raw_ok) {
        const float2 *src = reinterpret_cast<const float2 *>(rawp) + (i0 - a0);
        int r = tid / D, pp = tid - (tid / D) * D;
        const int dr = kGemmThreads / D, dp = kGemmThreads - dr * D;
        for (int s0 = tid; s0 < total; s0 += kGemmThreads) {
            const float2 v = src[s0];
            const float2 h = make_float2(tf32_round(v.x), tf32_round(v.y));
            const int off = (pp >> 1) * lo.a_plane + r * 16 + (pp & 1) * 8;
            *reinterpret_cast<float2 *>(gsm + lo.o_a + off) = h;
            *reinterpret_cast<float2 *>(gsm + lo.o_alo + off) =
                make_float2(tf32_round(v.x - h.x), tf32_round(v.y - h.y));
            pp += dp;
            r += dr;
            if (pp >= D) {
                pp -= D;
                ++r;
            }
        }
    } else if (!raw) {
        constexpr int U = 8;
        int r = tid / D, pp = tid - (tid / D) * D;
        const int dr = kGemmThreads / D, dp = kGemmThreads - dr * D;
        for (int s0 = tid; s0 < total; s0 += U * kGemmThreads) {
            float2 v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int s = s0 + u * kGemmThreads, i = i0 + s;
                v[u] = (s < total && i < n) ? __ldg(x + i) : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (s0 + u * kGemmThreads < total) {
                    const float2 h = make_float2(tf32_round(v[u].x), tf32_round(v[u].y));
                    const int off = (pp >> 1) * lo.a_plane + r * 16 + (pp & 1) * 8;
                    *reinterpret_cast<float2 *>(gsm + lo.o_a + off) = h;
                    *reinterpret_cast<float2 *>(gsm + lo.o_alo + off) =
                        make_float2(tf32_round(v[u].x - h.x), tf32_round(v[u].y - h.y));
                }
                pp += dp;
                r += dr;
                if (pp >= D) {
                    pp -= D;
                    ++r;
                }
            }
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the staging is read by the tensor core
    __syncthreads();
    if (!raw_ok && tid == 0) device_fault(fault, 5u);
    // the raw span has been consumed: its stage takes its arm
    if (tid == 0 && nb0 < NS && nb0 < L) {
        mbar_arrive_expect_tx(fullb + nb0, (unsigned)lo.b_stage);
        bulk_to_smem(gsm + lo.o_b + nb0 * lo.b_stage, gblk + (size_t)nb0 * lo.b_stage, (unsigned)lo.b_stage,
                     fullb + nb0);
    }

    if (tid == 0) {
        const uint32_t idesc = umma_idesc_tf32(N);
        const uint32_t bplane = (uint32_t)N * 16u;
        // descriptors of offset 0; the start-address field (16-byte units,
        // below 2^14 for any shared address) takes the offsets by addition
        const uint64_t dah0 = umma_desc(smem_u32(gsm + lo.o_a), (uint32_t)lo.a_plane, 128u);
        const uint64_t dal0 = umma_desc(smem_u32(gsm + lo.o_alo), (uint32_t)lo.a_plane, 128u);
        const uint64_t db0 = umma_desc(smem_u32(gsm + lo.o_b), bplane, 128u);
        const uint64_t a_step = (uint64_t)(2 * lo.a_plane) >> 4, b_step = (uint64_t)(2 * bplane) >> 4;
        const uint64_t b_lo = (uint64_t)((uint32_t)lo.planes * bplane) >> 4;
        const int nsteps = lo.planes / 2;
        bool ok = raw_ok;  // no staging, no MMAs (the fault is recorded above)
        // the x_hi*g_hi pass of arm u into accumulator u % NH; both correction
        // passes (2^-11 of it) into the last one, so no large accumulator is
        // rounded for the small terms
        const int NH = NA > 1 ? NA - 1 : 1;
        const uint32_t dcor = tmem + (uint32_t)((NA - 1) * N);
        uint32_t acc_cor = NA > 1 ? 0u : 1u;
        for (int u = 0; ok && u < L; ++u) {
            const uint32_t dacc = tmem + (uint32_t)((u % NH) * N);
            uint32_t acc = u < NH ? 0u : 1u;  // the first arm of an accumulator overwrites it
            const int stg = u % NS;
            if (!mbar_wait_bounded(fullb + stg, (unsigned)(u / NS) & 1u)) {
                ok = false;
                break;
            }
            tc_fence_after();
            uint64_t dah = dah0 + (uint64_t)(L - 1 - u);  // arm u reads the rows u earlier (16 bytes a row)
            uint64_t dal = dal0 + (uint64_t)(L - 1 - u);
            uint64_t dbh = db0 + ((uint64_t)(stg * lo.b_stage) >> 4);
            // the arm's x_hi*g_hi MMAs, then its correction MMAs: consecutive
            // MMAs stay on one accumulator (switching between them costs
            // tensor-core throughput)
            for (int s = 0; s < nsteps; ++s) {
                umma_tf32(dacc, dah + (uint64_t)s * a_step, dbh + (uint64_t)s * b_step, idesc, acc);
                acc = 1;
            }
            const uint32_t dc = NA > 1 ? dcor : dacc;
            for (int s = 0; s < nsteps; ++s) {
                umma_tf32(dc, dah + (uint64_t)s * a_step, dbh + (uint64_t)s * b_step + b_lo, idesc, acc_cor);
                acc_cor = 1;
                umma_tf32(dc, dal + (uint64_t)s * a_step, dbh + (uint64_t)s * b_step, idesc, 1u);
            }
            umma_commit(freeb + stg);
            // refill: with several stages, the previous arm's stage once its
            // MMAs are done (the current arm's keep the tensor core busy
            // meanwhile) takes arm u-1+NS; with one stage, this arm's stage
            // takes arm u+1 once this arm's MMAs are done
            const int t = NS > 1 ? u - 1 + NS : u + 1;  // arm to load
            if (t - NS >= 0 && t < L) {
                const int ps = t % NS;
                if (!mbar_wait_bounded(freeb + ps, (unsigned)((t - NS) / NS) & 1u)) {
                    ok = false;
                    break;
                }
                mbar_arrive_expect_tx(fullb + ps, (unsigned)lo.b_stage);
                bulk_to_smem(gsm + lo.o_b + ps * lo.b_stage, gblk + (size_t)t * lo.b_stage, (unsigned)lo.b_stage,
                             fullb + ps);
            }
        }
        if (!ok && raw_ok) device_fault(fault, 3u);
        umma_commit(accb);  // after every MMA issued above (at once when none was)
    }

    // epilogue: warp w reads TMEM lanes 32*(w%4).. (its 32 output rows) and
    // every other 16-column chunk starting at w/4
    // warp-uniform: the TMEM loads below are .sync.aligned
    const bool done = __all_sync(0xffffffffu, mbar_wait_bounded(accb, 0u));
    tc_fence_after();
    if (done) {
        const int qd = warp & 3;
        const int j = j0 + qd * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(qd * 32) << 16);
        for (int ch = warp >> 2; ch < N / 16; ch += 2) {
            float sum[16];
            // two accumulators in flight per wait
            for (int a = 0; a < NA; a += 2) {
                uint32_t v0[16], v1[16];
                tmem_ld16(lane_base + (uint32_t)(a * N + ch * 16), v0);
                if (a + 1 < NA) tmem_ld16(lane_base + (uint32_t)((a + 1) * N + ch * 16), v1);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    float t = __uint_as_float(v0[i]);
                    if (a + 1 < NA) t += __uint_as_float(v1[i]);
                    sum[i] = a == 0 ? t : sum[i] + t;
                }
            }
            if (j < g.n_out) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int c = ch * 8 + i;
                    if (c < g.nmem) {
                        const GemmOut o = outc[c];
                        const float2 rot = q64_phasor(o.base + (uint64_t)j * o.step);
                        ext[o.ext_off + j] = cmulf(make_float2(sum[2 * i], sum[2 * i + 1]), rot);
                    }
                }
            }
        }
    } else if (lane == 0) {
        device_fault(fault, 4u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

cudaError_t launch_gemm_pack(int ngroups, int max_l, cudaStream_t sm, const GemmGroup *groups, const int *members,
                             const SlotBlock *sbt, const ChanParams *prm, const float *taps, float *gb) {
    k_gemm_pack<<<dim3(max_l, ngroups, 8), 128, 0, sm>>>(groups, members, sbt, prm, taps, gb);
    return cudaGetLastError();
}

cudaError_t launch_extract_gemm(int grid, int smem, cudaStream_t sm, const int2 *work, const GemmGroup *groups,
                                const int *members, const SlotBlock *sbt, const ChanParams *prm, const ChanState *st,
                                const float2 *x, int n, const float *gb, float2 *ext, unsigned *fault) {
    static std::atomic<uint64_t> optin{0};
    cudaError_t e = smem_optin_once(optin, (const void *)k_extract_gemm, 220 * 1024);
    if (e != cudaSuccess) return e;
    k_extract_gemm<<<grid, kGemmThreads, smem, sm>>>(work, groups, members, sbt, prm, st, x, n, gb, ext, fault);
    return cudaGetLastError();
}

}  // namespace gpud

// Tensor-core (tcgen05) form of the raw-amplitude contraction F1:
//   S_tau[p][q][y][x][r][z] = sum_f A1[y][p][x][f] B1[q][r][z][f]
//                           + sum_m A2n[q][p][x][m] B2[y][r][z][m]
// (A2n holds -ovoo, so the ooov term is a plain second K segment).
//
// Operands are 16-bit hi/lo splits of the FP64 inputs, scaled by powers of two
// (fp16) or unscaled (bf16), stored as [h][...] so one 5-D tensor map covers
// both halves.  Each K step issues hi*hi + hi*lo + lo*hi into one FP32 TMEM
// accumulator.
//
// Tile: 128 rows = 8 p x 16 x, BN columns = BN/16 r x 16 z, K blocks of 64.
// Persistent CTAs (one per SM), warp roles: 0 TMA producer, 1 MMA issuer and
// TMEM owner, 2-5 epilogue (TMEM -> registers -> staging, FP32).
#pragma once
#include "common.cuh"
#include "tc_ptx.cuh"

namespace tb {

constexpr int kTcBM = 128;
constexpr int kTcBK = 64;

template <int BN>
struct TcCfg {
    static constexpr int A_BYTES = kTcBM * kTcBK * 2;
    static constexpr int B_BYTES = BN * kTcBK * 2;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int STAGES = (BN >= 256) ? 2 : 3;
    static constexpr int BAR_BYTES = 256;
    static constexpr int STORE_BYTES = 8 * 32 * 32 * 4;   // one 32 x 32 FP32 store box per epilogue warp
    static constexpr int SMEM = STAGES * STAGE_BYTES + STORE_BYTES + BAR_BYTES + 1024;
    static constexpr int RT = BN / 16;
    static constexpr int TMEM_COLS = 2 * BN;
};

struct TcF1Params {
    CUtensorMap tmS[6];       // per ordering with full 16 x 16 (x, z) blocks: S_tau as
                              // [p][q][y][x][r*16+z], box {32, 16, 1, 1, 2}, 128B swizzle
    int tmS_ok[6];            // 1 where tmS is valid (else plain stores)
    Dims d;
    ChunkDesc ch;
    int cum[7];        // prefix over orderings of tile counts
    int mt_count;      // p tiles of 8
    int nt_count;      // r tiles of BN/16
    int nkb1, nkb2;    // K blocks of the ovvv and ooov terms
    float *S;
    const float *out_scale;   // device scalar: 1 / (scale_A * scale_B)
    unsigned *wmax_bits;      // device: running max |W| of this chunk (float bits)
    int *err;
    int bf16;
    int kseg;                 // K blocks per TMEM accumulation segment
};

constexpr int kF1Threads = 320;   // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue

struct F1Tile {
    int tau, y, q, mt, nt;
};

__device__ __forceinline__ F1Tile f1_decode(const TcF1Params &P, int t) {
    F1Tile T;
    int tau = 0;
    while (tau + 1 < P.ch.nperm && t >= P.cum[tau + 1]) tau++;
    int rem = t - P.cum[tau];
    T.tau = tau;
    T.nt = rem % P.nt_count;
    rem /= P.nt_count;
    T.mt = rem % P.mt_count;
    rem /= P.mt_count;
    T.q = rem % P.d.o;
    T.y = rem / P.d.o;
    return T;
}

// Operand tensor maps of one W contraction (16-bit hi/lo splits).
struct F1Maps {
    CUtensorMap a1, b1, a2, b2;
};

// One problem's chunk in a batched launch: its maps and parameters, in device
// memory (written before the launch, 64-byte aligned).
struct alignas(64) F1Job {
    F1Maps m;
    TcF1Params P;
};

// Index j of the job that holds global work index t: start[j] <= t < start[j+1].
__device__ __forceinline__ int job_of(const int *__restrict__ start, int njobs, int t) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// BATCH = false: one chunk (maps M0, parameters P0).  BATCH = true: the tiles
// of njobs chunks (of different problems) numbered job after job
// (job_start[j] = first tile of job j, job_start[njobs] = total); every tile
// reads its job's maps and parameters.
template <int BN, bool BATCH>
__global__ void __launch_bounds__(kF1Threads, 1)
    k_f1_tc(const __grid_constant__ F1Maps M0, const __grid_constant__ TcF1Params P0,
            const F1Job *__restrict__ jobs, const int *__restrict__ job_start, int njobs) {
    using C = TcCfg<BN>;
    // job of global tile t (BATCH) and the tile's index within it
    // (each role walks its tiles in increasing order: after the first binary
    // search the job index only moves forward)
    int jcur = -1;
    auto job_tile = [&](int t, int &lt) -> int {
        if constexpr (BATCH) {
            if (jcur < 0) jcur = job_of(job_start, njobs, t);
            while (jcur + 1 < njobs && job_start[jcur + 1] <= t) jcur++;
            lt = t - job_start[jcur];
            return jcur;
        } else {
            lt = t;
            return 0;
        }
    };
    // the parameters themselves are bound with BATCH ? jobs[j].X : X0, which
    // folds to the __grid_constant__ parameter in the single-chunk kernel
    const TcF1Params &Pfirst = BATCH ? jobs[0].P : P0;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    float *sstore = (float *)(smem + C::STAGES * C::STAGE_BYTES);   // 1024-byte aligned boxes
    uint64_t *full = (uint64_t *)(smem + C::STAGES * C::STAGE_BYTES + C::STORE_BYTES);
    uint64_t *empty = full + C::STAGES;
    uint64_t *tfull = empty + C::STAGES;
    uint64_t *tempty = tfull + 2;
    uint64_t *drain = tempty + 2;
    uint32_t *tmem_slot = (uint32_t *)(drain + 1);
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 8);
        }
        mbar_init(drain, 1);
        fence_mbar_init();
    }
    if (!BATCH && warp == 0 && lane == 0) {
        tma_prefetch_desc(&M0.a1);
        tma_prefetch_desc(&M0.b1);
        tma_prefetch_desc(&M0.a2);
        tma_prefetch_desc(&M0.b2);
    }
    if (warp == 1) {
        tmem_alloc(tmem_slot, C::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    volatile int *abortp = &s_abort;
    const int total = BATCH ? job_start[njobs] : P0.cum[P0.ch.nperm];

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer ----------------
        int stage = 0;
        uint32_t phase = 0;
        uint32_t pend_phase[C::STAGES];
        bool pending[C::STAGES];
        for (int s = 0; s < C::STAGES; s++) pending[s] = false;
        bool ok = true;
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int lt;
            const int jb = job_tile(t, lt);
            const TcF1Params &P = BATCH ? jobs[jb].P : P0;
            const F1Maps &M = BATCH ? jobs[jb].m : M0;
            const F1Tile T = f1_decode(P, lt);
            const PermBlock &pb = P.ch.pb[T.tau];
            const int yg = pb.Y0 + T.y;
            const int nkb = P.nkb1 + P.nkb2;
            for (int kb = 0; kb < nkb; kb++) {
                if (!mbar_wait(&empty[stage], phase ^ 1u, abortp)) {
                    ok = false;
                    break;
                }
                pending[stage] = false;
                mbar_expect_tx(&full[stage], C::STAGE_BYTES);
                uint8_t *sA = smem + stage * C::STAGE_BYTES;
                uint8_t *sAl = sA + C::A_BYTES;
                uint8_t *sB = sAl + C::A_BYTES;
                uint8_t *sBl = sB + C::B_BYTES;
                if (kb < P.nkb1) {
                    const int f0 = kb * kTcBK;
                    tma_load_5d(sA, &M.a1, &full[stage], f0, pb.X0, T.mt * 8, yg, 0);
                    tma_load_5d(sAl, &M.a1, &full[stage], f0, pb.X0, T.mt * 8, yg, 1);
                    tma_load_5d(sB, &M.b1, &full[stage], f0, pb.Z0, T.nt * C::RT, T.q, 0);
                    tma_load_5d(sBl, &M.b1, &full[stage], f0, pb.Z0, T.nt * C::RT, T.q, 1);
                } else {
                    const int m0 = (kb - P.nkb1) * kTcBK;
                    tma_load_5d(sA, &M.a2, &full[stage], m0, pb.X0, T.mt * 8, T.q, 0);
                    tma_load_5d(sAl, &M.a2, &full[stage], m0, pb.X0, T.mt * 8, T.q, 1);
                    tma_load_5d(sB, &M.b2, &full[stage], m0, pb.Z0, T.nt * C::RT, yg, 0);
                    tma_load_5d(sBl, &M.b2, &full[stage], m0, pb.Z0, T.nt * C::RT, yg, 1);
                }
                pending[stage] = true;
                pend_phase[stage] = phase;
                if (++stage == C::STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
        }
        if (!ok) {
            *abortp = 1;
            atomicOr(Pfirst.err, 1);
            // let copies already in flight land before the CTA can exit
            for (int s = 0; s < C::STAGES; s++)
                if (pending[s]) {
                    for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(&full[s], pend_phase[s]); i++) {
                    }
                }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: one TMEM buffer per K segment ----------------
        const uint32_t idesc = make_idesc_f16(kTcBM, BN, Pfirst.bf16 != 0, false, false);
        int stage = 0;
        uint32_t phase = 0;
        int seg = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int lt;
            const int jb = job_tile(t, lt);
            const TcF1Params &P = BATCH ? jobs[jb].P : P0;
            const int nkb = P.nkb1 + P.nkb2;
            for (int k0 = 0; k0 < nkb && ok; k0 += P.kseg, seg++) {
                const int acc = seg & 1;
                const uint32_t accph = (seg >> 1) & 1;
                if (!mbar_wait(&tempty[acc], accph ^ 1u, abortp)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                const int k1 = (k0 + P.kseg < nkb) ? k0 + P.kseg : nkb;
                for (int kb = k0; kb < k1; kb++) {
                    if (!mbar_wait(&full[stage], phase, abortp)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_h = smem_u32(smem + stage * C::STAGE_BYTES);
                    const uint32_t a_l = a_h + C::A_BYTES;
                    const uint32_t b_h = a_l + C::A_BYTES;
                    const uint32_t b_l = b_h + C::B_BYTES;
#pragma unroll
                    for (int ks = 0; ks < kTcBK / 16; ks++) {
                        const uint64_t dah = make_sdesc_sw128(a_h + 32 * ks, 16, 1024);
                        const uint64_t dal = make_sdesc_sw128(a_l + 32 * ks, 16, 1024);
                        const uint64_t dbh = make_sdesc_sw128(b_h + 32 * ks, 16, 1024);
                        const uint64_t dbl = make_sdesc_sw128(b_l + 32 * ks, 16, 1024);
                        umma_f16(d_tmem, dah, dbh, idesc, (kb > k0 || ks > 0) ? 1u : 0u);
                        umma_f16(d_tmem, dah, dbl, idesc, 1u);
                        umma_f16(d_tmem, dal, dbh, idesc, 1u);
                    }
                    umma_commit(&empty[stage]);
                    if (++stage == C::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(&tfull[acc]);
            }
        }
        if (!ok) {
            *abortp = 1;
            atomicOr(Pfirst.err, 2);
        }
        // all MMAs of this thread complete before TMEM can be released
        umma_commit(drain);
        for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(drain, 0); i++) {
        }
    } else if (warp >= 2) {
        // ---------------- epilogue: sum the segments (FP32, round to nearest) ----------------
        constexpr int HC = BN / 2;          // columns handled by one epilogue warp
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        float wmax = 0.f;
        unsigned *wmax_dst = Pfirst.wmax_bits;   // running max |W| goes to the tile's problem
        const float sc0 = BATCH ? 0.f : *P0.out_scale;   // single chunk: read once
        int seg = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int lt;
            const int jb = job_tile(t, lt);
            const TcF1Params &P = BATCH ? jobs[jb].P : P0;
            const int o = P.d.o;
            const int nkb = P.nkb1 + P.nkb2;
            if (BATCH && P.wmax_bits != wmax_dst) {
                for (int off = 16; off > 0; off >>= 1) wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
                if (lane == 0 && wmax > 0.f) atomicMax(wmax_dst, __float_as_uint(wmax));
                wmax = 0.f;
                wmax_dst = P.wmax_bits;
            }
            float accf[HC];
#pragma unroll
            for (int j = 0; j < HC; j++) accf[j] = 0.f;
            for (int k0 = 0; k0 < nkb; k0 += P.kseg, seg++) {
                const int acc = seg & 1;
                const uint32_t accph = (seg >> 1) & 1;
                if (!mbar_wait(&tfull[acc], accph, abortp)) {
                    *abortp = 1;
                    atomicOr(Pfirst.err, 4);
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int c = 0; c < HC / 32; c++) {
                    uint32_t vv[32];
                    tmem_ld32(tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * BN + half * HC + c * 32),
                              vv);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 32; j++) accf[c * 32 + j] += __uint_as_float(vv[j]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[acc]);
            }
            if (!ok) break;
            const float sc = BATCH ? *P.out_scale : sc0;
            const F1Tile T = f1_decode(P, lt);
            const PermBlock &pb = P.ch.pb[T.tau];
            const int p = T.mt * 8 + row / 16;
            const int x = row % 16;
            const bool vrow = (p < o) && (x < pb.Tx);
            float *dst = P.S + pb.soff +
                         ((((long long)(p * o + T.q) * pb.Ty + T.y) * pb.Tx + x) * o) * pb.Tz;
            if (P.tmS_ok[T.tau]) {
                // Full blocks: each 32 x 32 piece (lane = row = 16 p-local x 16 x) goes to
                // this warp's 128B-swizzled shared box and leaves as one TMA store, so the
                // rows reach HBM as whole 128-byte lines instead of 32 scattered 16-byte
                // pieces per warp store.
                float *box = sstore + (warp - 2) * 32 * 32;
                const int p0 = T.mt * 8 + quarter * 2;
#pragma unroll
                for (int c = 0; c < HC / 32; c++) {
                    if (c > 0) {
                        if (lane == 0) bulk_wait_read0();
                        __syncwarp();
                    }
#pragma unroll
                    for (int ch = 0; ch < 8; ch++) {
                        float4 w;
                        w.x = accf[c * 32 + ch * 4 + 0] * sc;
                        w.y = accf[c * 32 + ch * 4 + 1] * sc;
                        w.z = accf[c * 32 + ch * 4 + 2] * sc;
                        w.w = accf[c * 32 + ch * 4 + 3] * sc;
                        if (vrow)
                            wmax = fmaxf(wmax, fmaxf(fmaxf(fabsf(w.x), fabsf(w.y)), fmaxf(fabsf(w.z), fabsf(w.w))));
                        *reinterpret_cast<float4 *>(box + lane * 32 + 4 * (ch ^ (lane & 7))) = w;
                    }
                    fence_proxy_async_smem();
                    __syncwarp();
                    const int rz0 = T.nt * BN + half * HC + c * 32;
                    if (lane == 0 && p0 < o && rz0 < o * 16) {
                        tma_store_5d(&P.tmS[T.tau], box, rz0, 0, T.y, T.q, p0);
                        bulk_commit();
                    }
                }
                if (lane == 0) bulk_wait_read0();
                __syncwarp();
            } else if (vrow) {
#pragma unroll
                for (int h = 0; h < HC / 16; h++) {
                    const int r = T.nt * C::RT + half * (HC / 16) + h;
                    if (r >= o) continue;
                    float *d = dst + (long long)r * pb.Tz;
                    if (pb.Tz == 16) {
                        float4 *d4 = reinterpret_cast<float4 *>(d);
#pragma unroll
                        for (int z4 = 0; z4 < 4; z4++) {
                            float4 w;
                            w.x = accf[h * 16 + z4 * 4 + 0] * sc;
                            w.y = accf[h * 16 + z4 * 4 + 1] * sc;
                            w.z = accf[h * 16 + z4 * 4 + 2] * sc;
                            w.w = accf[h * 16 + z4 * 4 + 3] * sc;
                            wmax = fmaxf(wmax, fmaxf(fmaxf(fabsf(w.x), fabsf(w.y)), fmaxf(fabsf(w.z), fabsf(w.w))));
                            d4[z4] = w;
                        }
                    } else {
#pragma unroll
                        for (int z = 0; z < 16; z++) {
                            if (z < pb.Tz) {
                                const float w1 = accf[h * 16 + z] * sc;
                                wmax = fmaxf(wmax, fabsf(w1));
                                d[z] = w1;
                            }
                        }
                    }
                }
            }
        }
        if (lane == 0) bulk_wait0();   // this warp's stores complete before the CTA retires
        for (int off = 16; off > 0; off >>= 1) wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
        if (lane == 0 && wmax > 0.f) atomicMax(wmax_dst, __float_as_uint(wmax));
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, C::TMEM_COLS);
    }
}

}  // namespace tb

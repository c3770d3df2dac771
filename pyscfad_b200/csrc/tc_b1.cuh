// Tensor-core (tcgen05) form of the adjoint contractions, one launch per
// ordering tau of a chunk.  Wbar_tau is staged by the epilogue as fp16/bf16
// hi/lo splits in the layout [h][y][p][x][q][r][z] (scaled by a per-chunk
// power of two), which serves all four products through 5-D TMA boxes:
//
//   kind 0  ovvv:  G_A1[y][p][x][f] += sum_{q,rz} Wbar[y][p][x][q][rz] B1[q][rz][f]
//                  rows (p,x) K-major, batch y, K = (q, rz)
//   kind 1  t2:    G_B1[q][rz][f]   += sum_{y,p,x} Wbar[y][p][x][q][rz] A1[y][p][x][f]
//                  rows rz MN-major, batch q, K = (y, p, x)
//   kind 2  ovoo:  G_A2[q][p][x][m] -= sum_{y,rz} Wbar[y][p][x][q][rz] B2[y][rz][m]
//                  rows (p,x) K-major, batch q, K = (y, rz)
//   kind 3  t2:    G_B2[y][rz][m]   += sum_{q,p,x} Wbar[y][p][x][q][rz] A2n[q][p][x][m]
//                  rows rz MN-major, batch y, K = (q, p, x)   (A2n = -ovoo)
//
// (the adjoint GEMMs of get_eris_amps_bar, ccsd_t_vjp.c:139-246, batched over
// all occupied indices).  The second operand is always MN-major.  Products:
// hi*hi + hi*lo + lo*hi into FP32 TMEM; the epilogue adds the descaled tile
// into the FP64 gradient buffer.
#pragma once
#include "common.cuh"
#include "tc_f1.cuh"
#include "tc_ptx.cuh"

namespace tb {

// One launch covers one kind for ALL orderings tau of a chunk (tiles numbered
// ordering by ordering), so small per-ordering tile counts do not leave SMs
// idle.  Orderings that share an X (or Z) block write the same gradient rows,
// hence the FP64 atomic adds in the epilogue.
struct TcB1Params {
    CUtensorMap tmA[6];     // per ordering: Wbar_tau (first operand)
    CUtensorMap tmB[6];     // per ordering: second operand
    Dims d;
    PermBlock pb[6];
    int nperm;
    int kind;
    int nbatch[6], ntile_m[6], ntile_n;
    int nk_outer[6], nk_inner[6];
    int cum[7];             // prefix of tile counts over orderings
    double *G;
    const double *wscale;   // device: per-chunk Wbar scale
    const double *oscale;   // device: scale of the second operand
    double sign;
    int *err;
    int bf16;
    int kseg;               // K blocks per TMEM accumulation segment
};

constexpr int kB1Threads = 320;   // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
// K segments summed in FP32 before the run goes into the FP64 gradient: runs of
// K <= 512 * 64 keep the rounding of the sum well below the fp16 split error
constexpr int kB1RunSegments = 512;

template <bool A_MN, int BN>
struct TcB1Cfg {
    static constexpr int A_BYTES = kTcBM * kTcBK * 2;
    static constexpr int B_BYTES = BN * kTcBK * 2;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int STAGES = (200 * 1024) / STAGE_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES + 256 + 1024;
    static constexpr int NACC = 4;   // TMEM accumulators: the epilogue sums them in pairs
    static constexpr int TMEM_COLS = NACC * BN < 32 ? 32 : NACC * BN;
    static_assert(NACC * BN <= 512, "TMEM holds 512 columns");
};

// BATCH = false: one chunk (parameters P0).  BATCH = true: the tiles of njobs
// chunks (of different problems, one kind) numbered job after job
// (job_start[j] = first tile of job j, job_start[njobs] = total), parameters
// in device memory.
template <bool A_MN, int BN, bool BATCH>
__global__ void __launch_bounds__(kB1Threads, 1)
    k_b1_tc(const __grid_constant__ TcB1Params P0, const TcB1Params *__restrict__ jobs,
            const int *__restrict__ job_start, int njobs) {
    using C = TcB1Cfg<A_MN, BN>;
    // job of global tile t (BATCH) and the tile's index within it (each role
    // walks its tiles in increasing order: after the first binary search the
    // job index only moves forward); parameters are bound with
    // BATCH ? jobs[j] : P0, the __grid_constant__ parameter in the
    // single-chunk kernel
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
    const TcB1Params &Pfirst = BATCH ? jobs[0] : P0;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + C::STAGES * C::STAGE_BYTES);
    uint64_t *empty = full + C::STAGES;
    uint64_t *tfull = empty + C::STAGES;
    uint64_t *tempty = tfull + C::NACC;
    uint64_t *drain = tempty + C::NACC;
    uint32_t *tmem_slot = (uint32_t *)(drain + 1);
    __shared__ int s_abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_abort = 0;
        for (int s = 0; s < C::STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < C::NACC; a++) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 8);
        }
        mbar_init(drain, 1);
        fence_mbar_init();
    }
    if (!BATCH && warp == 0 && lane == 0) {
        for (int t = 0; t < P0.nperm; t++) {
            tma_prefetch_desc(&P0.tmA[t]);
            tma_prefetch_desc(&P0.tmB[t]);
        }
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
    const int total = BATCH ? job_start[njobs] : P0.cum[P0.nperm];
    // tile t of the chunk with parameters P -> ordering, batch, M tile, N tile
    auto decode = [&](const TcB1Params &P, int t, int &tau, int &b, int &mt, int &nt) {
        tau = 0;
        while (tau + 1 < P.nperm && t >= P.cum[tau + 1]) tau++;
        int rem = t - P.cum[tau];
        const int per_batch = P.ntile_m[tau] * P.ntile_n;
        b = rem / per_batch;
        rem %= per_batch;
        mt = rem / P.ntile_n;
        nt = rem % P.ntile_n;
    };

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
            const TcB1Params &P = BATCH ? jobs[jb] : P0;
            int tau, b, mt, nt;
            decode(P, lt, tau, b, mt, nt);
            const PermBlock &pb = P.pb[tau];
            const int Ty = pb.Ty, Tz = pb.Tz;
            const int nk = P.nk_outer[tau] * P.nk_inner[tau];
            const CUtensorMap *tmA = &P.tmA[tau], *tmB = &P.tmB[tau];
            for (int kb = 0; kb < nk; kb++) {
                if (!mbar_wait(&empty[stage], phase ^ 1u, abortp)) {
                    ok = false;
                    break;
                }
                pending[stage] = false;
                mbar_expect_tx(&full[stage], C::STAGE_BYTES);
                uint8_t *sA = smem + stage * C::STAGE_BYTES;
                uint8_t *sB = sA + 2 * C::A_BYTES;
                const int ko = kb / P.nk_inner[tau], ki = kb % P.nk_inner[tau];
                for (int h = 0; h < 2; h++) {
                    uint8_t *a = sA + h * C::A_BYTES;
                    uint8_t *bb = sB + h * C::B_BYTES;
                    switch (P.kind) {
                    case 0:   // batch y, K = (q = ko, rz block = ki)
                        tma_load_5d(a, tmA, &full[stage], ki * 64, ko, 0, mt * 8, h * Ty + b);
                        for (int j = 0; j < BN / 64; j++)
                            tma_load_5d(bb + j * 8192, tmB, &full[stage], nt * BN + j * 64, pb.Z0, ki * 64 / Tz, ko, h);
                        break;
                    case 1:   // batch q, K = (y = ko, p group = ki)
                        for (int j = 0; j < 2; j++)
                            tma_load_5d(a + j * 8192, tmA, &full[stage], mt * 128 + j * 64, b, 0, ki * 4, h * Ty + ko);
                        for (int j = 0; j < BN / 64; j++)
                            tma_load_5d(bb + j * 8192, tmB, &full[stage], nt * BN + j * 64, pb.X0, ki * 4, pb.Y0 + ko, h);
                        break;
                    case 2:   // batch q, K = (y = ko, rz block = ki)
                        tma_load_5d(a, tmA, &full[stage], ki * 64, b, 0, mt * 8, h * Ty + ko);
                        for (int j = 0; j < BN / 64; j++)
                            tma_load_5d(bb + j * 8192, tmB, &full[stage], nt * BN + j * 64, pb.Z0, ki * 64 / Tz, pb.Y0 + ko, h);
                        break;
                    default:  // batch y, K = (q = ko, p group = ki)
                        for (int j = 0; j < 2; j++)
                            tma_load_5d(a + j * 8192, tmA, &full[stage], mt * 128 + j * 64, ko, 0, ki * 4, h * Ty + b);
                        for (int j = 0; j < BN / 64; j++)
                            tma_load_5d(bb + j * 8192, tmB, &full[stage], nt * BN + j * 64, pb.X0, ki * 4, ko, h);
                        break;
                    }
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
            atomicOr(Pfirst.err, 8);
            for (int s = 0; s < C::STAGES; s++)
                if (pending[s]) {
                    for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(&full[s], pend_phase[s]); i++) {
                    }
                }
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: one TMEM buffer per K segment ----------------
        const uint32_t idesc = make_idesc_f16(kTcBM, BN, Pfirst.bf16 != 0, A_MN, true);
        int stage = 0;
        uint32_t phase = 0;
        int seg = 0;   // running segment counter (same sequence as the epilogue)
        bool ok = true;
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int lt;
            const int jb = job_tile(t, lt);
            const TcB1Params &P = BATCH ? jobs[jb] : P0;
            int tau, b, mt, nt;
            decode(P, lt, tau, b, mt, nt);
            const int nk = P.nk_outer[tau] * P.nk_inner[tau];
            for (int k0 = 0; k0 < nk && ok; k0 += P.kseg, seg++) {
                const int acc = seg % C::NACC;
                const uint32_t accph = (seg / C::NACC) & 1;
                if (!mbar_wait(&tempty[acc], accph ^ 1u, abortp)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
                const int k1 = (k0 + P.kseg < nk) ? k0 + P.kseg : nk;
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
                        uint64_t dah, dal;
                        if (A_MN) {
                            dah = make_sdesc_sw128(a_h + 2048 * ks, 8192, 1024);
                            dal = make_sdesc_sw128(a_l + 2048 * ks, 8192, 1024);
                        } else {
                            dah = make_sdesc_sw128(a_h + 32 * ks, 16, 1024);
                            dal = make_sdesc_sw128(a_l + 32 * ks, 16, 1024);
                        }
                        const uint64_t dbh = make_sdesc_sw128(b_h + 2048 * ks, 8192, 1024);
                        const uint64_t dbl = make_sdesc_sw128(b_l + 2048 * ks, 8192, 1024);
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
            atomicOr(Pfirst.err, 16);
        }
        umma_commit(drain);
        for (uint32_t i = 0; i < kSpinLimit && !mbar_try_wait(drain, 0); i++) {
        }
    } else if (warp >= 2) {
        // ---------------- epilogue: G += sign * sum_seg D_seg / (wscale * oscale) ----------------
        constexpr int HC = BN / 2;            // columns per epilogue warp
        const int quarter = warp & 3;         // TMEM lane quarter this warp may access
        const int half = (warp - 2) >> 2;     // which half of the columns
        const int row = quarter * 32 + lane;
        const double sc0 = BATCH ? 0.0 : P0.sign / ((*P0.wscale) * (*P0.oscale));   // single chunk: read once
        int seg = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < total && ok; t += gridDim.x) {
            int lt;
            const int jb = job_tile(t, lt);
            const TcB1Params &P = BATCH ? jobs[jb] : P0;
            const int o = P.d.o, v = P.d.v, Kp = P.d.Kp;
            int tau, b, mt, nt;
            decode(P, lt, tau, b, mt, nt);
            const PermBlock &pb = P.pb[tau];
            const int Tz = pb.Tz;
            const int nk = P.nk_outer[tau] * P.nk_inner[tau];
            const double sc = BATCH ? P.sign / ((*P.wscale) * (*P.oscale)) : sc0;
            long long roff = -1;
            if (P.kind == 0 || P.kind == 2) {
                const int p = mt * 8 + row / 16, x = row % 16;
                if (p < o && x < pb.Tx) {
                    if (P.kind == 0)
                        roff = ((((long long)pb.Y0 + b) * o + p) * v + pb.X0 + x) * Kp;
                    else
                        roff = (((long long)b * o + p) * v + pb.X0 + x) * o;
                }
            } else {
                const int rz = mt * 128 + row;
                if (rz < o * Tz) {
                    const int r = rz / Tz, z = rz % Tz;
                    if (P.kind == 1)
                        roff = (((long long)b * o + r) * v + pb.Z0 + z) * Kp;
                    else
                        roff = ((((long long)pb.Y0 + b) * o + r) * v + pb.Z0 + z) * o;
                }
            }
            const int ncol = (P.kind <= 1) ? v : o;
            const int c0 = nt * BN + half * HC;
            float acc[HC];
#pragma unroll
            for (int j = 0; j < HC; j++) acc[j] = 0.f;
            // G += sc * acc, then acc = 0: the FP64 sum of a run of at most
            // kB1RunSegments FP32-summed segments
            auto flush = [&]() {
                if (roff >= 0) {
#pragma unroll
                    for (int j = 0; j < HC; j++) {
                        const int col = c0 + j;
                        if (col < ncol) atomicAdd(&P.G[roff + col], sc * (double)acc[j]);
                    }
                }
#pragma unroll
                for (int j = 0; j < HC; j++) acc[j] = 0.f;
            };
            // segments in pairs, added into the FP32 run sum; every kB1RunSegments
            // segments the run goes into G in FP64
            const int nseg = (nk + P.kseg - 1) / P.kseg;
            for (int s0 = 0; s0 < nseg; s0 += 2, seg += 2) {
                const bool two = s0 + 1 < nseg;
                const int accA = seg % C::NACC, accB = (seg + 1) % C::NACC;
                if (!mbar_wait(&tfull[accA], (uint32_t)((seg / C::NACC) & 1), abortp) ||
                    (two && !mbar_wait(&tfull[accB], (uint32_t)(((seg + 1) / C::NACC) & 1), abortp))) {
                    *abortp = 1;
                    atomicOr(Pfirst.err, 32);
                    ok = false;
                    break;
                }
                tc_fence_after();
#pragma unroll
                for (int c = 0; c < HC / 8; c++) {
                    const uint32_t lane_base = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * HC + c * 8);
                    uint32_t va[8], vb[8];
                    tmem_ld8(lane_base + (uint32_t)(accA * BN), va);
                    if (two) tmem_ld8(lane_base + (uint32_t)(accB * BN), vb);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const float sum = two ? __uint_as_float(va[j]) + __uint_as_float(vb[j]) : __uint_as_float(va[j]);
                        acc[c * 8 + j] += sum;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&tempty[accA]);
                    if (two) mbar_arrive(&tempty[accB]);
                }
                if (!two) seg -= 1;   // an odd tail used one accumulator
                if ((s0 + 2) % kB1RunSegments == 0 && s0 + 2 < nseg) flush();
            }
            if (!ok) break;
            flush();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem_base, C::TMEM_COLS);
    }
}

}  // namespace tb

// Chunk epilogue: energy and adjoint of the raw triples amplitudes.
//
// One CTA owns one occupied representative i >= j >= k and one triple of
// virtual sub-ranges (a-sub >= b-sub >= c-sub, SB wide).  Every raw
// amplitude w^{pqr}_{xyz} with {p,q,r} = {i,j,k} and {x,y,z} one value from
// each sub-range belongs to exactly one such CTA, and the CTA holds all of
// them: 36 regions = (distinct orderings of the sub-ranges) x (distinct
// orderings of ijk), each SB^3 values, staged in shared memory with
// coalesced loads.
//
// Per orbit item (a >= b >= c), with d = sigma_s(abc) the six orderings,
//   WW(d) = sum_tau w(tau(ijk), tau(d)),  VV(d) likewise from v,
//   Z(d)  = 4X(d) + X(d2,d0,d1) + X(d1,d2,d0) - 2[X(d2,d1,d0) + X(d0,d2,d1) + X(d1,d0,d2)],
//   X = WW + VV/2,
//   E    += (n_ijk n_abc / 18) sum_s WW Z / D,   D = e_i+e_j+e_k-e_a-e_b-e_c
// (the a>=b>=c restricted sum of pyscfad/cc/ccsd_t_slow.py:46-124 rewritten
// over occupied-triplet orbits), and the adjoint
//   Wbar(d) = c (Z + R WW)/D, Vbar(d) = c (R WW)/(2D), dE/dD = -c sum WW Z / D^2
// (ccsd_t_vjp.c:64-117) scattered back to every raw position of the orbit.
// Wbar goes to its own buffer in the layout the gradient contractions read:
// [h][y][p][x][q][r][z].  Vbar never leaves the CTA: since
//   v^{pqr}_{xyz} = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r]
// and the CTA already holds those factors in its V-term tables, its
// contributions to ovov_bar / t2_bar (row sums over the z run of a thread)
// and to t1_bar / fvo_bar (column sums, reduced across the warp) are added
// to the global gradients directly (FP64 reductions).
//
// Item results (Wbar, Vbar per ordering s) are written once per item into
// shared memory over the dead W tile; the write-back maps every raw position
// to its item(s) through the (sub-range ordering, occupied ordering) pairs of
// its region, which in degenerate cases (repeated indices) are several.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace tb {

struct F2Sub {
    int st[3];
    int len[3];
};
constexpr int kMaxSub = 64;

template <typename StageT>
struct F2P {
    Dims d;
    ChunkDesc ch;
    int nsub;
    F2Sub sub[kMaxSub];
    const int *ijk;
    const double *mo_e, *t1, *t2, *ovov, *fvo;
    const StageT *S;    // W per ordering tau: [p][q][y][x][r][z] at ch.pb[tau].soff
    void *SW;           // Wbar out; per tau at 2*soff: [h][y][p][x][q][r][z] (split) or at soff: [y][p][x][q][r][z]
    int split;          // 0: StageT, 1: fp16 hi/lo, 2: bf16 hi/lo
    const double *wscale;
    double ybar;
    int want_grad;
    double *e_part;     // energy partial of each CTA, at sub * n_ijk + rep
    int rep0, sub0;     // first occupied representative / sub-range triple of this launch
    int nsub_l;         // sub-range triples of this launch: block b -> sub0 + b % nsub_l, rep0 + b / nsub_l
    int n_ijk;          // occupied representatives (stride of e_part)
    double *mo_bar, *t1_bar, *fvo_bar, *ovov_bar, *t2_bar;
};

// Shared-memory region layout: element (y,x,z) at y*SY + x*SX + z.  The padded
// strides keep the permuted gathers of a warp within 2-way bank conflicts.
template <int SB>
struct F2Smem {
    static constexpr int SX = SB;
    static constexpr int SY = (SB == 8) ? 69 : SB * SB + 1;
    static constexpr int REG = SY * SB;
    // W tile (y, x, z) at y*SYW + x*SX + z: 8-byte aligned rows for the
    // 8-byte cp.async copies of the FP32 staging (SB = 8); item results keep SY
    static constexpr int SYW = (SB == 8) ? 70 : SY;
    static constexpr int REGW = SYW * SB;
    static constexpr int NV = 3 * SB;
    static constexpr int NVP = NV + 1;
    static constexpr int TAB = 6 * NV * NVP;
    static constexpr int ITEMS = SB * SB * SB;
    static constexpr int NT = (SB == 8) ? 256 : ITEMS;     // threads per CTA
    static constexpr int IPT = ITEMS / NT;                  // items per thread
    static_assert(12 * REG <= 36 * REGW, "item results overlay the W tile");
};

template <typename StageT, int SB>
__host__ __device__ constexpr size_t f2_smem_bytes() {
    return sizeof(StageT) * (36 * F2Smem<SB>::REGW + 2 * F2Smem<SB>::TAB + 2 * 3 * F2Smem<SB>::NV);
}

// 4- and 8-byte asynchronous copies global -> shared (L1-allocating, L2
// evict-first hint: the staging is streamed once); src_bytes < size
// zero-fills the rest of the destination without reading past src_bytes.
__device__ __forceinline__ uint64_t f2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void f2_cp_async(void *smem_dst, const void *gsrc, int size, int src_bytes,
                                            uint64_t pol) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    if (size == 8)
        asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2, %3;" ::"r"(d), "l"(gsrc),
                     "r"(src_bytes), "l"(pol)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2, %3;" ::"r"(d), "l"(gsrc),
                     "r"(src_bytes), "l"(pol)
                     : "memory");
}

__host__ __device__ constexpr inline int pair_index(int sp, int sq) { return 2 * sp + (sq > sp ? sq - 1 : sq); }

// A z run of N contiguous values moved with the widest aligned vector access:
// one warp instruction then fills whole 32-byte sectors instead of touching
// 32 sectors with a 2- or 4-byte write each.  Partial or unaligned runs
// (remainder blocks) fall back to scalar accesses.
template <typename T, int N>
union RunBuf {
    static constexpr int BYTES = N * (int)sizeof(T);
    static constexpr int VB = BYTES >= 16 ? 16 : (BYTES >= 8 ? 8 : 4);
    T e[N];
    uint4 u4[BYTES / 16 > 0 ? BYTES / 16 : 1];
    uint2 u2[BYTES / 8 > 0 ? BYTES / 8 : 1];
};

template <typename T, int N>
__device__ __forceinline__ void st_run(T *dst, const RunBuf<T, N> &b, int n) {
    using B = RunBuf<T, N>;
    const uintptr_t a = reinterpret_cast<uintptr_t>(dst);
    if (n == N && B::VB == 16 && (a & 15) == 0) {
#pragma unroll
        for (int c = 0; c < B::BYTES / 16; c++) reinterpret_cast<uint4 *>(dst)[c] = b.u4[c];
    } else if (n == N && B::VB == 8 && (a & 7) == 0) {
#pragma unroll
        for (int c = 0; c < B::BYTES / 8; c++) reinterpret_cast<uint2 *>(dst)[c] = b.u2[c];
    } else {
#pragma unroll
        for (int z = 0; z < N; z++)
            if (z < n) dst[z] = b.e[z];
    }
}

template <typename T, int N>
__device__ __forceinline__ void ld_run(RunBuf<T, N> &b, const T *src, int n) {
    using B = RunBuf<T, N>;
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    if (n == N && B::VB == 16 && (a & 15) == 0) {
#pragma unroll
        for (int c = 0; c < B::BYTES / 16; c++) b.u4[c] = reinterpret_cast<const uint4 *>(src)[c];
    } else {
#pragma unroll
        for (int z = 0; z < N; z++) b.e[z] = (z < n) ? src[z] : (T)0;
    }
}

// Region bookkeeping of a CTA depends only on which of i, j, k coincide and
// which sub-ranges coincide (4 x 4 patterns), so it is tabulated once on the
// host and read from constant memory.  For a pattern:
//   reg[pi*6 + rho]   region of (sub-range ordering pi, occupied ordering rho)
//   rep[g]            representative pi*6 + rho of region g (first in order)
//   combo[g][0..ncombo[g])  all pi*6 + rho of region g, ascending
//   sof[pi*6 + rho]   the ordering s with perm_compose(s, rho) = pi
struct F2Pattern {
    unsigned char nrole, npi;
    unsigned char reg[36];
    unsigned char rep[36];
    unsigned char ncombo[36];
    unsigned char combo[36][36];
    unsigned char sof[36];
};
constexpr int kF2Patterns = 16;
__constant__ F2Pattern c_f2pat[kF2Patterns];

// pattern index: 4 * (i==j==k ? 3 : i==j ? 1 : j==k ? 2 : 0) + (sub-ranges likewise)
__host__ __device__ inline int f2_pattern_index(int i, int j, int k, int a, int b, int c) {
    const int pij = (i == k) ? 3 : (i == j ? 1 : (j == k ? 2 : 0));
    const int pab = (a == c) ? 3 : (a == b ? 1 : (b == c ? 2 : 0));
    return 4 * pij + pab;
}

inline void f2_build_patterns(F2Pattern out[kF2Patterns]) {
    const int vals[4][3] = {{2, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0}};
    for (int pij = 0; pij < 4; pij++)
        for (int pab = 0; pab < 4; pab++) {
            F2Pattern &T = out[4 * pij + pab];
            const int *ijk = vals[pij], *st = vals[pab];
            auto same = [&](const int *val, int ra, int rb) {
                int qa[3], qb[3];
                perm_of(ra, qa);
                perm_of(rb, qb);
                return val[qa[0]] == val[qb[0]] && val[qa[1]] == val[qb[1]] && val[qa[2]] == val[qb[2]];
            };
            // dense index of an ordering among the distinct orderings (first occurrence order)
            auto dense = [&](const int *val, int r, int &count) {
                int first_at = r;
                for (int r2 = 5; r2 >= 0; r2--)
                    if (same(val, r2, r)) first_at = r2;
                int id = 0;
                count = 0;
                for (int r2 = 0; r2 < 6; r2++) {
                    bool first = true;
                    for (int r3 = 0; r3 < r2; r3++)
                        if (same(val, r2, r3)) first = false;
                    if (first) {
                        count++;
                        if (r2 < first_at) id++;
                    }
                }
                return id;
            };
            int nrole = 0, npi = 0;
            for (int t = 0; t < 36; t++) {
                const int pi = t / 6, rho = t % 6;
                const int rid = dense(ijk, rho, nrole), pid = dense(st, pi, npi);
                T.reg[t] = (unsigned char)(pid * nrole + rid);
                for (int s2 = 0; s2 < 6; s2++)
                    if (perm_compose(s2, rho) == pi) T.sof[t] = (unsigned char)s2;
            }
            T.nrole = (unsigned char)nrole;
            T.npi = (unsigned char)npi;
            for (int g = 0; g < 36; g++) {
                T.ncombo[g] = 0;
                T.rep[g] = 0;
            }
            for (int t = 0; t < 36; t++) {
                const int g = T.reg[t];
                if (T.ncombo[g] == 0) T.rep[g] = (unsigned char)t;
                T.combo[g][T.ncombo[g]++] = (unsigned char)t;
            }
        }
}

// Sum NV (power of two) per-lane values over aligned groups of G lanes
// (NV <= G <= 32, G a power of two); afterwards lane l holds the group total
// of value (l % NV).
template <int NV, int G, typename T>
__device__ __forceinline__ T group_reduce_scatter(T (&v)[NV], int lane) {
#pragma unroll
    for (int h = NV / 2; h >= 1; h /= 2) {
        const bool up = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const T send = up ? v[i] : v[i + h];
            const T keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    T r = v[0];
#pragma unroll
    for (int h = NV; h < G; h *= 2) r += __shfl_xor_sync(0xffffffffu, r, h);
    return r;
}

// BATCH = false: the CTAs of one launch segment (parameters P0).  BATCH =
// true: the CTAs of njobs segments (chunks of different problems) numbered job
// after job (job_start[j] = first CTA of job j), parameters in device memory.
template <typename StageT, int SB, bool BATCH>
__global__ void __launch_bounds__(F2Smem<SB>::NT, (SB == 8) ? 2 : 4)
    k_f2t(const __grid_constant__ F2P<StageT> P0, const F2P<StageT> *__restrict__ jobs,
          const int *__restrict__ job_start, int njobs) {
    int blk = (int)blockIdx.x;
    const F2P<StageT> *Pp = &P0;
    if constexpr (BATCH) {
        int lo = 0, hi = njobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (job_start[mid] <= blk) lo = mid;
            else hi = mid - 1;
        }
        blk -= job_start[lo];
        Pp = &jobs[lo];
    }
    const F2P<StageT> &P = *Pp;
    using C = F2Smem<SB>;
    constexpr int NT = C::NT, IPT = C::IPT;
    constexpr int REG = C::REG, NV = C::NV, NVP = C::NVP;
    constexpr int SX = C::SX, SY = C::SY;
    constexpr int REGW = C::REGW, SYW = C::SYW;
    constexpr int NW = NT / 32;
    extern __shared__ __align__(16) uint8_t f2_smem[];
    StageT *sW = reinterpret_cast<StageT *>(f2_smem);
    StageT *sG = sW;                      // item results [12][REG] (padded) once W is consumed
    StageT *tOV = sW + 36 * REGW;
    StageT *tT2 = tOV + C::TAB;
    StageT *tT1 = tT2 + C::TAB;
    StageT *tFV = tT1 + 3 * NV;
    __shared__ double s_ev[NV];
    __shared__ double s_red[2][NW];
    __shared__ int s_rd[36][9];               // per region: pi, rho, tau, lx, ly, lz, p, q, r
    __shared__ long long s_gb[36], s_wb[36];  // staging / Wbar base offsets of each region
    __shared__ int s_gs[36][2], s_ws[36][2];  // (y, x) strides in staging / Wbar

    const Dims &d = P.d;
    const int o = d.o, v = d.v;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // linear grid, sub-range triple fastest: the blocks of one representative
    // run together, so the two 16-byte halves of each Wbar sector meet in L2
    const int sub = P.sub0 + (int)((unsigned)blk % (unsigned)P.nsub_l);
    const int rep = P.rep0 + (int)((unsigned)blk / (unsigned)P.nsub_l);
    const F2Sub &R = P.sub[sub];
    const int ijk[3] = {P.ijk[3 * rep], P.ijk[3 * rep + 1], P.ijk[3 * rep + 2]};

    // canonical sub-range slot of each role (identical ranges share a slot)
    int cs[3];
    cs[0] = 0;
    cs[1] = (R.st[1] == R.st[0]) ? 0 : 1;
    cs[2] = (R.st[2] == R.st[1]) ? cs[1] : ((R.st[2] == R.st[0]) ? 0 : 2);
    const F2Pattern &pat = c_f2pat[f2_pattern_index(ijk[0], ijk[1], ijk[2], R.st[0], R.st[1], R.st[2])];
    const int nreg = pat.nrole * pat.npi;
    for (int e = tid; e < NV; e += NT) s_ev[e] = 0.0;

    // region descriptors; find the staging ordering tau of a sub-range ordering
    auto block_of = [&](int start) {
        for (int t = 0; t < 3; t++)
            if (start >= P.ch.base[t] && start < P.ch.base[t] + P.ch.nabc[t]) return P.ch.blk[t];
        return -1;
    };
    auto tau_of = [&](int pi) {
        int pp[3];
        perm_of(pi, pp);
        const int bx = block_of(R.st[pp[0]]), by = block_of(R.st[pp[1]]), bz = block_of(R.st[pp[2]]);
        int t = 0;
        for (; t < P.ch.nperm - 1; t++)
            if (P.ch.pb[t].bx == bx && P.ch.pb[t].by == by && P.ch.pb[t].bz == bz) break;
        return t;
    };
    if (tid < nreg) {
        const int pi = pat.rep[tid] / 6, rho = pat.rep[tid] % 6;
        int pp[3], pr[3];
        perm_of(pi, pp);
        perm_of(rho, pr);
        const int tau = tau_of(pi);
        const int p = pr[0] == 0 ? ijk[0] : (pr[0] == 1 ? ijk[1] : ijk[2]);
        const int q = pr[1] == 0 ? ijk[0] : (pr[1] == 1 ? ijk[1] : ijk[2]);
        const int r = pr[2] == 0 ? ijk[0] : (pr[2] == 1 ? ijk[1] : ijk[2]);
        int *rd = s_rd[tid];
        rd[0] = pi;
        rd[1] = rho;
        rd[2] = tau;
        rd[3] = R.len[pp[0]];
        rd[4] = R.len[pp[1]];
        rd[5] = R.len[pp[2]];
        rd[6] = p;
        rd[7] = q;
        rd[8] = r;
        const PermBlock &pb = P.ch.pb[tau];
        const int xs = R.st[pp[0]] - pb.X0, ys = R.st[pp[1]] - pb.Y0, zs = R.st[pp[2]] - pb.Z0;
        // staging S_tau[p][q][y][x][r][z]
        const long long gy = (long long)pb.Tx * o * pb.Tz, gx = (long long)o * pb.Tz;
        s_gb[tid] = pb.soff + (long long)(p * o + q) * pb.Ty * gy + ys * gy + xs * gx + (long long)r * pb.Tz + zs;
        s_gs[tid][0] = (int)gy;
        s_gs[tid][1] = (int)gx;
        // Wbar_tau[y][p][x][q][rzp]
        const long long wx = (long long)o * pb.rzp, wy = (long long)o * pb.Tx * wx;
        s_wb[tid] = (long long)ys * wy + (long long)p * pb.Tx * wx + xs * wx + (long long)q * pb.rzp + (long long)r * pb.Tz + zs;
        s_ws[tid][0] = (int)wy;
        s_ws[tid][1] = (int)wx;
    }
    __syncthreads();

    // ---- load the distinct regions, one (y, x) run of z values per thread step;
    //      LB runs are fetched before any is stored, so their latencies overlap ----
    // distinct sub-ranges: the tables need only the blocks of two different ranges
    const bool distinct_rng = (cs[1] == 1 && cs[2] == 2);
    if constexpr (sizeof(StageT) == 4 && SB == 8) {
        // FP32 staging: four lanes per 32-byte run, 8-byte cp.async (two 4-byte
        // copies where the run is not 8-byte aligned), zero-filled past the run
        const uint64_t pol = f2_policy_evict_first();
        const int npiece = nreg * SB * SB * 4;
        for (int e = tid; e < npiece; e += NT) {
            const int run = e >> 2, c = e & 3;
            const int reg = run / (SB * SB), yy = (run / SB) % SB, xx = run % SB;
            const int *rd = s_rd[reg];
            if (xx < rd[3] && yy < rd[4]) {
                const int n = rd[5] - 2 * c;   // valid values of this 2-value piece (<= 0: none)
                const StageT *run0 = P.S + s_gb[reg] + (long long)yy * s_gs[reg][0] + (long long)xx * s_gs[reg][1];
                const StageT *src = n > 0 ? run0 + 2 * c : run0;   // nothing is read when n <= 0
                StageT *dst = sW + reg * REGW + yy * SYW + xx * SX + 2 * c;
                if (n >= 2 && (reinterpret_cast<uintptr_t>(src) & 7) == 0) {
                    f2_cp_async(dst, src, 8, 8, pol);
                } else {
                    f2_cp_async(dst, src, 4, n >= 1 ? 4 : 0, pol);
                    f2_cp_async(dst + 1, n >= 2 ? src + 1 : src, 4, n >= 2 ? 4 : 0, pol);
                }
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    } else {
        constexpr int LB = 3;
        const int nrun = nreg * SB * SB;
        for (int e0 = tid; e0 < nrun; e0 += LB * NT) {
            RunBuf<StageT, SB> b[LB];
            StageT *dst[LB];
            int lzs[LB];
#pragma unroll
            for (int u = 0; u < LB; u++) {
                const int e = e0 + u * NT;
                dst[u] = nullptr;
                lzs[u] = 0;
                if (e < nrun) {
                    const int reg = e / (SB * SB), yy = (e / SB) % SB, xx = e % SB;
                    const int *rd = s_rd[reg];
                    if (xx < rd[3] && yy < rd[4]) {
                        lzs[u] = rd[5];
                        ld_run(b[u], P.S + s_gb[reg] + (long long)yy * s_gs[reg][0] + (long long)xx * s_gs[reg][1],
                               lzs[u]);
                        dst[u] = sW + reg * REGW + yy * SYW + xx * SX;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < LB; u++)
                if (dst[u] != nullptr) {
#pragma unroll
                    for (int zz = 0; zz < SB; zz++)
                        if (zz < lzs[u]) dst[u][zz] = b[u].e[zz];
                }
        }
    }
    // ---- tables for the V terms (TB entries fetched per batch) ----
    {
        constexpr int TB = 4;
        for (int e0 = tid; e0 < 6 * NV * NV; e0 += TB * NT) {
            double ov[TB], tt[TB];
            int te[TB];
#pragma unroll
            for (int u = 0; u < TB; u++) {
                const int e = e0 + u * NT;
                ov[u] = tt[u] = 0.0;
                te[u] = -1;
                if (e < 6 * NV * NV) {
                    const int pair = e / (NV * NV), xl = (e / NV) % NV, yl = e % NV;
                    te[u] = (pair * NV + xl) * NVP + yl;
                    const int sp = pair / 2, rem = pair % 2;
                    const int sq = (rem < sp) ? rem : rem + 1;   // inverse of pair_index
                    const int sx = xl / SB, sy = yl / SB;
                    if (xl % SB < R.len[sx] && yl % SB < R.len[sy] && !(distinct_rng && sx == sy)) {
                        const int x = R.st[sx] + xl % SB, y = R.st[sy] + yl % SB;
                        const int p = (sp == 0) ? ijk[0] : (sp == 1 ? ijk[1] : ijk[2]);
                        const int q = (sq == 0) ? ijk[0] : (sq == 1 ? ijk[1] : ijk[2]);
                        ov[u] = P.ovov[(((long long)p * v + x) * o + q) * v + y];
                        tt[u] = P.t2[(((long long)q * o + p) * v + y) * v + x];
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < TB; u++)
                if (te[u] >= 0) {
                    tOV[te[u]] = (StageT)ov[u];
                    tT2[te[u]] = (StageT)tt[u];
                }
        }
    }
    for (int e = tid; e < 3 * NV; e += NT) {
        const int sr = e / NV, zl = e % NV, sz = zl / SB;
        StageT a1 = 0, f1 = 0;
        if (zl % SB < R.len[sz]) {
            const int z = R.st[sz] + zl % SB, r = (sr == 0) ? ijk[0] : (sr == 1 ? ijk[1] : ijk[2]);
            a1 = (StageT)P.t1[(long long)r * v + z];
            f1 = (StageT)P.fvo[(long long)z * o + r];
        }
        tT1[e] = a1;
        tFV[e] = f1;
    }
    __syncthreads();

    // ---- orbit items (IPT per thread) ----
    const int i = ijk[0], j = ijk[1], k = ijk[2];
    const int n_ijk = (i == k) ? 1 : ((i == j || j == k) ? 3 : 6);
    const double e_ijk = P.mo_e[i] + P.mo_e[j] + P.mo_e[k];
    double e_loc = 0.0, dd_loc = 0.0;
    StageT gres[IPT][12];
    bool gvalid[IPT];
#pragma unroll
    for (int it = 0; it < IPT; it++) {
        const int item = tid + it * NT;
        const int loc[3] = {item / (SB * SB), (item / SB) % SB, item % SB};
        bool valid = loc[0] < R.len[0] && loc[1] < R.len[1] && loc[2] < R.len[2];
        const int abc[3] = {R.st[0] + loc[0], R.st[1] + loc[1], R.st[2] + loc[2]};
        if (valid && cs[1] == 0 && abc[0] < abc[1]) valid = false;
        if (valid && cs[2] == cs[1] && abc[1] < abc[2]) valid = false;
        gvalid[it] = valid;
        double ddi = 0.0;
        if (valid) {
            const int vl[3] = {cs[0] * SB + loc[0], cs[1] * SB + loc[1], cs[2] * SB + loc[2]};
            double WW[6], X[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                double sw = 0.0;
                StageT sv = 0;   // V term: products of staged (StageT) factors
#pragma unroll
                for (int tau = 0; tau < 6; tau++) {
                    const int pi = perm_compose(s, tau);
                    int pp[3], pt[3];
                    perm_of(pi, pp);
                    perm_of(tau, pt);
                    sw += (double)sW[pat.reg[pi * 6 + tau] * REGW + loc[pp[1]] * SYW + loc[pp[0]] * SX + loc[pp[2]]];
                    const int pair = pair_index(pt[0], pt[1]);
                    const int xl = vl[pp[0]], yl = vl[pp[1]], zl = vl[pp[2]];
                    sv += tOV[(pair * NV + xl) * NVP + yl] * tT1[pt[2] * NV + zl] +
                          tT2[(pair * NV + xl) * NVP + yl] * tFV[pt[2] * NV + zl];
                }
                WW[s] = sw;
                X[s] = sw + 0.5 * (double)sv;
            }
            double Z[6], RW[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                Z[s] = 4.0 * X[s] + X[perm_compose(s, 4)] + X[perm_compose(s, 3)] -
                       2.0 * (X[perm_compose(s, 5)] + X[perm_compose(s, 1)] + X[perm_compose(s, 2)]);
                RW[s] = 4.0 * WW[s] + WW[perm_compose(s, 4)] + WW[perm_compose(s, 3)] -
                        2.0 * (WW[perm_compose(s, 5)] + WW[perm_compose(s, 1)] + WW[perm_compose(s, 2)]);
            }
            const int n_abc = (abc[0] == abc[2]) ? 1 : ((abc[0] == abc[1] || abc[1] == abc[2]) ? 3 : 6);
            const double cfac = (double)(n_ijk * n_abc) / 18.0;
            const double Dn = e_ijk - P.mo_e[o + abc[0]] - P.mo_e[o + abc[1]] - P.mo_e[o + abc[2]];
            const double rD = 1.0 / Dn;
            double esum = 0.0;
#pragma unroll
            for (int s = 0; s < 6; s++) esum += WW[s] * Z[s];
            e_loc += cfac * esum * rD;
            if (P.want_grad) {
                const double g0 = P.ybar * cfac * rD;
                ddi = -P.ybar * cfac * esum * rD * rD;
#pragma unroll
                for (int s = 0; s < 6; s++) {
                    gres[it][s] = (StageT)(g0 * (Z[s] + RW[s]));
                    gres[it][6 + s] = (StageT)(g0 * 0.5 * RW[s]);
                }
                if (SB * SB < 32) atomicAdd(&s_ev[vl[0]], -ddi);
                atomicAdd(&s_ev[vl[1]], -ddi);
                atomicAdd(&s_ev[vl[2]], -ddi);
            }
        }
        dd_loc += ddi;
        // with SB^2 >= 32 the a-slot index (item / SB^2) is uniform across a warp: reduce first
        if (SB * SB >= 32 && P.want_grad) {
            double dsum = -ddi;
            for (int off = 16; off > 0; off >>= 1) dsum += __shfl_down_sync(0xffffffffu, dsum, off);
            const int la = item / (SB * SB);
            if (lane == 0 && la < R.len[0] && dsum != 0.0) atomicAdd(&s_ev[cs[0] * SB + la], dsum);
        }
    }

    // ---- block reductions: chunk energy partial, occupied-energy gradient ----
    for (int off = 16; off > 0; off >>= 1) {
        e_loc += __shfl_down_sync(0xffffffffu, e_loc, off);
        dd_loc += __shfl_down_sync(0xffffffffu, dd_loc, off);
    }
    if (lane == 0) {
        s_red[0][warp] = e_loc;
        s_red[1][warp] = dd_loc;
    }
    __syncthreads();   // all reads of the W tile are done: it becomes the item-result buffer
    if (tid == 0) {
        double es = 0.0, ds = 0.0;
        for (int w = 0; w < NW; w++) {
            es += s_red[0][w];
            ds += s_red[1][w];
        }
        P.e_part[(long long)sub * P.n_ijk + rep] = es;
        if (P.want_grad && ds != 0.0) {
            atomicAdd(&P.mo_bar[ijk[0]], ds);
            atomicAdd(&P.mo_bar[ijk[1]], ds);
            atomicAdd(&P.mo_bar[ijk[2]], ds);
        }
    }
    if (!P.want_grad) return;
#pragma unroll
    for (int it = 0; it < IPT; it++)
        if (gvalid[it]) {
            const int item = tid + it * NT;
            // item (l0, l1, l2) at l0*SY + l1*SX + l2 in each of the 12 planes: the
            // padded strides keep the write-back gathers within 2-way bank conflicts
            const int gi = (item / (SB * SB)) * SY + ((item / SB) % SB) * SX + item % SB;
#pragma unroll
            for (int c = 0; c < 12; c++) sG[c * REG + gi] = gres[it][c];
        }
    __syncthreads();
    for (int e = tid; e < NV; e += NT) {
        const int sl = e / SB, l = e % SB;
        if (l < R.len[sl] && s_ev[e] != 0.0) atomicAdd(&P.mo_bar[o + R.st[sl] + l], s_ev[e]);
    }

    // ---- write back Wbar; V-term gradients from the run's Vbar ----
    // A group of GL lanes takes whole regions (RPL runs of z values per lane),
    // so the columns (r, z) of the t1 / fvo sums are fixed per group and the
    // column partials of all its runs are reduced once per region.
    constexpr int RPR = SB * SB;                 // runs per region
    constexpr int GL = RPR < 32 ? RPR : 32;      // lanes per region group
    constexpr int RPL = RPR / GL;                // runs per lane
    constexpr int NG = NT / GL;                  // groups per CTA
    // every region holds one (pi, rho) pair and no ordering constraint applies
    const bool simple = (n_ijk == 6) && distinct_rng;
    const float wscf = (P.split != 0) ? (float)*P.wscale : 1.0f;
    const int grp = tid / GL, gl = tid % GL;
    const int nround = (nreg + NG - 1) / NG;
    for (int rr = 0; rr < nround; rr++) {
        const int reg_ = grp + rr * NG;
        const bool inrange = reg_ < nreg;
        const int reg = inrange ? reg_ : 0;
        const int *rd = s_rd[reg];
        const int lx = rd[3], ly = rd[4], lz = rd[5];
        int pp[3], pt[3];
        perm_of(rd[0], pp);
        perm_of(rd[1], pt);
        auto cslot = [&](int j) { return j == 0 ? cs[0] : (j == 1 ? cs[1] : cs[2]); };
        auto stride = [&](int j) { return j == 0 ? SY : (j == 1 ? SX : 1); };   // item-result layout
        const int zl0 = cslot(pp[2]) * SB;
        const int p = rd[6], q = rd[7], r = rd[8];
        const int pair = pair_index(pt[0], pt[1]);
        const StageT *a1 = tT1 + pt[2] * NV + zl0, *f1 = tFV + pt[2] * NV + zl0;
        const PermBlock &pb = P.ch.pb[rd[2]];
        const long long half = (long long)pb.Ty * o * pb.Tx * o * pb.rzp;
        // V-term partials in the staging precision (FP32 in the mixed modes: 8-term
        // row sums and the warp's 64-run column sums), added to the FP64 gradients
        StageT colv[2 * SB];
#pragma unroll
        for (int c = 0; c < 2 * SB; c++) colv[c] = 0;
#pragma unroll
        for (int u = 0; u < RPL; u++) {
            const int run = gl + u * GL;
            const int yy = run / SB, xx = run % SB;
            if (!(inrange && xx < lx && yy < ly)) continue;
            StageT wb[SB], vb[SB];
            if (simple) {
                const int s = pat.sof[rd[0] * 6 + rd[1]];
                const int base = xx * stride(pp[0]) + yy * stride(pp[1]), st2 = stride(pp[2]);
                const StageT *gw = sG + s * REG + base, *gv = sG + (6 + s) * REG + base;
#pragma unroll
                for (int zz = 0; zz < SB; zz++) {
                    wb[zz] = (zz < lz) ? gw[zz * st2] : (StageT)0;
                    vb[zz] = (zz < lz) ? gv[zz * st2] : (StageT)0;
                }
            } else {
                double wd[SB], vd[SB];   // several (s, tau) per position: sum in FP64
#pragma unroll
                for (int zz = 0; zz < SB; zz++) wd[zz] = vd[zz] = 0.0;
                const int nc = pat.ncombo[reg];
                for (int c = 0; c < nc; c++) {
                    const int pr = pat.combo[reg][c];
                    const int s = pat.sof[pr];
                    int q3[3];
                    perm_of(pr / 6, q3);
                    // item slot j takes the region coordinate whose ordering slot is j
                    const int base = xx * stride(q3[0]) + yy * stride(q3[1]), st2 = stride(q3[2]);
                    const StageT *gw = sG + s * REG, *gv = sG + (6 + s) * REG;
#pragma unroll
                    for (int zz = 0; zz < SB; zz++) {
                        if (zz >= lz) continue;
                        const int l0 = (q3[0] == 0) ? xx : ((q3[1] == 0) ? yy : zz);
                        const int l1 = (q3[0] == 1) ? xx : ((q3[1] == 1) ? yy : zz);
                        const int l2 = (q3[0] == 2) ? xx : ((q3[1] == 2) ? yy : zz);
                        bool ok = true;
                        if (cs[1] == 0 && l0 < l1) ok = false;
                        if (cs[2] == cs[1] && l1 < l2) ok = false;
                        if (ok) {
                            const int item = base + zz * st2;
                            wd[zz] += (double)gw[item];
                            vd[zz] += (double)gv[item];
                        }
                    }
                }
#pragma unroll
                for (int zz = 0; zz < SB; zz++) {
                    wb[zz] = (StageT)wd[zz];
                    vb[zz] = (StageT)vd[zz];
                }
            }
            // Wbar out
            const long long wl = s_wb[reg] + (long long)yy * s_ws[reg][0] + (long long)xx * s_ws[reg][1];
            if (P.split == 0) {
                RunBuf<StageT, SB> bw;
#pragma unroll
                for (int zz = 0; zz < SB; zz++) bw.e[zz] = (StageT)wb[zz];
                st_run(reinterpret_cast<StageT *>(P.SW) + pb.swoff + wl, bw, lz);
            } else if (P.split == 1) {
                // exact power-of-two scaling, then a two-term 16-bit split in FP32
                RunBuf<__half, SB> bh, bl;
#pragma unroll
                for (int zz = 0; zz < SB; zz++) {
                    const float xs = (float)wb[zz] * wscf;
                    bh.e[zz] = __float2half_rn(xs);
                    bl.e[zz] = __float2half_rn(xs - __half2float(bh.e[zz]));
                }
                __half *dst = reinterpret_cast<__half *>(P.SW) + 2 * pb.swoff + wl;
                st_run(dst, bh, lz);
                st_run(dst + half, bl, lz);
            } else {
                RunBuf<__nv_bfloat16, SB> bh, bl;
#pragma unroll
                for (int zz = 0; zz < SB; zz++) {
                    const float xs = (float)wb[zz] * wscf;
                    bh.e[zz] = __float2bfloat16_rn(xs);
                    bl.e[zz] = __float2bfloat16_rn(xs - __bfloat162float(bh.e[zz]));
                }
                __nv_bfloat16 *dst = reinterpret_cast<__nv_bfloat16 *>(P.SW) + 2 * pb.swoff + wl;
                st_run(dst, bh, lz);
                st_run(dst + half, bl, lz);
            }
            // V-term gradients: v = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r]
            const int x = R.st[pp[0]] + xx, y = R.st[pp[1]] + yy;
            const int te = (pair * NV + cslot(pp[0]) * SB + xx) * NVP + cslot(pp[1]) * SB + yy;
            const StageT ovv = tOV[te], t2v = tT2[te];
            StageT rs1 = 0, rs2 = 0;
#pragma unroll
            for (int zz = 0; zz < SB; zz++) {
                rs1 += vb[zz] * a1[zz];
                rs2 += vb[zz] * f1[zz];
                colv[zz] += vb[zz] * ovv;
                colv[SB + zz] += vb[zz] * t2v;
            }
            atomicAdd(&P.ovov_bar[(((long long)p * v + x) * o + q) * v + y], (double)rs1);
            atomicAdd(&P.t2_bar[(((long long)q * o + p) * v + y) * v + x], (double)rs2);
        }
        // column sums over the region's runs: t1_bar[r, z], fvo_bar[z, r]
        const double cv = (double)group_reduce_scatter<2 * SB, GL>(colv, lane);
        const int cidx = lane % (2 * SB);
        if (inrange && gl < 2 * SB && (cidx % SB) < lz && cv != 0.0) {
            const int z = R.st[pp[2]] + cidx % SB;
            if (cidx < SB) atomicAdd(&P.t1_bar[(long long)r * v + z], cv);
            else atomicAdd(&P.fvo_bar[(long long)z * o + r], cv);
        }
    }
}

// Sum of the per-CTA energy partials of one epilogue launch, in a fixed order.
__device__ __forceinline__ void energy_sum_body(const double *__restrict__ e_part, int n, double *e_acc) {
    __shared__ double s[256];
    double acc = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) acc += e_part[b];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *e_acc += s[0];
}

__global__ void k_f2_energy_sum(const double *__restrict__ e_part, int n, double *e_acc) {
    energy_sum_body(e_part, n, e_acc);
}

}  // namespace tb

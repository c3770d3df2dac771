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
// Vbar overwrites W in place; Wbar goes to its own buffer in the layout the
// gradient contractions read: [h][y][p][x][q][r][z].
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
    StageT *S;          // W in, Vbar out; per ordering tau: [p][q][y][x][r][z] at ch.pb[tau].soff
    void *SW;           // Wbar out; per tau at 2*soff: [h][y][p][x][q][r][z] (split) or at soff: [y][p][x][q][r][z]
    int split;          // 0: StageT, 1: fp16 hi/lo, 2: bf16 hi/lo
    const double *wscale;
    double ybar;
    int want_grad;
    double *e_part, *e_acc;
    unsigned *counter;
    double *mo_bar;
};

template <int SB>
struct F2Smem {
    static constexpr int REG = SB * SB * SB;
    static constexpr int NV = 3 * SB;
    static constexpr int TAB = 6 * NV * NV;
};

template <typename StageT, int SB>
__host__ __device__ constexpr size_t f2_smem_bytes() {
    return sizeof(StageT) * (2 * 36 * F2Smem<SB>::REG + 2 * F2Smem<SB>::TAB + 2 * 3 * F2Smem<SB>::NV);
}

__device__ __forceinline__ int pair_index(int sp, int sq) { return 2 * sp + (sq > sp ? sq - 1 : sq); }

template <typename StageT, int SB>
__global__ void __launch_bounds__(SB *SB *SB) k_f2t(F2P<StageT> P) {
    constexpr int NT = SB * SB * SB;
    constexpr int REG = F2Smem<SB>::REG;
    constexpr int NV = F2Smem<SB>::NV;
    extern __shared__ __align__(16) uint8_t f2_smem[];
    StageT *sW = reinterpret_cast<StageT *>(f2_smem);
    StageT *sWb = sW + 36 * REG;
    StageT *tOV = sWb + 36 * REG;
    StageT *tT2 = tOV + F2Smem<SB>::TAB;
    StageT *tT1 = tT2 + F2Smem<SB>::TAB;
    StageT *tFV = tT1 + 3 * NV;
    __shared__ double s_ev[NV];
    __shared__ double s_red[2][NT / 32 > 0 ? NT / 32 : 1];
    __shared__ int s_reg[6][6];     // [ordering pi][role rho] -> region
    __shared__ int s_rd[36][9];     // per region: pi, rho, tau, lx, ly, lz, p, q, r
    __shared__ int s_ntile[2];

    const Dims &d = P.d;
    const int o = d.o, v = d.v;
    const int tid = threadIdx.x;
    const int rep = blockIdx.x;
    const F2Sub &R = P.sub[blockIdx.y];
    const int ijk[3] = {P.ijk[3 * rep], P.ijk[3 * rep + 1], P.ijk[3 * rep + 2]};

    // canonical sub-range slot of each role (identical ranges share a slot)
    int cs[3];
    cs[0] = 0;
    cs[1] = (R.st[1] == R.st[0]) ? 0 : 1;
    cs[2] = (R.st[2] == R.st[1]) ? cs[1] : ((R.st[2] == R.st[0]) ? 0 : 2);

    if (tid == 0) {
        // distinct occupied orderings and distinct sub-range orderings
        int rid[6], pid[6], nrole = 0, npi = 0;
        for (int rho = 0; rho < 6; rho++) {
            int pr[3];
            perm_of(rho, pr);
            rid[rho] = -1;
            for (int r2 = 0; r2 < rho; r2++) {
                int q2[3];
                perm_of(r2, q2);
                if (ijk[pr[0]] == ijk[q2[0]] && ijk[pr[1]] == ijk[q2[1]] && ijk[pr[2]] == ijk[q2[2]]) {
                    rid[rho] = rid[r2];
                    break;
                }
            }
            if (rid[rho] < 0) rid[rho] = nrole++;
        }
        for (int pi = 0; pi < 6; pi++) {
            int pp[3];
            perm_of(pi, pp);
            pid[pi] = -1;
            for (int p2 = 0; p2 < pi; p2++) {
                int q2[3];
                perm_of(p2, q2);
                if (R.st[pp[0]] == R.st[q2[0]] && R.st[pp[1]] == R.st[q2[1]] && R.st[pp[2]] == R.st[q2[2]]) {
                    pid[pi] = pid[p2];
                    break;
                }
            }
            if (pid[pi] < 0) pid[pi] = npi++;
        }
        for (int pi = 0; pi < 6; pi++)
            for (int rho = 0; rho < 6; rho++) s_reg[pi][rho] = pid[pi] * nrole + rid[rho];
        s_ntile[0] = nrole;
        s_ntile[1] = npi;
        for (int a = 35; a >= 0; a--) {   // first (pi, rho) of each region wins
            const int pi = a / 6, rho = a % 6, reg = s_reg[pi][rho];
            int pp[3], pr[3];
            perm_of(pi, pp);
            perm_of(rho, pr);
            s_rd[reg][0] = pi;
            s_rd[reg][1] = rho;
            s_rd[reg][3] = R.len[pp[0]];
            s_rd[reg][4] = R.len[pp[1]];
            s_rd[reg][5] = R.len[pp[2]];
            s_rd[reg][6] = ijk[pr[0]];
            s_rd[reg][7] = ijk[pr[1]];
            s_rd[reg][8] = ijk[pr[2]];
        }
    }
    for (int e = tid; e < NV; e += NT) s_ev[e] = 0.0;
    __syncthreads();
    const int nrole = s_ntile[0], npi = s_ntile[1];

    // region descriptors are recomputed per use from (pi, rho); find the
    // staging ordering tau of a sub-range ordering
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

    const int nreg = nrole * npi;
    if (tid < nreg) s_rd[tid][2] = tau_of(s_rd[tid][0]);
    __syncthreads();

    // ---- load the distinct regions: element (reg, yy, xx, zz) ----
    for (int e = tid; e < nreg * REG; e += NT) {
        const int reg = e / REG;
        const int zz = e % SB, xx = (e / SB) % SB, yy = (e / (SB * SB)) % SB;
        const int *rd = s_rd[reg];
        const int lx = rd[3], ly = rd[4], lz = rd[5];
        if (xx >= lx || yy >= ly || zz >= lz) continue;
        int pp[3];
        perm_of(rd[0], pp);
        const PermBlock &pb = P.ch.pb[rd[2]];
        const int p = rd[6], q = rd[7], r = rd[8];
        const int x = R.st[pp[0]] + xx, y = R.st[pp[1]] + yy, z = R.st[pp[2]] + zz;
        const long long g = pb.soff +
                            ((((long long)(p * o + q) * pb.Ty + (y - pb.Y0)) * pb.Tx + (x - pb.X0)) * o + r) *
                                pb.Tz +
                            (z - pb.Z0);
        sW[reg * REG + (yy * lx + xx) * lz + zz] = P.S[g];
    }
    // ---- tables for the V terms ----
    for (int e = tid; e < 6 * NV * NV; e += NT) {
        const int pair = e / (NV * NV), xl = (e / NV) % NV, yl = e % NV;
        const int sp = pair / 2, rem = pair % 2;
        const int sq = (rem < sp) ? rem : rem + 1;   // inverse of pair_index
        const int sx = xl / SB, sy = yl / SB;
        StageT ov = 0, tt = 0;
        if (xl % SB < R.len[sx] && yl % SB < R.len[sy]) {
            const int x = R.st[sx] + xl % SB, y = R.st[sy] + yl % SB;
            const int p = ijk[sp], q = ijk[sq];
            ov = (StageT)P.ovov[(((long long)p * v + x) * o + q) * v + y];
            tt = (StageT)P.t2[(((long long)q * o + p) * v + y) * v + x];
        }
        tOV[e] = ov;
        tT2[e] = tt;
    }
    for (int e = tid; e < 3 * NV; e += NT) {
        const int sr = e / NV, zl = e % NV, sz = zl / SB;
        StageT a1 = 0, f1 = 0;
        if (zl % SB < R.len[sz]) {
            const int z = R.st[sz] + zl % SB, r = ijk[sr];
            a1 = (StageT)P.t1[(long long)r * v + z];
            f1 = (StageT)P.fvo[(long long)z * o + r];
        }
        tT1[e] = a1;
        tFV[e] = f1;
    }
    __syncthreads();

    // ---- one orbit item per thread ----
    double e_loc = 0.0, dd_loc = 0.0;
    const int loc[3] = {tid / (SB * SB), (tid / SB) % SB, tid % SB};
    bool valid = loc[0] < R.len[0] && loc[1] < R.len[1] && loc[2] < R.len[2];
    const int abc[3] = {R.st[0] + loc[0], R.st[1] + loc[1], R.st[2] + loc[2]};
    if (valid && cs[1] == 0 && abc[0] < abc[1]) valid = false;
    if (valid && cs[2] == cs[1] && abc[1] < abc[2]) valid = false;
    if (valid) {
        const int vl[3] = {cs[0] * SB + loc[0], cs[1] * SB + loc[1], cs[2] * SB + loc[2]};
        double WW[6], X[6];
        int idx[6][6];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            double sw = 0.0, sv = 0.0;
#pragma unroll
            for (int tau = 0; tau < 6; tau++) {
                const int pi = perm_compose(s, tau);
                int pp[3], pt[3];
                perm_of(pi, pp);
                perm_of(tau, pt);
                const int lx = R.len[pp[0]], lz = R.len[pp[2]];
                const int id = s_reg[pi][tau] * REG + (loc[pp[1]] * lx + loc[pp[0]]) * lz + loc[pp[2]];
                idx[s][tau] = id;
                sw += (double)sW[id];
                const int pair = pair_index(pt[0], pt[1]);
                const int xl = vl[pp[0]], yl = vl[pp[1]], zl = vl[pp[2]];
                sv += (double)tOV[(pair * NV + xl) * NV + yl] * (double)tT1[pt[2] * NV + zl] +
                      (double)tT2[(pair * NV + xl) * NV + yl] * (double)tFV[pt[2] * NV + zl];
            }
            WW[s] = sw;
            X[s] = sw + 0.5 * sv;
        }
        double Z[6], RW[6];
#pragma unroll
        for (int s = 0; s < 6; s++) {
            Z[s] = 4.0 * X[s] + X[perm_compose(s, 4)] + X[perm_compose(s, 3)] -
                   2.0 * (X[perm_compose(s, 5)] + X[perm_compose(s, 1)] + X[perm_compose(s, 2)]);
            RW[s] = 4.0 * WW[s] + WW[perm_compose(s, 4)] + WW[perm_compose(s, 3)] -
                    2.0 * (WW[perm_compose(s, 5)] + WW[perm_compose(s, 1)] + WW[perm_compose(s, 2)]);
        }
        const int i = ijk[0], j = ijk[1], k = ijk[2];
        const int n_ijk = (i == k) ? 1 : ((i == j || j == k) ? 3 : 6);
        const int n_abc = (abc[0] == abc[2]) ? 1 : ((abc[0] == abc[1] || abc[1] == abc[2]) ? 3 : 6);
        const double cfac = (double)(n_ijk * n_abc) / 18.0;
        const double Dn = P.mo_e[i] + P.mo_e[j] + P.mo_e[k] - P.mo_e[o + abc[0]] - P.mo_e[o + abc[1]] -
                          P.mo_e[o + abc[2]];
        const double rD = 1.0 / Dn;
        double esum = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) esum += WW[s] * Z[s];
        e_loc = cfac * esum * rD;
        if (P.want_grad) {
            const double g0 = P.ybar * cfac * rD;
            const double dD = -P.ybar * cfac * esum * rD * rD;
            dd_loc = dD;
#pragma unroll
            for (int s = 0; s < 6; s++)
#pragma unroll
                for (int tau = 0; tau < 6; tau++) {
                    sW[idx[s][tau]] = (StageT)0;
                    sWb[idx[s][tau]] = (StageT)0;
                }
#pragma unroll
            for (int s = 0; s < 6; s++) {
                const StageT gw = (StageT)(g0 * (Z[s] + RW[s]));
                const StageT gv = (StageT)(g0 * 0.5 * RW[s]);
#pragma unroll
                for (int tau = 0; tau < 6; tau++) {
                    sWb[idx[s][tau]] += gw;
                    sW[idx[s][tau]] += gv;
                }
            }
            atomicAdd(&s_ev[vl[0]], -dD);
            atomicAdd(&s_ev[vl[1]], -dD);
            atomicAdd(&s_ev[vl[2]], -dD);
        }
    }

    // ---- block reductions ----
    for (int off = 16; off > 0; off >>= 1) {
        e_loc += __shfl_down_sync(0xffffffffu, e_loc, off);
        dd_loc += __shfl_down_sync(0xffffffffu, dd_loc, off);
    }
    if ((tid & 31) == 0) {
        s_red[0][tid >> 5] = e_loc;
        s_red[1][tid >> 5] = dd_loc;
    }
    __syncthreads();
    if (tid == 0) {
        double es = 0.0, ds = 0.0;
        for (int w = 0; w < (NT + 31) / 32; w++) {
            es += s_red[0][w];
            ds += s_red[1][w];
        }
        P.e_part[blockIdx.y * gridDim.x + blockIdx.x] = es;
        if (P.want_grad && ds != 0.0) {
            atomicAdd(&P.mo_bar[ijk[0]], ds);
            atomicAdd(&P.mo_bar[ijk[1]], ds);
            atomicAdd(&P.mo_bar[ijk[2]], ds);
        }
    }

    if (P.want_grad) {
        for (int e = tid; e < NV; e += NT) {
            const int sl = e / SB, l = e % SB;
            if (l < R.len[sl] && s_ev[e] != 0.0) atomicAdd(&P.mo_bar[o + R.st[sl] + l], s_ev[e]);
        }
        // ---- write back: Vbar in place, Wbar to its buffer ----
        const double wsc = (P.split != 0) ? *P.wscale : 1.0;
        for (int e = tid; e < nreg * REG; e += NT) {
            const int reg = e / REG;
            const int zz = e % SB, xx = (e / SB) % SB, yy = (e / (SB * SB)) % SB;
            const int *rd = s_rd[reg];
            const int lx = rd[3], ly = rd[4], lz = rd[5];
            if (xx >= lx || yy >= ly || zz >= lz) continue;
            int pp[3];
            perm_of(rd[0], pp);
            const PermBlock &pb = P.ch.pb[rd[2]];
            const int p = rd[6], q = rd[7], r = rd[8];
            const int xl = R.st[pp[0]] + xx - pb.X0, yl = R.st[pp[1]] + yy - pb.Y0, zl = R.st[pp[2]] + zz - pb.Z0;
            const int si = reg * REG + (yy * lx + xx) * lz + zz;
            const long long g = pb.soff + ((((long long)(p * o + q) * pb.Ty + yl) * pb.Tx + xl) * o + r) * pb.Tz + zl;
            P.S[g] = sW[si];
            const long long wl =
                ((((long long)yl * o + p) * pb.Tx + xl) * o + q) * pb.rzp + (long long)r * pb.Tz + zl;
            const double wb = (double)sWb[si];
            if (P.split == 0) {
                reinterpret_cast<StageT *>(P.SW)[pb.swoff + wl] = sWb[si];
            } else {
                const long long half = (long long)pb.Ty * o * pb.Tx * o * pb.rzp;
                const double xs = wb * wsc;
                if (P.split == 1) {
                    __half *dst = reinterpret_cast<__half *>(P.SW) + 2 * pb.swoff;
                    const __half hi = __double2half(xs);
                    dst[wl] = hi;
                    dst[half + wl] = __double2half(xs - (double)__half2float(hi));
                } else {
                    __nv_bfloat16 *dst = reinterpret_cast<__nv_bfloat16 *>(P.SW) + 2 * pb.swoff;
                    const __nv_bfloat16 hi = __double2bfloat16(xs);
                    dst[wl] = hi;
                    dst[half + wl] = __double2bfloat16(xs - (double)__bfloat162float(hi));
                }
            }
        }
    }

    // ---- deterministic chunk energy: the last CTA sums the partials in a fixed order ----
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (tid == 0) {
        const unsigned prev = atomicAdd(P.counter, 1u);
        s_last = (prev == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        const int nblk = gridDim.x * gridDim.y;
        double acc = 0.0;
        for (int b = tid; b < nblk; b += NT) acc += ((volatile double *)P.e_part)[b];
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        __syncthreads();
        if ((tid & 31) == 0) s_red[0][tid >> 5] = acc;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < (NT + 31) / 32; w++) tot += s_red[0][w];
            P.e_acc[0] += tot;
            *P.counter = 0u;
        }
    }
}

}  // namespace tb

// LNO (T): the triples energy with a projector on the first occupied index,
//   E = (1/3) sum_{ijk, abc} Wt[ijk,abc] Q[ijk,abc],
//   Wt[i..] = sum_l mat[l,i] WW[l..],   Q = r3(WW + VV/2) / D,
// the energy of lnoccsdt_contract (pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c:6-29
// with the job weights of lno_ccsd_t.c:73-94 and the 2/3 of
// pyscfad/lno/ccsd_t.py:111; mat = identity gives the canonical E(T)), and
// its adjoint (lnoccsdt_energy_vjp, lno_ccsd_t_vjp.c:74-122 and 400-566):
//   Qbar = (ybar/3) Wt,   Wtbar = (ybar/3) Q,
//   mat_bar[l,i] = sum WW[l..] Wtbar[i..],
//   Zbar = Qbar / D,   Dbar = -Qbar Q / D,   Xbar = r3^T(Zbar),
//   WWbar = P^T(Wtbar) + Xbar,   VVbar = Xbar / 2,
//   wbar = sum_sigma WWbar(sigma pos),  vbar = sum_sigma VVbar(sigma pos).
//
// The projector couples all values of the first occupied index, which the
// canonical epilogue's orbit tiles keep apart, so one chunk takes four passes
// over FP64 work arrays in the staging layout (position = (tau; p, q, y, x,
// r, z), p outermost, "column" = everything after p):
//   1. tile forward  (orbit tiles in shared memory): WW -> B0, Q -> B2
//   2. projection    (streaming over columns, all p of a column in a tile):
//                    energy; with the adjoint also mat_bar, Dbar -> B2 (over Q),
//                    Zbar -> B3 and P^T(Wtbar) -> B1
//   3. tile adjoint  (orbit tiles): Xbar, WWbar, VVbar, their orbit sums;
//                    wbar -> Wbar staging of the adjoint contractions, vbar -> B0
//   4. V gradients   (streaming over (r, z) rows of vbar and Dbar): the V-term
//                    gradients and the Dbar reduction into mo_energy_bar
// An orbit tile is one occupied representative i >= j >= k with all its
// permutations, times one triple of virtual sub-blocks with all its
// orderings: closed under the simultaneous permutations of the orbit sums and
// the virtual-only permutations of r3, so passes 1 and 3 gather only within
// shared memory.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace tb {

constexpr int kLnoMaxO = 64;    // largest nocc of the LNO path (projection tiles)
constexpr int kLnoMaxTv = 16;   // largest virtual block
constexpr int kLnoThreads = 256;
constexpr int kLnoTile = 32;    // columns per projection tile
constexpr int kLnoSB = 4;       // virtual sub-block edge of an orbit tile
constexpr int kLnoRegion = kLnoSB * kLnoSB * kLnoSB;
// slab layout in shared memory: slot s at s + 3 (s / 16) (fewer bank conflicts
// on the permuted gathers), 73 doubles per slab
constexpr int kLnoSlab = kLnoRegion + 3 * (kLnoRegion / 16 - 1) + 1;
__host__ __device__ constexpr int lno_pad(int slot) { return slot + 3 * (slot >> 4); }
constexpr int kLnoMaxSub = 64;  // sub-block triples per chunk: (16/4)^3
constexpr int kLnoWaves = 4;    // waves of the streaming passes

struct LnoSub {
    int st[3];
    int len[3];
};

struct LnoArgs {
    Dims d;
    ChunkDesc ch;
    signed char tau_of[27];                // ordering of (slot x, slot y, slot z); slots 0..2 = A, B, C
    int nsub;
    LnoSub sub[kLnoMaxSub];
    const int *ijk;                        // occupied representatives i >= j >= k
    const void *S;                         // raw w of the chunk (staging, FP64 or FP32)
    double *B0, *B1, *B2, *B3;             // chunk-shaped work arrays (staging layout)
    const double *mat, *mo_e, *t1, *t2, *ovov, *fvo;
    void *SW;                              // Wbar staging per ordering: FP64 [y][p][x][q][rzp], or
                                           // 16-bit hi/lo planes [h][y][p][x][q][rzp] at 2 swoff
    const double *wscale;                  // power-of-two scale of the fp16 split
    double *mat_bar, *mo_bar, *t1_bar, *t2_bar, *ovov_bar, *fvo_bar;
    double ybar;
    int want_grad;
    double *part;                          // energy partials, gridDim.x * nperm
    int n_ijk;                             // occupied representatives
};

// r3 on the virtual indices (pyscfad/cc/ccsd_t_slow.py:84-87):
// Z(j) = sum_s c_s X(i) with i[s[k]] = j[k], s = (0,1,2), (1,2,0), (2,0,1),
// (2,1,0), (0,2,1), (1,0,2) (the orderings of lno_build_tables).
__constant__ double c_r3_coef[6] = {4.0, 1.0, 1.0, -2.0, -2.0, -2.0};

__device__ __forceinline__ int lno_slot(const ChunkDesc &ch, int g) {
    return (g >= ch.base[0] && g < ch.base[0] + ch.nabc[0]) ? 0
           : (g >= ch.base[1] && g < ch.base[1] + ch.nabc[1]) ? 1
                                                               : 2;
}

__device__ __forceinline__ double lno_warp_sum(double s) {
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

// ---------------------------------------------------------------------------
// orbit tiles
// ---------------------------------------------------------------------------
// Candidate region c = 6 pi + rho: occupied triple (ijk[pi0], ijk[pi1], ijk[pi2])
// and virtual sub-ranges (U[rho0], U[rho1], U[rho2]).  Candidates with the same
// triple and ranges hold the same positions; the first of them is "primary"
// and owns a 4x4x4 slab of the shared arrays.  A position is (slab, slot),
// slot = (4 l0 + l1) 4 + l2 for local virtual indices l.  The gather tables
// give, per candidate and permutation, the candidate holding the permuted
// position, and per slot and permutation the permuted slot.
constexpr int kLnoIt = (36 * kLnoRegion + kLnoThreads - 1) / kLnoThreads;   // positions per thread

// Gather tables, the same for every tile (built on the host, lno_build_tables):
// per candidate and permutation the candidate holding the permuted position,
// per permutation and slot the permuted slot; sigma runs over the six
// simultaneous permutations, s over the six terms of r3 (0: forward
// i[m] = j[sinv[m]], 1: adjoint j[k] = i[s[k]]).
struct alignas(16) LnoTables {
    unsigned char symsl[6][kLnoRegion];      // 16-byte multiples first: copied as uint4
    unsigned char r3sl[2][6][kLnoRegion];
    unsigned char symc[36][6];
    unsigned char r3c[2][36][6];
};
// global (not constant) memory: threads read different entries at once
__device__ LnoTables c_lno_tab;

inline void lno_build_tables(LnoTables &t) {
    static const int r3p[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}, {0, 2, 1}, {1, 0, 2}};
    for (int cc = 0; cc < 36; cc++)
        for (int s = 0; s < 6; s++) {
            int pp[3], pr[3], ps[3], m[3];
            perm_of(cc / 6, pp);
            perm_of(cc % 6, pr);
            perm_of(s, ps);
            t.symc[cc][s] = (unsigned char)(6 * perm_index(pp[ps[0]], pp[ps[1]]) + perm_index(pr[ps[0]], pr[ps[1]]));
            for (int k = 0; k < 3; k++) m[r3p[s][k]] = k;
            t.r3c[0][cc][s] = (unsigned char)(6 * (cc / 6) + perm_index(pr[m[0]], pr[m[1]]));
            for (int k = 0; k < 3; k++) m[k] = r3p[s][k];
            t.r3c[1][cc][s] = (unsigned char)(6 * (cc / 6) + perm_index(pr[m[0]], pr[m[1]]));
        }
    for (int s = 0; s < 6; s++)
        for (int sl = 0; sl < kLnoRegion; sl++) {
            const int l[3] = {sl / (kLnoSB * kLnoSB), (sl / kLnoSB) % kLnoSB, sl % kLnoSB};
            int ps[3], m[3];
            perm_of(s, ps);
            t.symsl[s][sl] = (unsigned char)lno_pad((l[ps[0]] * kLnoSB + l[ps[1]]) * kLnoSB + l[ps[2]]);
            for (int k = 0; k < 3; k++) m[r3p[s][k]] = k;
            t.r3sl[0][s][sl] = (unsigned char)lno_pad((l[m[0]] * kLnoSB + l[m[1]]) * kLnoSB + l[m[2]]);
            for (int k = 0; k < 3; k++) m[k] = r3p[s][k];
            t.r3sl[1][s][sl] = (unsigned char)lno_pad((l[m[0]] * kLnoSB + l[m[1]]) * kLnoSB + l[m[2]]);
        }
}

// Duplicate candidates depend only on which occupied indices coincide
// (i == j, j == k) and which virtual sub-ranges coincide (U0 == U1, U1 == U2):
// 16 patterns, each listing its slabs' candidates and every candidate's slab.
struct LnoPattern {
    unsigned char nslab;
    unsigned char cand[36];
    unsigned char prim[36];
};
__device__ LnoPattern c_lno_pat[16];

inline void lno_build_patterns(LnoPattern pats[16]) {
    for (int pid = 0; pid < 16; pid++) {
        const int eo01 = (pid >> 3) & 1, eo12 = (pid >> 2) & 1, ev01 = (pid >> 1) & 1, ev12 = pid & 1;
        int occ[3] = {2, 1, 0}, vr[3] = {2, 1, 0};
        if (eo12) occ[1] = occ[2];
        if (eo01) occ[0] = occ[1];
        if (ev12) vr[1] = vr[2];
        if (ev01) vr[0] = vr[1];
        int key[36][6], first[36];
        for (int c = 0; c < 36; c++) {
            int pp[3], pr[3];
            perm_of(c / 6, pp);
            perm_of(c % 6, pr);
            for (int k = 0; k < 3; k++) {
                key[c][k] = occ[pp[k]];
                key[c][3 + k] = vr[pr[k]];
            }
            first[c] = c;
            for (int c2 = 0; c2 < c; c2++) {
                bool same = true;
                for (int k = 0; k < 6; k++) same = same && key[c2][k] == key[c][k];
                if (same) {
                    first[c] = c2;
                    break;
                }
            }
        }
        LnoPattern &P = pats[pid];
        int n = 0, prim[36];
        for (int c = 0; c < 36; c++)
            if (first[c] == c) {
                prim[c] = n;
                P.cand[n++] = (unsigned char)c;
            }
        for (int c = n; c < 36; c++) P.cand[c] = 0;
        for (int c = 0; c < 36; c++) P.prim[c] = (unsigned char)prim[first[c]];
        P.nslab = (unsigned char)n;
    }
}

// A block handles one virtual sub-block triple and kLnoReps consecutive
// occupied representatives.  What depends only on the virtual side (per
// candidate ordering: staging bases and strides, validity, energies) is set
// up once per block; per representative only the occupied offsets of the
// slabs are recomputed (ALU and shared memory only).
constexpr int kLnoReps = 16;

struct LnoTile {
    // per candidate (virtual side)
    long long soff_v[36], swoff_v[36], swbase_c[36], plane_c[36];
    int strP[36], strQ[36], swP[36], rzp[36], tz[36];
    long long bov_v[36];
    int bt2_v[36], bt1_v[36], bfv_v[36];
    int roff[36][kLnoSB * kLnoSB];  // staging offset of local (l0, l1, 0)
    int swro[36][kLnoSB * kLnoSB];  // Wbar staging offset of local (l0, l1, 0)
    unsigned long long vmask_c[36]; // slots inside the ranges
    unsigned char cpr[36][3];       // which sub-range fills each virtual slot
    double ev_r[3][kLnoSB];         // virtual orbital energies of the three sub-ranges
    double s_eo[kLnoMaxO];
    unsigned char symc[36][6], r3c[2][36][6];
    LnoPattern pat[16];
    int ijk[kLnoReps][3];
    // per slab (current representative)
    long long soff[36], swoff[36], b_ov[36], b_t2[36];
    int b_t1[36], b_fv[36], cand[36];
    double eocc[36];
    short symg[36][6], r3g[2][36][6];
    int nslab, nrep;
};

// once per block: the virtual side of all 36 candidates
__device__ void lno_tile_setup_block(const LnoArgs &A, LnoTile &T) {
    const int o = A.d.o, v = A.d.v;
    const LnoSub &U = A.sub[blockIdx.x];
    const int r0 = blockIdx.y * kLnoReps;
    if (threadIdx.x == 0) T.nrep = min(kLnoReps, A.n_ijk - r0);
    for (int e = threadIdx.x; e < kLnoReps * 3; e += blockDim.x)
        T.ijk[e / 3][e % 3] = r0 + e / 3 < A.n_ijk ? A.ijk[3 * r0 + e] : 0;
    for (int e = threadIdx.x; e < o; e += blockDim.x) T.s_eo[e] = A.mo_e[e];
    for (int e = threadIdx.x; e < 36; e += blockDim.x) T.cand[e] = 0;
    for (int e = threadIdx.x; e < 3 * kLnoSB; e += blockDim.x) {
        const int k = e / kLnoSB, l = e % kLnoSB;
        T.ev_r[k][l] = l < U.len[k] ? A.mo_e[o + U.st[k] + l] : 0.0;
    }
    for (int e = threadIdx.x; e < 36 * 6; e += blockDim.x) {
        T.symc[e / 6][e % 6] = c_lno_tab.symc[e / 6][e % 6];
        T.r3c[0][e / 6][e % 6] = c_lno_tab.r3c[0][e / 6][e % 6];
        T.r3c[1][e / 6][e % 6] = c_lno_tab.r3c[1][e / 6][e % 6];
    }
    for (int e = threadIdx.x; e < (int)sizeof(T.pat); e += blockDim.x)
        reinterpret_cast<unsigned char *>(T.pat)[e] = reinterpret_cast<const unsigned char *>(c_lno_pat)[e];
    const int cc = threadIdx.x;
    if (cc < 36) {
        int pr[3], vst[3], vl[3];
        perm_of(cc % 6, pr);
        for (int k = 0; k < 3; k++) {
            vst[k] = U.st[pr[k]];
            vl[k] = U.len[pr[k]];
            T.cpr[cc][k] = (unsigned char)pr[k];
        }
        const int x0 = vst[0], y0 = vst[1], z0 = vst[2];
        const int t = A.tau_of[(lno_slot(A.ch, x0) * 3 + lno_slot(A.ch, y0)) * 3 + lno_slot(A.ch, z0)];
        const PermBlock &pb = A.ch.pb[t];
        const int oTz = o * pb.Tz;
        const int sx = oTz, sy = pb.Tx * oTz;
        T.strQ[cc] = pb.Ty * sy;
        T.strP[cc] = o * pb.Ty * sy;
        T.tz[cc] = pb.Tz;
        T.soff_v[cc] = pb.soff + (long long)(y0 - pb.Y0) * sy + (long long)(x0 - pb.X0) * sx + (z0 - pb.Z0);
        const int wx = o * pb.rzp, wy = o * pb.Tx * wx;
        T.swP[cc] = pb.Tx * wx;
        T.rzp[cc] = pb.rzp;
        T.swoff_v[cc] = pb.swoff + (long long)(y0 - pb.Y0) * wy + (long long)(x0 - pb.X0) * wx + (z0 - pb.Z0);
        T.plane_c[cc] = (long long)pb.Ty * wy;
        T.swbase_c[cc] = pb.swoff;
        T.bov_v[cc] = (long long)x0 * o * v + y0;
        T.bt2_v[cc] = y0 * v + x0;
        T.bt1_v[cc] = z0;
        T.bfv_v[cc] = z0 * o;
        for (int l01 = 0; l01 < kLnoSB * kLnoSB; l01++) {
            const int l0 = l01 / kLnoSB, l1 = l01 % kLnoSB;
            T.roff[cc][l01] = l1 * sy + l0 * sx;
            T.swro[cc][l01] = l1 * wy + l0 * wx;
        }
        unsigned long long m = 0ull;
        for (int sl = 0; sl < kLnoRegion; sl++) {
            const int l0 = sl / (kLnoSB * kLnoSB), l1 = (sl / kLnoSB) % kLnoSB, l2 = sl % kLnoSB;
            if (l0 < vl[0] && l1 < vl[1] && l2 < vl[2]) m |= 1ull << sl;
        }
        T.vmask_c[cc] = m;
    }
    __syncthreads();
}

// per representative n: the occupied side of its slabs
__device__ void lno_tile_setup_rep(const LnoArgs &A, LnoTile &T, int n) {
    const int o = A.d.o, v = A.d.v;
    const LnoSub &U = A.sub[blockIdx.x];
    const int ijk[3] = {T.ijk[n][0], T.ijk[n][1], T.ijk[n][2]};
    const int pid = ((ijk[0] == ijk[1]) << 3) | ((ijk[1] == ijk[2]) << 2) | ((U.st[0] == U.st[1]) << 1) |
                    (U.st[1] == U.st[2]);
    const LnoPattern &P = T.pat[pid];
    const int c = threadIdx.x;
    if (c == 0) T.nslab = P.nslab;
    if (c < P.nslab) {
        const int cc = P.cand[c];
        int pp[3];
        perm_of(cc / 6, pp);
        const int p = ijk[pp[0]], q = ijk[pp[1]], r = ijk[pp[2]];
        T.cand[c] = cc;
        T.soff[c] = T.soff_v[cc] + (long long)p * T.strP[cc] + (long long)q * T.strQ[cc] + r * T.tz[cc];
        T.swoff[c] = T.swoff_v[cc] + (long long)p * T.swP[cc] + (long long)q * T.rzp[cc] + r * T.tz[cc];
        T.b_ov[c] = ((long long)p * v * o + q) * v + T.bov_v[cc];
        T.b_t2[c] = ((long long)q * o + p) * v * v + T.bt2_v[cc];
        T.b_t1[c] = r * v + T.bt1_v[cc];
        T.b_fv[c] = T.bfv_v[cc] + r;
        T.eocc[c] = T.s_eo[p] + T.s_eo[q] + T.s_eo[r];
        for (int s = 0; s < 6; s++) {
            T.symg[c][s] = (short)(P.prim[T.symc[cc][s]] * kLnoSlab);
            T.r3g[0][c][s] = (short)(P.prim[T.r3c[0][cc][s]] * kLnoSlab);
            T.r3g[1][c][s] = (short)(P.prim[T.r3c[1][cc][s]] * kLnoSlab);
        }
    }
    __syncthreads();
}

// Per-thread constants: a thread's slot in its slabs is the same at every
// iteration (kLnoThreads is a multiple of the slab size), so its local
// indices and the permuted slots of its gathers are loaded once.
struct LnoLane {
    int sl, l0, l1, l2, l01, psl;
    unsigned sym[2], r3[2][2];   // 8-bit permuted padded slots, four per word (six used)

    __device__ __forceinline__ void init() {
        sl = threadIdx.x % kLnoRegion;
        l0 = sl / (kLnoSB * kLnoSB);
        l1 = (sl / kLnoSB) % kLnoSB;
        l2 = sl % kLnoSB;
        l01 = l0 * kLnoSB + l1;
        psl = lno_pad(sl);
        sym[0] = sym[1] = r3[0][0] = r3[0][1] = r3[1][0] = r3[1][1] = 0u;
        for (int s = 0; s < 6; s++) {
            sym[s >> 2] |= (unsigned)c_lno_tab.symsl[s][sl] << (8 * (s & 3));
            r3[0][s >> 2] |= (unsigned)c_lno_tab.r3sl[0][s][sl] << (8 * (s & 3));
            r3[1][s >> 2] |= (unsigned)c_lno_tab.r3sl[1][s][sl] << (8 * (s & 3));
        }
    }
    __device__ __forceinline__ int symsl(int s) const { return (sym[s >> 2] >> (8 * (s & 3))) & 0xff; }
    __device__ __forceinline__ int r3sl(int a, int s) const { return (r3[a][s >> 2] >> (8 * (s & 3))) & 0xff; }
};

// it-th position of this thread: slab g (candidate cg), shared index si, staging offset goff
#define LNO_POS(T, L, it)                                                                                           \
    const int g = (int)(threadIdx.x / kLnoRegion) + (it) * (kLnoThreads / kLnoRegion);                            \
    const bool inr = g < (T).nslab;                                                                               \
    const int cg = inr ? (T).cand[g] : 0;                                                                         \
    const int si = g * kLnoSlab + (L).psl;                                                                        \
    const bool valid = inr && (((T).vmask_c[cg] >> (L).sl) & 1ull);                                                \
    const long long goff = (T).soff[g] + (T).roff[cg][(L).l01] + (L).l2

// pass 1: WW -> B0, Q = r3(WW + VV/2) / D -> B2
template <typename StageT>
__global__ void __launch_bounds__(kLnoThreads) k_lno_tile_fwd(LnoArgs A) {
    const StageT *S = reinterpret_cast<const StageT *>(A.S);
    __shared__ LnoTile T;
    extern __shared__ double lno_sm[];
    double *sW = lno_sm, *sV = lno_sm + 36 * kLnoSlab;
    LnoLane L;
    L.init();
    lno_tile_setup_block(A, T);
    const int o = A.d.o, v = A.d.v;
    const int ovl = L.l0 * o * v + L.l1, t2l = L.l1 * v + L.l0, fvl = L.l2 * o;
    for (int n = 0; n < T.nrep; n++) {
    lno_tile_setup_rep(A, T, n);
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        if (!inr) break;
        double w = 0.0, vv = 0.0;
        if (valid) {
            // v = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r]
            w = (double)S[goff];
            vv = A.ovov[T.b_ov[g] + ovl] * A.t1[T.b_t1[g] + L.l2] + A.t2[T.b_t2[g] + t2l] * A.fvo[T.b_fv[g] + fvl];
        }
        sW[si] = w;
        sV[si] = vv;
    }
    __syncthreads();
    double xr[kLnoIt];
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)si;
        xr[it] = 0.0;
        if (!valid) continue;
        double ww = 0.0, vv = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            const int k = T.symg[g][s] + L.symsl(s);
            ww += sW[k];
            vv += sV[k];
        }
        A.B0[goff] = ww;
        xr[it] = ww + 0.5 * vv;
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)valid;
        (void)goff;
        if (inr) sW[si] = xr[it];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)si;
        if (!valid) continue;
        double z = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) z += c_r3_coef[s] * sW[T.r3g[0][g][s] + L.r3sl(0, s)];
        const double D = T.eocc[g] - T.ev_r[T.cpr[cg][0]][L.l0] - T.ev_r[T.cpr[cg][1]][L.l1] -
                         T.ev_r[T.cpr[cg][2]][L.l2];
        A.B2[goff] = z / D;
    }
    __syncthreads();   // slab data and shared arrays are reused by the next representative
    }
}

// pass 3: Xbar = r3^T(Zbar (B3)), WWbar = P^T(Wtbar) (B1) + Xbar, VVbar = Xbar/2;
// wbar = orbit sum of WWbar -> Wbar staging, vbar = orbit sum of VVbar -> B0.
// SPLIT 0: FP64 staging; 1: fp16 hi/lo of wbar * wscale (exact power of two);
// 2: bf16 hi/lo, unscaled -- the operand formats of the adjoint contractions.
template <int SPLIT>
__global__ void __launch_bounds__(kLnoThreads) k_lno_tile_adj(LnoArgs A) {
    __shared__ LnoTile T;
    extern __shared__ double lno_sm[];
    double *sZ = lno_sm, *sW = lno_sm + 36 * kLnoSlab;
    LnoLane L;
    L.init();
    lno_tile_setup_block(A, T);
    const float wsc = SPLIT == 1 ? (float)*A.wscale : 1.0f;
    for (int n = 0; n < T.nrep; n++) {
    lno_tile_setup_rep(A, T, n);
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        if (!inr) break;
        sZ[si] = valid ? A.B3[goff] : 0.0;
        sW[si] = valid ? A.B1[goff] : 0.0;
    }
    __syncthreads();
    double xr[kLnoIt];
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)goff;
        xr[it] = 0.0;
        if (!valid) continue;
        double xb = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) xb += c_r3_coef[s] * sZ[T.r3g[1][g][s] + L.r3sl(1, s)];
        xr[it] = xb;
        sW[si] += xb;   // only this thread reads sW[si] in this phase
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)valid;
        (void)goff;
        if (inr) sZ[si] = 0.5 * xr[it];
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kLnoIt; it++) {
        LNO_POS(T, L, it);
        (void)si;
        if (!valid) continue;
        double wb = 0.0, vb = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            const int k = T.symg[g][s] + L.symsl(s);
            wb += sW[k];
            vb += sZ[k];
        }
        const long long wl = T.swoff[g] + T.swro[cg][L.l01] + L.l2;
        if (SPLIT == 0) {
            reinterpret_cast<double *>(A.SW)[wl] = wb;
        } else if (SPLIT == 1) {
            const float xs = (float)wb * wsc;
            const __half h = __float2half_rn(xs);
            __half *dst = reinterpret_cast<__half *>(A.SW) + T.swbase_c[cg] + wl;   // 2 swoff + local offset
            dst[0] = h;
            dst[T.plane_c[cg]] = __float2half_rn(xs - __half2float(h));
        } else {
            const float xs = (float)wb;
            const __nv_bfloat16 h = __float2bfloat16_rn(xs);
            __nv_bfloat16 *dst = reinterpret_cast<__nv_bfloat16 *>(A.SW) + T.swbase_c[cg] + wl;
            dst[0] = h;
            dst[T.plane_c[cg]] = __float2bfloat16_rn(xs - __bfloat162float(h));
        }
        A.B0[goff] = vb;
    }
    __syncthreads();   // slab data and shared arrays are reused by the next representative
    }
}

#undef LNO_POS

// ---------------------------------------------------------------------------
// pass 2: projection along the first occupied index, streaming over columns
// ---------------------------------------------------------------------------
// Column c of ordering pb = (((q Ty + y) Tx + x) o + r) Tz + z (< 2^31); position p c.
// Per 32-column tile with all o rows of WW (B0) and Q (B2) in shared memory:
//   Wt[i,c] = sum_l mat[l,i] WW[l,c],  energy += Wt Q;
//   with the adjoint: Zbar = f Wt / D -> B3, Dbar = -f Wt Q / D -> B2 (over Q),
//   P^T(Wtbar)[l,c] = f sum_i mat[l,i] Q[i,c] -> B1, Gram WW Q^T -> mat_bar
//   (f = ybar / 3).
// The three products run on the FP64 tensor cores (mma.sync m8n8k4, FP64 in
// and out): per 8x8 output tile a thread holds D[g][2t], D[g][2t+1]
// (g = lane / 4, t = lane % 4), A[g][t] and B[t][g] of each k-step.
constexpr int kLnoLd = 36;   // row stride of the shared tiles (conflict-free fragment loads)

inline size_t lno_proj_smem(int o) {
    return (size_t)(4 * kLnoMaxO * kLnoLd + o * o + kLnoMaxO + 2 * kLnoTile) * sizeof(double);
}

// 8-byte global -> shared copy that bypasses registers; ok = false writes zero
__device__ __forceinline__ void lno_cp_async8(double *dst, const double *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void lno_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void lno_cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ void lno_dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kLnoThreads, 2) k_lno_proj(LnoArgs A) {
    extern __shared__ double lno_sm[];
    // two buffers of the WW / Q tiles: the next tile streams in while this one is used
    double *sw_b = lno_sm, *sq_b = sw_b + 2 * kLnoMaxO * kLnoLd, *sM = sq_b + 2 * kLnoMaxO * kLnoLd;
    const int o = A.d.o;
    double *s_eo = sM + o * o, *s_ecol_b = s_eo + kLnoMaxO;
    __shared__ double red[kLnoThreads / 32];
    const int o4 = (o + 3) & ~3, o8 = (o + 7) / 8, rows = 8 * o8;
    const PermBlock &pb = A.ch.pb[blockIdx.y];
    const int stride_p = o * o * pb.Tx * pb.Ty * pb.Tz;
    const int ntile = (stride_p + kLnoTile - 1) / kLnoTile;
    const double f = A.ybar / 3.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fg = lane >> 2, ft = lane & 3;   // fragment row group / thread in group
    const bool grad = A.want_grad != 0;
    for (int k = threadIdx.x; k < o * o; k += blockDim.x) sM[k] = A.mat[k];
    for (int k = threadIdx.x; k < o; k += blockDim.x) s_eo[k] = A.mo_e[k];
    constexpr int kG = (kLnoMaxO / 8) * (kLnoMaxO / 8) / (kLnoThreads / 32);   // Gram tiles per warp
    const int ngram = o8 * o8;
    double acc[kG][2];
#pragma unroll
    for (int k = 0; k < kG; k++) acc[k][0] = acc[k][1] = 0.0;
    double en = 0.0;
    const double *W = A.B0 + pb.soff, *Qg = A.B2 + pb.soff;
    // issue the copies of tile tb into buffer b (and its column energies)
    auto issue = [&](int tb, int b) {
        const int c0 = tb * kLnoTile;
        double *sw = sw_b + b * kLnoMaxO * kLnoLd, *sq = sq_b + b * kLnoMaxO * kLnoLd;
        for (int e = threadIdx.x; e < rows * kLnoTile; e += blockDim.x) {
            const int l = e / kLnoTile, j = e % kLnoTile;
            const bool ok = l < o && c0 + j < stride_p;
            const long long at = ok ? (long long)l * stride_p + c0 + j : 0;
            lno_cp_async8(sw + l * kLnoLd + j, W + at, ok);
            lno_cp_async8(sq + l * kLnoLd + j, Qg + at, ok);
        }
        lno_cp_commit();
        if (grad && threadIdx.x < kLnoTile) {
            int cc = c0 + threadIdx.x;
            double ec = 0.0;
            if (cc < stride_p) {
                const int zl = cc % pb.Tz;
                cc /= pb.Tz;
                const int r = cc % o;
                cc /= o;
                const int xl = cc % pb.Tx;
                cc /= pb.Tx;
                const int yl = cc % pb.Ty;
                const int q = cc / pb.Ty;
                ec = A.mo_e[q] + A.mo_e[r] - A.mo_e[o + pb.X0 + xl] - A.mo_e[o + pb.Y0 + yl] -
                     A.mo_e[o + pb.Z0 + zl];
            }
            s_ecol_b[b * kLnoTile + threadIdx.x] = ec;
        }
    };
    int buf = 0;
    if ((int)blockIdx.x < ntile) issue(blockIdx.x, 0);
    for (int tb = blockIdx.x; tb < ntile; tb += gridDim.x) {
        const int c0 = tb * kLnoTile;
        if (tb + (int)gridDim.x < ntile)
            issue(tb + gridDim.x, buf ^ 1);
        else
            lno_cp_commit();   // empty group: keeps the wait count uniform
        lno_cp_wait1();        // this thread's copies of tile tb have landed
        __syncthreads();       // ... and everyone's
        const double *sw = sw_b + buf * kLnoMaxO * kLnoLd, *sq = sq_b + buf * kLnoMaxO * kLnoLd;
        const double *s_ecol = s_ecol_b + buf * kLnoTile;
        // Wt and P^T(Q) tiles (rows i / l in 8-blocks, columns in 8-blocks) and their epilogue
        for (int tile = warp; tile < o8 * (kLnoTile / 8); tile += kLnoThreads / 32) {
            const int mt = tile / (kLnoTile / 8), nt = tile % (kLnoTile / 8);
            const int i = mt * 8 + fg;
            double w0 = 0.0, w1 = 0.0, p0 = 0.0, p1 = 0.0;
            for (int k0 = 0; k0 < o4; k0 += 4) {
                const int l = k0 + ft;
                const bool in = i < o && l < o;
                lno_dmma(w0, w1, in ? sM[l * o + i] : 0.0, sw[l * kLnoLd + nt * 8 + fg]);
                if (grad) lno_dmma(p0, p1, in ? sM[i * o + l] : 0.0, sq[l * kLnoLd + nt * 8 + fg]);
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int cl = nt * 8 + 2 * ft + h;
                const double wt = h ? w1 : w0;
                const double qv = sq[i * kLnoLd + cl];
                en += wt * qv;
                const int c = c0 + cl;
                if (grad && i < o && c < stride_p) {
                    const double D = s_eo[i] + s_ecol[cl];
                    const double qb = f * wt;
                    const long long at = pb.soff + (long long)i * stride_p + c;
                    A.B3[at] = qb / D;
                    A.B2[at] = -qb * qv / D;
                    A.B1[at] = f * (h ? p1 : p0);
                }
            }
        }
        if (grad) {
            // Gram[l, i] += sum_c WW[l, c] Q[i, c]: warp-owned 8x8 tiles, k over the 32 columns
#pragma unroll
            for (int k = 0; k < kG; k++) {
                const int gt = warp + k * (kLnoThreads / 32);
                if (gt < ngram) {
                    const int mt = gt / o8, nt = gt % o8;
#pragma unroll
                    for (int k0 = 0; k0 < kLnoTile; k0 += 4)
                        lno_dmma(acc[k][0], acc[k][1], sw[(mt * 8 + fg) * kLnoLd + k0 + ft],
                                 sq[(nt * 8 + fg) * kLnoLd + k0 + ft]);
                }
            }
        }
        __syncthreads();   // buffer buf is refilled two tiles from now
        buf ^= 1;
    }
    en = lno_warp_sum(en);
    if (lane == 0) red[warp] = en;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kLnoThreads / 32; w++) s += red[w];
        A.part[blockIdx.y * gridDim.x + blockIdx.x] = s / 3.0;
    }
    if (!grad) return;
#pragma unroll
    for (int k = 0; k < kG; k++) {
        const int gt = warp + k * (kLnoThreads / 32);
        if (gt < ngram) {
            const int l = (gt / o8) * 8 + fg;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int i = (gt % o8) * 8 + 2 * ft + h;
                const double gv = h ? acc[k][1] : acc[k][0];
                if (l < o && i < o && gv != 0.0) atomicAdd(&A.mat_bar[l * o + i], f * gv);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// pass 4: V-term and denominator gradients from vbar (B0) and Dbar (B2), one
// warp per (p, q, y, x) row of o Tz contiguous (r, z) values:
//   ovov_bar[p,x,q,y] += sum_rz vbar t1[r,z],   t2_bar[q,p,y,x] += sum_rz vbar fvo[z,r],
//   t1_bar[r,z] += sum vbar ovov[p,x,q,y],      fvo_bar[z,r] += sum vbar t2[q,p,y,x],
//   mo_bar[p], [q], [r] += sum Dbar;  mo_bar[o+x], [o+y], [o+z] -= sum Dbar.
// Lane k of every warp owns elements k, k+32, ... of the row (M per lane) and
// keeps their sums in registers across rows.
// ---------------------------------------------------------------------------
template <int M>
__global__ void __launch_bounds__(kLnoThreads) k_lno_vgrad(LnoArgs A) {
    __shared__ double s_t1[kLnoMaxO * kLnoMaxTv], s_fv[kLnoMaxO * kLnoMaxTv], s_rz[kLnoMaxO * kLnoMaxTv];
    __shared__ double s_occ[kLnoThreads / 32][kLnoMaxO], s_vir[kLnoThreads / 32][2][kLnoMaxTv];
    const int o = A.d.o, v = A.d.v;
    const PermBlock &pb = A.ch.pb[blockIdx.y];
    const int oTz = o * pb.Tz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < oTz; k += blockDim.x) s_t1[k] = s_fv[k] = s_rz[k] = 0.0;
    for (int k = lane; k < kLnoMaxO; k += 32) s_occ[warp][k] = 0.0;
    for (int k = lane; k < 2 * kLnoMaxTv; k += 32) s_vir[warp][k / kLnoMaxTv][k % kLnoMaxTv] = 0.0;
    __syncthreads();
    double a1[M], af[M], ar[M];
#pragma unroll
    for (int m = 0; m < M; m++) a1[m] = af[m] = ar[m] = 0.0;
    const int npr = o * o * pb.Ty * pb.Tx;
    const int nwarp = gridDim.x * (blockDim.x >> 5);
    for (int pr = blockIdx.x * (blockDim.x >> 5) + warp; pr < npr; pr += nwarp) {
        const int xl = pr % pb.Tx, yl = (pr / pb.Tx) % pb.Ty;
        const int q = (pr / (pb.Tx * pb.Ty)) % o, p = pr / (pb.Tx * pb.Ty * o);
        const int x = pb.X0 + xl, y = pb.Y0 + yl;
        const long long iov = (((long long)p * v + x) * o + q) * v + y;
        const long long it2 = (((long long)q * o + p) * v + y) * v + x;
        const double ovv = A.ovov[iov], t2v = A.t2[it2];
        const double *rv = A.B0 + pb.soff + (long long)pr * oTz;
        const double *rd = A.B2 + pb.soff + (long long)pr * oTz;
        double s_ov = 0.0, s_t2 = 0.0, s_d = 0.0;
#pragma unroll
        for (int m = 0; m < M; m++) {
            const int k = lane + 32 * m;
            if (k < oTz) {
                const int r = k / pb.Tz, z = pb.Z0 + k % pb.Tz;
                const double vb = rv[k], db = rd[k];
                s_ov += vb * __ldg(&A.t1[r * v + z]);
                s_t2 += vb * __ldg(&A.fvo[z * o + r]);
                s_d += db;
                a1[m] += vb * ovv;
                af[m] += vb * t2v;
                ar[m] += db;
            }
        }
        s_ov = lno_warp_sum(s_ov);
        s_t2 = lno_warp_sum(s_t2);
        s_d = lno_warp_sum(s_d);
        if (lane == 0) {
            if (s_ov != 0.0) atomicAdd(&A.ovov_bar[iov], s_ov);
            if (s_t2 != 0.0) atomicAdd(&A.t2_bar[it2], s_t2);
            s_occ[warp][p] += s_d;
            s_occ[warp][q] += s_d;
            s_vir[warp][0][xl] -= s_d;
            s_vir[warp][1][yl] -= s_d;
        }
    }
    // combine the warps' register sums (one warp at a time: no atomics)
    for (int w = 0; w < kLnoThreads / 32; w++) {
        if (warp == w) {
#pragma unroll
            for (int m = 0; m < M; m++) {
                const int k = lane + 32 * m;
                if (k < oTz) {
                    s_t1[k] += a1[m];
                    s_fv[k] += af[m];
                    s_rz[k] += ar[m];
                }
            }
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < oTz; k += blockDim.x) {
        const int r = k / pb.Tz, z = pb.Z0 + k % pb.Tz;
        if (s_t1[k] != 0.0) atomicAdd(&A.t1_bar[(long long)r * v + z], s_t1[k]);
        if (s_fv[k] != 0.0) atomicAdd(&A.fvo_bar[(long long)z * o + r], s_fv[k]);
        if (s_rz[k] != 0.0) {
            atomicAdd(&A.mo_bar[r], s_rz[k]);
            atomicAdd(&A.mo_bar[o + z], -s_rz[k]);
        }
    }
    for (int k = threadIdx.x; k < o; k += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < kLnoThreads / 32; w++) t += s_occ[w][k];
        if (t != 0.0) atomicAdd(&A.mo_bar[k], t);
    }
    for (int k = threadIdx.x; k < 2 * kLnoMaxTv; k += blockDim.x) {
        const int role = k / kLnoMaxTv, kk = k % kLnoMaxTv;
        const int len = role == 0 ? pb.Tx : pb.Ty;
        if (kk >= len) continue;
        double t = 0.0;
        for (int w = 0; w < kLnoThreads / 32; w++) t += s_vir[w][role][kk];
        if (t != 0.0) atomicAdd(&A.mo_bar[o + (role == 0 ? pb.X0 : pb.Y0) + kk], t);
    }
}

inline size_t lno_tile_smem() { return 2 * 36 * kLnoSlab * sizeof(double); }

}  // namespace tb

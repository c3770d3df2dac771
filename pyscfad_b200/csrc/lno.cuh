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
// The projector couples occupied triples that the canonical epilogue keeps
// apart, so these steps work on whole-chunk FP64 arrays in the staging layout
// (position = (tau; p, q, y, x, r, z), p outermost) instead of orbit tiles.
// A chunk is closed under the index permutations involved (simultaneous
// occupied/virtual permutations, the virtual-only permutations of r3, and
// any change of p), so every gather stays inside the chunk.
#pragma once
#include "common.cuh"

namespace tb {

constexpr int kLnoMaxO = 64;    // largest nocc of the LNO path (shared-memory tiles)
constexpr int kLnoMaxTv = 16;   // largest virtual block
constexpr int kLnoThreads = 256;
constexpr int kLnoTile = 32;    // columns of a projection tile

struct LnoArgs {
    Dims d;
    ChunkDesc ch;
    signed char tau_of[27];                // ordering of (slot x, slot y, slot z); slots 0..2 = A, B, C
    const double *S;                       // raw w of the chunk (FP64 staging)
    double *B0, *B1, *B2, *B3;             // chunk-shaped work arrays (staging layout)
    const double *mat, *mo_e, *t1, *t2, *ovov, *fvo;
    double *SW;                            // FP64 Wbar staging [y][p][x][q][rzp] per ordering
    double *mat_bar, *mo_bar, *t1_bar, *t2_bar, *ovov_bar, *fvo_bar;
    double ybar;
    double *part;                          // energy partials, gridDim.x * nperm
};

// r3 on the virtual indices (pyscfad/cc/ccsd_t_slow.py:84-87):
// Z(j) = sum_s c_s X(i) with i[s[k]] = j[k].
__constant__ int c_r3_perm[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}, {0, 2, 1}, {1, 0, 2}};
__constant__ double c_r3_coef[6] = {4.0, 1.0, 1.0, -2.0, -2.0, -2.0};

__device__ __forceinline__ int lno_slot(const ChunkDesc &ch, int g) {
    return (g >= ch.base[0] && g < ch.base[0] + ch.nabc[0]) ? 0
           : (g >= ch.base[1] && g < ch.base[1] + ch.nabc[1]) ? 1
                                                               : 2;
}

// staging offset of position (p,q,r; x,y,z), global virtual indices
__device__ __forceinline__ long long lno_off(const LnoArgs &A, int p, int q, int r, int x, int y, int z) {
    const int o = A.d.o;
    const int sx = lno_slot(A.ch, x), sy = lno_slot(A.ch, y), sz = lno_slot(A.ch, z);
    const PermBlock &pb = A.ch.pb[A.tau_of[(sx * 3 + sy) * 3 + sz]];
    return pb.soff + ((((long long)p * o + q) * pb.Ty + (y - pb.Y0)) * pb.Tx + (x - pb.X0)) * o * pb.Tz +
           (long long)r * pb.Tz + (z - pb.Z0);
}

struct LnoPos {
    int p, q, r, x, y, z;
    long long off;
};

// position idx of ordering pb (staging order p, q, y, x, r, z)
__device__ __forceinline__ LnoPos lno_decode(const LnoArgs &A, const PermBlock &pb, long long idx) {
    const int o = A.d.o;
    LnoPos P;
    P.off = pb.soff + idx;
    P.z = (int)(idx % pb.Tz) + pb.Z0;
    idx /= pb.Tz;
    P.r = (int)(idx % o);
    idx /= o;
    P.x = (int)(idx % pb.Tx) + pb.X0;
    idx /= pb.Tx;
    P.y = (int)(idx % pb.Ty) + pb.Y0;
    idx /= pb.Ty;
    P.q = (int)(idx % o);
    P.p = (int)(idx / o);
    return P;
}

__device__ __forceinline__ long long lno_npos(const LnoArgs &A, const PermBlock &pb) {
    const long long o = A.d.o;
    return o * o * o * pb.Tx * pb.Ty * pb.Tz;
}

__device__ __forceinline__ double lno_v(const LnoArgs &A, int p, int q, int r, int x, int y, int z) {
    const int o = A.d.o, v = A.d.v;
    return A.ovov[(((long long)p * v + x) * o + q) * v + y] * A.t1[(long long)r * v + z] +
           A.t2[(((long long)q * o + p) * v + y) * v + x] * A.fvo[(long long)z * o + r];
}

__device__ __forceinline__ double lno_D(const LnoArgs &A, int p, int q, int r, int x, int y, int z) {
    const int o = A.d.o;
    return A.mo_e[p] + A.mo_e[q] + A.mo_e[r] - A.mo_e[o + x] - A.mo_e[o + y] - A.mo_e[o + z];
}

__device__ __forceinline__ double lno_warp_sum(double s) {
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    return s;
}

// one thread per position of ordering blockIdx.y
#define LNO_FOR_POSITIONS(A)                                                                                       \
    const PermBlock &pb = (A).ch.pb[blockIdx.y];                                                                 \
    const long long npos = lno_npos((A), pb);                                                                    \
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < npos;                          \
         idx += (long long)gridDim.x * blockDim.x)

// B0 = WW, B1 = X = WW + VV/2
__global__ void __launch_bounds__(kLnoThreads) k_lno_ww(LnoArgs A) {
    LNO_FOR_POSITIONS(A) {
        const LnoPos P = lno_decode(A, pb, idx);
        const int oc[3] = {P.p, P.q, P.r}, vi[3] = {P.x, P.y, P.z};
        double ww = 0.0, vv = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            int ps[3];
            perm_of(s, ps);
            const int p = oc[ps[0]], q = oc[ps[1]], r = oc[ps[2]];
            const int x = vi[ps[0]], y = vi[ps[1]], z = vi[ps[2]];
            ww += A.S[lno_off(A, p, q, r, x, y, z)];
            vv += lno_v(A, p, q, r, x, y, z);
        }
        A.B0[P.off] = ww;
        A.B1[P.off] = ww + 0.5 * vv;
    }
}

// B2 = Q = r3(X) / D
__global__ void __launch_bounds__(kLnoThreads) k_lno_q(LnoArgs A) {
    LNO_FOR_POSITIONS(A) {
        const LnoPos P = lno_decode(A, pb, idx);
        const int j[3] = {P.x, P.y, P.z};
        double zsum = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            int i[3];
#pragma unroll
            for (int k = 0; k < 3; k++) i[c_r3_perm[s][k]] = j[k];
            zsum += c_r3_coef[s] * A.B1[lno_off(A, P.p, P.q, P.r, i[0], i[1], i[2])];
        }
        A.B2[P.off] = zsum / lno_D(A, P.p, P.q, P.r, P.x, P.y, P.z);
    }
}

// Projection along the first occupied index, out[i, rest] = f sum_l M(l,i) in[l, rest]:
// transpose = 1: M(l,i) = mat[l,i] (Wt from WW); 0: M(l,i) = mat[i,l] (P^T, the adjoint).
// A block stages in[:, c0:c0+32] in shared memory and writes all o rows of
// those columns.
__global__ void __launch_bounds__(kLnoThreads) k_lno_project(LnoArgs A, const double *__restrict__ in,
                                                             double *__restrict__ out, int transpose, double f) {
    __shared__ double tile[kLnoMaxO][kLnoTile + 1];
    const int o = A.d.o;
    const PermBlock &pb = A.ch.pb[blockIdx.y];
    const long long stride_p = lno_npos(A, pb) / o;
    const long long ntile = (stride_p + kLnoTile - 1) / kLnoTile;
    for (long long tb = blockIdx.x; tb < ntile; tb += gridDim.x) {
        const long long c0 = tb * kLnoTile;
        __syncthreads();
        for (int e = threadIdx.x; e < o * kLnoTile; e += blockDim.x) {
            const int l = e / kLnoTile, j = e % kLnoTile;
            tile[l][j] = (c0 + j < stride_p) ? in[pb.soff + l * stride_p + c0 + j] : 0.0;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < o * kLnoTile; e += blockDim.x) {
            const int i = e / kLnoTile, j = e % kLnoTile;
            if (c0 + j >= stride_p) continue;
            double s = 0.0;
            for (int l = 0; l < o; l++)
                s += (transpose ? __ldg(&A.mat[l * o + i]) : __ldg(&A.mat[i * o + l])) * tile[l][j];
            out[pb.soff + i * stride_p + c0 + j] = f * s;
        }
    }
}

// energy partials (1/3) sum Wt Q (B3 = Wt, B2 = Q), one per block
__global__ void __launch_bounds__(kLnoThreads) k_lno_energy(LnoArgs A) {
    __shared__ double red[kLnoThreads / 32];
    double e = 0.0;
    LNO_FOR_POSITIONS(A) e += A.B3[pb.soff + idx] * A.B2[pb.soff + idx];
    e = lno_warp_sum(e);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kLnoThreads / 32; w++) s += red[w];
        A.part[blockIdx.y * gridDim.x + blockIdx.x] = s / 3.0;
    }
}

// mat_bar[l,i] += (ybar/3) sum_rest WW[l, rest] Q[i, rest]
__global__ void __launch_bounds__(kLnoThreads) k_lno_matbar(LnoArgs A) {
    __shared__ double sw[kLnoMaxO][kLnoTile + 1], sq[kLnoMaxO][kLnoTile + 1];
    constexpr int kAcc = kLnoMaxO * kLnoMaxO / kLnoThreads;
    const int o = A.d.o;
    const PermBlock &pb = A.ch.pb[blockIdx.y];
    const long long stride_p = lno_npos(A, pb) / o;
    const long long ntile = (stride_p + kLnoTile - 1) / kLnoTile;
    double acc[kAcc];
#pragma unroll
    for (int k = 0; k < kAcc; k++) acc[k] = 0.0;
    for (long long tb = blockIdx.x; tb < ntile; tb += gridDim.x) {
        const long long c0 = tb * kLnoTile;
        __syncthreads();
        for (int e = threadIdx.x; e < o * kLnoTile; e += blockDim.x) {
            const int l = e / kLnoTile, j = e % kLnoTile;
            const bool ok = c0 + j < stride_p;
            sw[l][j] = ok ? A.B0[pb.soff + l * stride_p + c0 + j] : 0.0;
            sq[l][j] = ok ? A.B2[pb.soff + l * stride_p + c0 + j] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kAcc; k++) {
            const int pair = threadIdx.x + k * kLnoThreads;
            if (pair < o * o) {
                const int l = pair / o, i = pair % o;
                double s = 0.0;
#pragma unroll 8
                for (int j = 0; j < kLnoTile; j++) s += sw[l][j] * sq[i][j];
                acc[k] += s;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kAcc; k++) {
        const int pair = threadIdx.x + k * kLnoThreads;
        if (pair < o * o && acc[k] != 0.0) atomicAdd(&A.mat_bar[pair], A.ybar / 3.0 * acc[k]);
    }
}

// One thread per pair row (p,q,y,x) of ordering blockIdx.y, looping over (r,z);
// the loop is warp-uniform so that every lane takes part in the shuffles.
#define LNO_FOR_PAIR_ROWS(A)                                                                                       \
    const PermBlock &pb = (A).ch.pb[blockIdx.y];                                                                 \
    const long long npr = (long long)(A).d.o * (A).d.o * pb.Ty * pb.Tx;                                          \
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < npr;                 \
         base += (long long)gridDim.x * blockDim.x)

// B3: Wt -> Zbar = (ybar/3) Wt / D in place; Dbar = -(ybar/3) Wt Q / D into mo_bar
__global__ void __launch_bounds__(kLnoThreads) k_lno_zbar(LnoArgs A) {
    __shared__ double s_occ[kLnoMaxO], s_vir[3][kLnoMaxTv];
    const int o = A.d.o;
    for (int e = threadIdx.x; e < kLnoMaxO; e += blockDim.x) s_occ[e] = 0.0;
    for (int e = threadIdx.x; e < 3 * kLnoMaxTv; e += blockDim.x) s_vir[e / kLnoMaxTv][e % kLnoMaxTv] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    LNO_FOR_PAIR_ROWS(A) {
        const long long pr = base + lane;
        const bool active = pr < npr;
        const int xl = (int)(pr % pb.Tx), yl = (int)((pr / pb.Tx) % pb.Ty);
        const int q = (int)((pr / ((long long)pb.Tx * pb.Ty)) % o), p = (int)(pr / ((long long)pb.Tx * pb.Ty * o));
        const int x = pb.X0 + xl, y = pb.Y0 + yl;
        double zacc[kLnoMaxTv];
#pragma unroll
        for (int z = 0; z < kLnoMaxTv; z++) zacc[z] = 0.0;
        double dsum = 0.0;
        for (int r = 0; r < o; r++) {
            double dr = 0.0;
#pragma unroll
            for (int zl = 0; zl < kLnoMaxTv; zl++) {
                if (zl < pb.Tz) {
                    double db = 0.0;
                    if (active) {
                        const long long off = pb.soff + (pr * o + r) * pb.Tz + zl;
                        const double D = lno_D(A, p, q, r, x, y, pb.Z0 + zl);
                        const double qb = A.ybar / 3.0 * A.B3[off];
                        db = -qb * A.B2[off] / D;
                        A.B3[off] = qb / D;
                    }
                    dr += db;
                    zacc[zl] += db;
                }
            }
            dsum += dr;
            const double wr = lno_warp_sum(dr);   // every lane has the same r
            if (lane == 0 && wr != 0.0) atomicAdd(&s_occ[r], wr);
        }
#pragma unroll
        for (int zl = 0; zl < kLnoMaxTv; zl++) {
            if (zl < pb.Tz) {
                const double wz = lno_warp_sum(zacc[zl]);
                if (lane == 0 && wz != 0.0) atomicAdd(&s_vir[2][zl], -wz);
            }
        }
        if (active && dsum != 0.0) {
            atomicAdd(&s_occ[p], dsum);
            atomicAdd(&s_occ[q], dsum);
            atomicAdd(&s_vir[0][xl], -dsum);
            atomicAdd(&s_vir[1][yl], -dsum);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < o; e += blockDim.x)
        if (s_occ[e] != 0.0) atomicAdd(&A.mo_bar[e], s_occ[e]);
    for (int e = threadIdx.x; e < 3 * kLnoMaxTv; e += blockDim.x) {
        const int role = e / kLnoMaxTv, k = e % kLnoMaxTv;
        const int g0 = role == 0 ? pb.X0 : role == 1 ? pb.Y0 : pb.Z0;
        const int len = role == 0 ? pb.Tx : role == 1 ? pb.Ty : pb.Tz;
        if (k < len && s_vir[role][k] != 0.0) atomicAdd(&A.mo_bar[o + g0 + k], s_vir[role][k]);
    }
}

// Xbar(i) = sum_s c_s Zbar(j), j[k] = i[s[k]] (the transpose of r3);
// B0 += Xbar (WWbar), B1 = Xbar / 2 (VVbar)
__global__ void __launch_bounds__(kLnoThreads) k_lno_xbar(LnoArgs A) {
    LNO_FOR_POSITIONS(A) {
        const LnoPos P = lno_decode(A, pb, idx);
        const int i[3] = {P.x, P.y, P.z};
        double xb = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++)
            xb += c_r3_coef[s] *
                  A.B3[lno_off(A, P.p, P.q, P.r, i[c_r3_perm[s][0]], i[c_r3_perm[s][1]], i[c_r3_perm[s][2]])];
        A.B0[P.off] += xb;
        A.B1[P.off] = 0.5 * xb;
    }
}

// wbar, vbar: orbit sums of WWbar (B0) and VVbar (B1).  wbar goes to the FP64
// Wbar staging that the adjoint contractions read; vbar to the V-term gradients
// of v = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r].
__global__ void __launch_bounds__(kLnoThreads) k_lno_scatter(LnoArgs A) {
    __shared__ double s_t1[kLnoMaxO][kLnoMaxTv], s_fv[kLnoMaxO][kLnoMaxTv];
    const int o = A.d.o, v = A.d.v;
    for (int e = threadIdx.x; e < kLnoMaxO * kLnoMaxTv; e += blockDim.x) {
        s_t1[e / kLnoMaxTv][e % kLnoMaxTv] = 0.0;
        s_fv[e / kLnoMaxTv][e % kLnoMaxTv] = 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    LNO_FOR_PAIR_ROWS(A) {
        const long long pr = base + lane;
        const bool active = pr < npr;
        const int xl = (int)(pr % pb.Tx), yl = (int)((pr / pb.Tx) % pb.Ty);
        const int q = (int)((pr / ((long long)pb.Tx * pb.Ty)) % o), p = (int)(pr / ((long long)pb.Tx * pb.Ty * o));
        const int x = pb.X0 + xl, y = pb.Y0 + yl;
        const long long iov = (((long long)p * v + x) * o + q) * v + y;
        const long long it2 = (((long long)q * o + p) * v + y) * v + x;
        const double ovv = active ? A.ovov[iov] : 0.0, t2v = active ? A.t2[it2] : 0.0;
        const long long wx = (long long)o * pb.rzp, wy = (long long)o * pb.Tx * wx;
        const long long swrow = pb.swoff + yl * wy + (long long)p * pb.Tx * wx + xl * wx + (long long)q * pb.rzp;
        double a_ov = 0.0, a_t2 = 0.0;
        for (int r = 0; r < o; r++) {
            for (int zl = 0; zl < pb.Tz; zl++) {
                const int z = pb.Z0 + zl;
                double vb = 0.0;
                if (active) {
                    const int occ[3] = {p, q, r}, vir[3] = {x, y, z};
                    double wb = 0.0;
#pragma unroll
                    for (int s = 0; s < 6; s++) {
                        int ps[3];
                        perm_of(s, ps);
                        const long long off = lno_off(A, occ[ps[0]], occ[ps[1]], occ[ps[2]], vir[ps[0]], vir[ps[1]],
                                                      vir[ps[2]]);
                        wb += A.B0[off];
                        vb += A.B1[off];
                    }
                    A.SW[swrow + (long long)r * pb.Tz + zl] = wb;
                    a_ov += vb * A.t1[(long long)r * v + z];
                    a_t2 += vb * A.fvo[(long long)z * o + r];
                }
                // every lane has the same (r, z)
                const double w1 = lno_warp_sum(vb * ovv), w2 = lno_warp_sum(vb * t2v);
                if (lane == 0) {
                    if (w1 != 0.0) atomicAdd(&s_t1[r][zl], w1);
                    if (w2 != 0.0) atomicAdd(&s_fv[r][zl], w2);
                }
            }
        }
        if (active) {
            if (a_ov != 0.0) atomicAdd(&A.ovov_bar[iov], a_ov);
            if (a_t2 != 0.0) atomicAdd(&A.t2_bar[it2], a_t2);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < o * pb.Tz; e += blockDim.x) {
        const int r = e / pb.Tz, zl = e % pb.Tz;
        if (s_t1[r][zl] != 0.0) atomicAdd(&A.t1_bar[(long long)r * v + pb.Z0 + zl], s_t1[r][zl]);
        if (s_fv[r][zl] != 0.0) atomicAdd(&A.fvo_bar[(long long)(pb.Z0 + zl) * o + r], s_fv[r][zl]);
    }
}

#undef LNO_FOR_POSITIONS
#undef LNO_FOR_PAIR_ROWS

}  // namespace tb

// FP64 GEMM tile with multi-index operand maps.  This is the "plain FP64
// GPU form" of the (T) contractions: the same chunked algorithm as the
// mixed-precision path, computed on the FP64 tensor cores
// (mma.sync.m8n8k4.f64: per 8x8 output tile a thread holds D[g][2t..2t+1],
// and A[g][t], B[t][g] of each k-step, g = lane / 4, t = lane % 4).
//
//   C(m,n) = alpha * [ sum_k A(m,k) B(n,k) + alpha2 * sum_k A2(m,k) B2(n,k) ]
//            (+ C(m,n) when accumulate)
//   A(m,k) = A.p[apply(A.mn, m) + apply(A.k, k)], likewise B, A2, B2, C.
//
// 128x128 output tile, 256 threads (8 warps as 2 x 4, each 64 x 32 = 8 x 4
// MMA tiles), K tiles of 8 (two k-steps of 4), register-staged double
// buffering.  The k part of every operand offset is
// tabulated per K tile in shared memory two tiles ahead (16 threads, one
// apply() each), so the loads themselves are one add per element.
#pragma once
#include "common.cuh"

namespace tb {

template <typename T>
struct GOpT {
    const T *p;
    Map4 mn;
    Map4 k;
    int kfast;  // 1: operand contiguous along k -> load along k
};
using GOp = GOpT<double>;

// TA: element type of the A operand (FP32 staging in the mixed-precision path)
template <typename TA>
struct GemmArgsT {
    int M, N, K, K2;
    GOpT<TA> A;
    GOp B, A2, B2;
    double *C;
    Map4 cm, cn;
    double alpha, alpha2;
    int accumulate;   // 1: C += result (2: as an FP64 atomic add, for tiles that share outputs)
};
using GemmArgs = GemmArgsT<double>;

constexpr int kGBM = 128, kGBN = 128, kGBK = 8;

// Row stride 132 = 4 (mod 16): the fragment loads of a half-warp (g in 0..3,
// t in 0..3 at t * 132 + g) hit 16 distinct 8-byte banks.
constexpr int kGLd = kGBM + 4;

struct GemmSmem {
    double As[2][kGBK][kGLd];
    double Bs[2][kGBK][kGLd];
    long long rowA[kGBM], rowB[kGBN], rowA2[kGBM], rowB2[kGBN];
    long long koff[2][2][kGBK];   // [tile parity][A, B][k in tile]: k part of the offset (-1: k >= K)
};

template <typename T>
__device__ __forceinline__ void gemm_load_tile(const GOpT<T> &op, const long long *rows, const long long *koff,
                                               int tid, double scale, double (&r)[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int e = tid + 256 * i;
        int ml, kl;
        if (op.kfast) {
            kl = e & 7;
            ml = e >> 3;
        } else {
            ml = e & 127;
            kl = e >> 7;
        }
        const long long ro = rows[ml], ko = koff[kl];
        double val = 0.0;
        if (ro >= 0 && ko >= 0) val = (double)op.p[ro + ko] * scale;
        r[i] = val;
    }
}

__device__ __forceinline__ void gemm_store_tile(double (*S)[kGLd], int kfast, int tid,
                                                const double (&r)[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int e = tid + 256 * i;
        int ml, kl;
        if (kfast) {
            kl = e & 7;
            ml = e >> 3;
        } else {
            ml = e & 127;
            kl = e >> 7;
        }
        S[kl][ml] = r[i];
    }
}

__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <typename TA>
__device__ void gemm_fp64_tile(const GemmArgsT<TA> &g, int m0, int n0, GemmSmem &sm) {
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int fg = lane >> 2, ft = lane & 3;                 // fragment row / k index
    const int wm0 = (warp >> 2) * 64, wn0 = (warp & 3) * 32;  // this warp's 64 x 32 block
    if (tid < 128) {
        int m = m0 + tid;
        bool ok = m < g.M;
        sm.rowA[tid] = ok ? apply(g.A.mn, m) : -1;
        sm.rowA2[tid] = (ok && g.K2 > 0) ? apply(g.A2.mn, m) : -1;
    } else {
        int t = tid - 128;
        int n = n0 + t;
        bool ok = n < g.N;
        sm.rowB[t] = ok ? apply(g.B.mn, n) : -1;
        sm.rowB2[t] = (ok && g.K2 > 0) ? apply(g.B2.mn, n) : -1;
    }
    __syncthreads();

    double acc[8][4][2];   // [m tile][n tile][column pair]
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int kt1 = (g.K + kGBK - 1) / kGBK;
    const int kt2 = (g.K2 > 0) ? (g.K2 + kGBK - 1) / kGBK : 0;
    const int kt_total = kt1 + kt2;
    double ra[4], rb[4];

    // threads 0-15 tabulate the k offsets of tile kt (A for t < 8, B for 8 <= t < 16)
    auto tab_koff = [&](int kt) {
        if (tid < 2 * kGBK && kt < kt_total) {
            const int which = tid >> 3, kl = tid & 7;
            long long off = -1;
            if (kt < kt1) {
                const int k = kt * kGBK + kl;
                if (k < g.K) off = which == 0 ? apply(g.A.k, k) : apply(g.B.k, k);
            } else {
                const int k = (kt - kt1) * kGBK + kl;
                if (k < g.K2) off = which == 0 ? apply(g.A2.k, k) : apply(g.B2.k, k);
            }
            sm.koff[kt & 1][which][kl] = off;
        }
    };
    auto load = [&](int kt) {
        const long long *ka = sm.koff[kt & 1][0], *kb = sm.koff[kt & 1][1];
        if (kt < kt1) {
            gemm_load_tile(g.A, sm.rowA, ka, tid, 1.0, ra);
            gemm_load_tile(g.B, sm.rowB, kb, tid, 1.0, rb);
        } else {
            gemm_load_tile(g.A2, sm.rowA2, ka, tid, g.alpha2, ra);
            gemm_load_tile(g.B2, sm.rowB2, kb, tid, 1.0, rb);
        }
    };
    auto kfA = [&](int kt) { return kt < kt1 ? g.A.kfast : g.A2.kfast; };
    auto kfB = [&](int kt) { return kt < kt1 ? g.B.kfast : g.B2.kfast; };

    tab_koff(0);
    tab_koff(1);
    __syncthreads();
    if (kt_total > 0) {
        load(0);
        gemm_store_tile(sm.As[0], kfA(0), tid, ra);
        gemm_store_tile(sm.Bs[0], kfB(0), tid, rb);
    }
    __syncthreads();
    for (int kt = 0; kt < kt_total; kt++) {
        const int buf = kt & 1;
        if (kt + 1 < kt_total) load(kt + 1);
        // tile kt + 2 reuses the k table of tile kt, whose loads are done
        tab_koff(kt + 2);
#pragma unroll
        for (int ks = 0; ks < kGBK; ks += 4) {
            double a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; i++) a[i] = sm.As[buf][ks + ft][wm0 + 8 * i + fg];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = sm.Bs[buf][ks + ft][wn0 + 8 * j + fg];
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma_884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        if (kt + 1 < kt_total) {
            gemm_store_tile(sm.As[buf ^ 1], kfA(kt + 1), tid, ra);
            gemm_store_tile(sm.Bs[buf ^ 1], kfB(kt + 1), tid, rb);
        }
        __syncthreads();
    }

#pragma unroll
    for (int i = 0; i < 8; i++) {
        int m = m0 + wm0 + 8 * i + fg;
        if (m >= g.M) continue;
        long long cmo = apply(g.cm, m);
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
            const int j = jj >> 1, c = jj & 1;
            int n = n0 + wn0 + 8 * j + 2 * ft + c;
            if (n >= g.N) continue;
            long long off = cmo + apply(g.cn, n);
            double val = g.alpha * acc[i][j][c];
            if (g.accumulate == 2) {
                atomicAdd(&g.C[off], val);
                continue;
            }
            if (g.accumulate) val += g.C[off];
            g.C[off] = val;
        }
    }
}

}  // namespace tb

// Shared definitions for the (T) kernels.
//
// Index conventions (o = nocc, v = nvir, Kp = padded virtual length of the
// contraction axis):
//   raw triples amplitude, the quantity the reference builds per job in
//   get_wv (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t.c:121-152):
//     w^{pqr}_{xyz} = sum_f ovvv[p,x,f,y] t2[r,q,z,f] - sum_m ovoo[p,x,m,q] t2[r,m,z,y]
//     v^{pqr}_{xyz} = ovov[p,x,q,y] t1[r,z] + t2[q,p,y,x] fvo[z,r]
//   Device operand layouts built once per call (prep kernels):
//     A1[y][p][x][f] = ovvv[p,x,f,y]     B1[q][r][z][f] = t2[r,q,z,f]
//     A2[q][p][x][m] = ovoo[p,x,m,q]     B2[y][r][z][m] = t2[r,m,z,y]
//   so that, for fixed (y,q), w is the two-term GEMM
//     W[(p,x),(r,z)] = A1[y][(p,x),:] . B1[q][(r,z),:]^T - A2[q][(p,x),:] . B2[y][(r,z),:]^T
//
// Work is split into "chunks": a triple of virtual blocks A >= B >= C (block
// size Tv) together with ALL occupied indices.  A chunk is closed under the
// simultaneous (occupied, virtual) index permutations that couple raw
// amplitudes in the energy, so its epilogue needs nothing outside the chunk.
// For each distinct ordering tau = (X,Y,Z) of (A,B,C) the raw amplitudes are
// staged as S_tau[p][q][y][x][r][z] (x in X, y in Y, z in Z, local indices).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

constexpr int kBig = 1 << 30;

// idx -> (i0,i1,i2,i3), i0 = idx % e0, i1 = (idx/e0) % e1, i2 = (idx/e0/e1) % e2,
// i3 = rest; offset = sum i_k * s_k (elements).
struct Map4 {
    int e0, e1, e2;
    long long s0, s1, s2, s3;
};

__host__ __device__ inline Map4 map1(long long s0) { return Map4{kBig, 1, 1, s0, 0, 0, 0}; }
__host__ __device__ inline Map4 map2(int e0, long long s0, long long s1) {
    return Map4{e0, kBig, 1, s0, s1, 0, 0};
}
__host__ __device__ inline Map4 map3(int e0, int e1, long long s0, long long s1, long long s2) {
    return Map4{e0, e1, kBig, s0, s1, s2, 0};
}
__host__ __device__ inline Map4 map4(int e0, int e1, int e2, long long s0, long long s1,
                                     long long s2, long long s3) {
    return Map4{e0, e1, e2, s0, s1, s2, s3};
}

__device__ __forceinline__ long long apply(const Map4 &m, int idx) {
    int i0 = idx % m.e0;
    int t = idx / m.e0;
    int i1 = t % m.e1;
    t /= m.e1;
    int i2 = t % m.e2;
    int i3 = t / m.e2;
    return (long long)i0 * m.s0 + (long long)i1 * m.s1 + (long long)i2 * m.s2 +
           (long long)i3 * m.s3;
}

// One distinct ordering (X,Y,Z) of a chunk's virtual blocks.
struct PermBlock {
    int bx, by, bz;        // block indices
    int X0, Tx, Y0, Ty, Z0, Tz;
    long long soff;        // offset of S_tau in the staging buffer (elements)
    int rzp;               // o*Tz rounded up to 8 (16-byte rows of 16-bit Wbar)
    long long swoff;       // offset of Wbar_tau (values) in the Wbar buffer
};

struct ChunkDesc {
    int nperm;
    int blk[3];            // A >= B >= C block indices
    int nabc[3];           // sizes of blocks A, B, C
    int base[3];           // first virtual index of A, B, C
    PermBlock pb[6];
};

struct Dims {
    int o, v, n, Kp, Tv;   // Tv: power-of-two block size
};

// Virtual blocks: v / Tv full blocks of Tv, then the remainder split into
// descending powers of two (so every block size divides 64).
__host__ __device__ inline int num_blocks(const Dims &d) {
    int nfull = d.v / d.Tv, rem = d.v - nfull * d.Tv, n = nfull;
    for (int bit = d.Tv >> 1; bit > 0; bit >>= 1)
        if (rem & bit) n++;
    return n;
}
__host__ __device__ inline int block_size(const Dims &d, int b) {
    int nfull = d.v / d.Tv;
    if (b < nfull) return d.Tv;
    int rem = d.v - nfull * d.Tv, k = b - nfull;
    for (int bit = d.Tv >> 1; bit > 0; bit >>= 1)
        if (rem & bit) {
            if (k == 0) return bit;
            --k;
        }
    return 0;
}
__host__ __device__ inline int block_start(const Dims &d, int b) {
    int nfull = d.v / d.Tv;
    if (b <= nfull) return b * d.Tv;
    int s = nfull * d.Tv, rem = d.v - s, k = b - nfull;
    for (int bit = d.Tv >> 1; bit > 0; bit >>= 1)
        if (rem & bit) {
            if (k == 0) return s;
            s += bit;
            --k;
        }
    return s;
}

// The six orderings of three slots, lexicographic: index = 2*first + (second is
// the larger of the two remaining).
__host__ __device__ constexpr inline void perm_of(int s, int out[3]) {
    const int first = s >> 1;
    const int lo = (first == 0) ? 1 : 0;
    const int hi = (first == 2) ? 1 : 2;
    out[0] = first;
    out[1] = (s & 1) ? hi : lo;
    out[2] = (s & 1) ? lo : hi;
}

__host__ __device__ constexpr inline int perm_index(int a, int b) {
    int lo = (a == 0) ? 1 : 0;  // smallest remaining slot
    return 2 * a + (b == lo ? 0 : 1);
}

// index of the ordering t -> P[s][P[pi][t]]
__host__ __device__ constexpr inline int perm_compose(int s, int pi) {
    int ps[3] = {0, 0, 0}, pp[3] = {0, 0, 0};
    perm_of(s, ps);
    perm_of(pi, pp);
    return perm_index(ps[pp[0]], ps[pp[1]]);
}

}  // namespace tb

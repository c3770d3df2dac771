// Chunk epilogue, common case: one occupied representative i > j > k (or,
// DEG = 1 / 2, i = j > k / i > j = k) and three distinct, full 8-wide virtual
// sub-ranges (a work item).  Same math and the same outputs as k_f2t (f2.cuh),
// which keeps every other case (i = j = k, coinciding or short sub-ranges, the
// FP64 mode):
//
//   WW(s) = sum_tau w(tau(ijk), tau(s abc)),  VV(s) likewise from v,
//   X = WW + VV/2,  Z = r3(X),  E += 2 sum_s WW Z / D,
//   Wbar(s) = c (Z + r3 WW)/D,  Vbar(s) = c r3(WW)/(2D)   (c = 2 ybar)
// (pyscfad/cc/ccsd_t_slow.py:46-124, pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:64-117).
//
// With nothing degenerate, the 36 regions of a work item are exactly the
// pairs (sub-range ordering pi, occupied ordering rho), region pi*6 + rho,
// and each raw amplitude belongs to one orbit item and one ordering s, so
// every index map is a compile-time constant once the (s, tau) loops unroll.
// With two equal occupied indices (DEG) the occupied orderings rho and
// rho' = (the swap of the two equal slots) o rho name the same raw amplitudes:
// only the region of the smaller of the two is loaded (18 regions) and read
// for both, so every sum over tau is the one of k_f2t; the orbit weight
// n_ijk n_abc / 18 is 1 instead of 2; and that region writes Wbar and the
// V-term gradients of both orderings, s(pi, rho) + s(pi, rho').
//
// Persistent and software-pipelined: one CTA of 512 threads per SM walks the
// work items w = blockIdx.x + k*grid.  The W tile of item k+1 (36 regions x
// 64 runs of 8 z values, read as whole 32-byte sectors by four lanes each,
// 8-byte cp.async, L2 evict-first) streams into the second of two shared
// buffers while item k is computed and written back; one orbit item per
// thread.  Per item:
//   B0  V-term tables of item k (prefetched into registers) -> shared
//       {ovov[p,x,q,y], t2[q,p,y,x]} [pair][sub-range pair][8][8], t1, fvo;
//       copies of item k+1 issued; wait for item k's copies
//   B1  items: WW, VV, Z, energy, Wbar / Vbar, d E / d e_abc
//   B2  item results overlay the consumed W buffer; energy and orbital-energy
//       partials written (per-warp partials, fixed summation order)
//   B3  write-back: 72 half regions (one 8-wide z run per lane) over the 16
//       warps: Wbar leaves as 16-byte fp16/bf16 hi and lo runs, V-term
//       gradients as row sums (registers) and column sums (warp shuffles)
//       added to the FP64 gradients; set-up of items k+1 / k+2 and the table
//       loads of item k+1 run here.
// Region descriptors of the copies (item k+1) and of the write-back (item k,
// double-buffered) are built by 36 threads one item ahead.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "f2.cuh"
#include "tc_ptx.cuh"

namespace tb {

struct F2pTile {
    static constexpr int SB = 8;
    static constexpr int SX = 8, SY = 70;           // W tile: (y, x, z) at y*SY + x*SX + z (floats);
                                                    // 8-byte rows, <= 2-way bank conflicts in the six permuted gathers
    static constexpr int REG = SB * SY;             // 560 floats per region
    // item results {Wbar, Vbar} per ordering s: float2 planes, item (la, lb, lc)
    // at la*RA + lb*RB + lc*RC (strides keep the write-back gathers within
    // 2-way bank conflicts per half-warp)
    static constexpr int RA = 70, RB = 9, RC = 2;
    static constexpr int PLANE = 7 * RA + 7 * RB + 7 * RC + 1;   // 568 float2
    static constexpr int TS = 9;                    // V-term table rows: [pair][sub-range pair][x][y] at x*TS + y
    static constexpr int TBLK = 8 * TS;
    static constexpr int TAB = 36 * TBLK;           // float2 {ovov, t2}
    static_assert((36 * REG) % 2 == 0, "float2 tables start 8-byte aligned");
};

__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// 8-byte asynchronous copy global -> shared (L1-allocating; L2 policy hint)
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gsrc, uint64_t pol) {
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(smem_u32(smem_dst)),
                 "l"(gsrc), "l"(pol)
                 : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// the ordering s with perm_compose(s, rho) == pi
__host__ __device__ constexpr int f2p_sof(int pi, int rho) {
    int r = 0;
    for (int s = 0; s < 6; s++)
        if (perm_compose(s, rho) == pi) r = s;
    return r;
}

template <int H>   // 1: fp16 hi/lo, 2: bf16 hi/lo
__device__ __forceinline__ void f2p_split8(const float (&w)[8], float scale, uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float a = w[2 * c] * scale, b = w[2 * c + 1] * scale;
        if (H == 1) {
            const __half2 hh = __floats2half2_rn(a, b);
            const float2 hf = __half22float2(hh);
            const __half2 ll = __floats2half2_rn(a - hf.x, b - hf.y);
            h[c] = *reinterpret_cast<const uint32_t *>(&hh);
            l[c] = *reinterpret_cast<const uint32_t *>(&ll);
        } else {
            const __nv_bfloat162 hh = __floats2bfloat162_rn(a, b);
            const float2 hf = __bfloat1622float2(hh);
            const __nv_bfloat162 ll = __floats2bfloat162_rn(a - hf.x, b - hf.y);
            h[c] = *reinterpret_cast<const uint32_t *>(&hh);
            l[c] = *reinterpret_cast<const uint32_t *>(&ll);
        }
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ int sel3(int a, int b, int c, int i) { return i == 0 ? a : (i == 1 ? b : c); }

// DEG = 1 (i = j): ordering 2 swaps the values 0 and 1 of an occupied
// ordering; DEG = 2 (j = k): ordering 1 swaps 1 and 2.  The partner of rho
// names the same occupied triple; the three rho below their partner are
// {0, 1, 4} and {0, 2, 3}.
__host__ __device__ constexpr int f2p_partner(int deg, int rho) { return perm_compose(deg == 1 ? 2 : 1, rho); }
__host__ __device__ constexpr int f2p_lead(int deg, int rho) {
    return f2p_partner(deg, rho) < rho ? f2p_partner(deg, rho) : rho;
}
__host__ __device__ constexpr int f2p_act(int deg, int k) { return k == 0 ? 0 : (deg == 1 ? (k == 1 ? 1 : 4) : (k == 1 ? 2 : 3)); }
static_assert(f2p_partner(1, 0) == 2 && f2p_partner(1, 1) == 3 && f2p_partner(1, 4) == 5, "i = j partners");
static_assert(f2p_partner(2, 0) == 1 && f2p_partner(2, 2) == 4 && f2p_partner(2, 3) == 5, "j = k partners");

// f2p_sof(PI, rho) for a run-time rho, from compile-time constants
template <int PI>
__device__ __forceinline__ int f2p_sof_rt(int rho) {
    return (rho == 0) ? f2p_sof(PI, 0) : (rho == 1) ? f2p_sof(PI, 1) : (rho == 2) ? f2p_sof(PI, 2)
         : (rho == 3) ? f2p_sof(PI, 3) : (rho == 4) ? f2p_sof(PI, 4) : f2p_sof(PI, 5);
}


struct F2pSmem {
    using C = F2pTile;
    static constexpr int NT = 512;
    static constexpr int NW = NT / 32;
    static constexpr int WTILE = 36 * C::REG;   // floats per W buffer
    static constexpr size_t BYTES = sizeof(float) * (2 * WTILE + 2 * C::TAB + 2 * 3 * 24);
    static_assert(2 * 6 * C::PLANE <= WTILE, "item results overlay the consumed W buffer");
    static_assert((2 * WTILE * 4) % 16 == 0 && (2 * C::TAB * 4) % 16 == 0, "16-byte aligned sections");
};

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Staging offset and strides of region (pi, rho) = reg of a work item (the
// W copy), and the Wbar offset and strides of the same region (write-back).
struct F2pRegion {
    long long gb, wb, half;
    int gs0, gs1, ws0, ws1;
};

__device__ __forceinline__ F2pRegion f2p_region_desc(const F2P<float> &P, int i0, int i1, int i2,
                                                     const F2Sub &R, int reg) {
    const int o = P.d.o;
    const int pi = reg / 6, rho = reg % 6;
    int pp[3], pr[3];
    perm_of(pi, pp);
    perm_of(rho, pr);
    int bk[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bk[c] = -1;
#pragma unroll
        for (int t = 0; t < 3; t++)
            if (R.st[c] >= P.ch.base[t] && R.st[c] < P.ch.base[t] + P.ch.nabc[t]) bk[c] = P.ch.blk[t];
    }
    const int bx = sel3(bk[0], bk[1], bk[2], pp[0]), by = sel3(bk[0], bk[1], bk[2], pp[1]),
              bz = sel3(bk[0], bk[1], bk[2], pp[2]);
    int tau = 0;
    for (; tau < P.ch.nperm - 1; tau++)
        if (P.ch.pb[tau].bx == bx && P.ch.pb[tau].by == by && P.ch.pb[tau].bz == bz) break;
    const PermBlock &pb = P.ch.pb[tau];
    const int p = sel3(i0, i1, i2, pr[0]), q = sel3(i0, i1, i2, pr[1]), r = sel3(i0, i1, i2, pr[2]);
    const int sx = sel3(R.st[0], R.st[1], R.st[2], pp[0]), sy = sel3(R.st[0], R.st[1], R.st[2], pp[1]),
              sz = sel3(R.st[0], R.st[1], R.st[2], pp[2]);
    const int xs = sx - pb.X0, ys = sy - pb.Y0, zs = sz - pb.Z0;
    F2pRegion g;
    const long long gy = (long long)pb.Tx * o * pb.Tz, gx = (long long)o * pb.Tz;
    g.gb = pb.soff + (long long)(p * o + q) * pb.Ty * gy + ys * gy + xs * gx + (long long)r * pb.Tz + zs;
    g.gs0 = (int)gy;
    g.gs1 = (int)gx;
    const long long wx = (long long)o * pb.rzp, wy = (long long)o * pb.Tx * wx;
    g.wb = 2 * pb.swoff + (long long)ys * wy + (long long)p * pb.Tx * wx + xs * wx + (long long)q * pb.rzp +
           (long long)r * pb.Tz + zs;
    g.ws0 = (int)wy;
    g.ws1 = (int)wx;
    g.half = (long long)pb.Ty * o * pb.Tx * o * pb.rzp;
    return g;
}

// Write-back of one z run of region (sub-range ordering PI, occupied ordering
// rho): Wbar hi/lo out (16-byte halves of the 32-byte sectors whose other
// half comes from the item with the other 8-wide half of this z block,
// scheduled next to it), V-term gradients in (row sums per run, column sums
// over the warp's 32 runs).  DEG: the item results of ordering rho2 (the same
// raw amplitudes) are added first.
template <int H, int PI, int DEG>
__device__ __forceinline__ void f2p_run(const F2P<float> &P, const float2 *sG, const float2 *tOT,
                                        const float *tT1, const float *tFV, int i0, int i1, int i2,
                                        int st0, int st1, int st2, int rho, int rho2, int lane, int run,
                                        long long wbase, int ws0, int ws1, long long half, float wscf) {
    using C = F2pTile;
    constexpr int pp0 = (PI >> 1), pp1 = (PI & 1) ? ((pp0 == 2) ? 1 : 2) : ((pp0 == 0) ? 1 : 0);
    constexpr int pp2 = 3 - pp0 - pp1;
    constexpr int str[3] = {C::RA, C::RB, C::RC};
    constexpr int spair = 2 * pp0 + (pp1 > pp0 ? pp1 - 1 : pp1);
    const int pt0 = rho >> 1;
    const int pt1 = (rho & 1) ? ((pt0 == 2) ? 1 : 2) : ((pt0 == 0) ? 1 : 0);
    const int pt2 = 3 - pt0 - pt1;
    const int s = f2p_sof_rt<PI>(rho);
    const int p = sel3(i0, i1, i2, pt0), q = sel3(i0, i1, i2, pt1), r = sel3(i0, i1, i2, pt2);
    const int o = P.d.o, v = P.d.v;
    const int yy = run >> 3, xx = run & 7;
    const float2 *g = sG + s * C::PLANE + xx * str[pp0] + yy * str[pp1];
    float wb[8], vb[8];
#pragma unroll
    for (int z = 0; z < 8; z++) {
        const float2 gv = g[z * str[pp2]];
        wb[z] = gv.x;
        vb[z] = gv.y;
    }
    if constexpr (DEG != 0) {
        const float2 *g2 = sG + f2p_sof_rt<PI>(rho2) * C::PLANE + xx * str[pp0] + yy * str[pp1];
#pragma unroll
        for (int z = 0; z < 8; z++) {
            const float2 gv = g2[z * str[pp2]];
            wb[z] += gv.x;
            vb[z] += gv.y;
        }
    }
    uint4 hi, lo;
    f2p_split8<H>(wb, wscf, hi, lo);
    const long long wl = wbase + (long long)yy * ws0 + (long long)xx * ws1;
    *reinterpret_cast<uint4 *>(reinterpret_cast<uint16_t *>(P.SW) + wl) = hi;
    *reinterpret_cast<uint4 *>(reinterpret_cast<uint16_t *>(P.SW) + wl + half) = lo;
    const float4 *ra = reinterpret_cast<const float4 *>(tT1 + pt2 * 24 + pp2 * 8);
    const float4 *rf = reinterpret_cast<const float4 *>(tFV + pt2 * 24 + pp2 * 8);
    const float4 a_lo = ra[0], a_hi = ra[1], f_lo = rf[0], f_hi = rf[1];
    const float a1[8] = {a_lo.x, a_lo.y, a_lo.z, a_lo.w, a_hi.x, a_hi.y, a_hi.z, a_hi.w};
    const float f1[8] = {f_lo.x, f_lo.y, f_lo.z, f_lo.w, f_hi.x, f_hi.y, f_hi.z, f_hi.w};
    const float2 ot = tOT[(rho * 6 + spair) * C::TBLK + xx * C::TS + yy];   // pair_index(pt0, pt1) == rho
    float rs1 = 0.f, rs2 = 0.f, colv[16];
#pragma unroll
    for (int z = 0; z < 8; z++) {
        rs1 = fmaf(vb[z], a1[z], rs1);
        rs2 = fmaf(vb[z], f1[z], rs2);
        colv[z] = vb[z] * ot.x;
        colv[8 + z] = vb[z] * ot.y;
    }
    const int x = sel3(st0, st1, st2, pp0) + xx, y = sel3(st0, st1, st2, pp1) + yy;
    atomicAdd(&P.ovov_bar[(((long long)p * v + x) * o + q) * v + y], (double)rs1);
    atomicAdd(&P.t2_bar[(((long long)q * o + p) * v + y) * v + x], (double)rs2);
    // column sums over the warp's 32 runs: t1_bar[r, z], fvo_bar[z, r]
    const double cv = (double)group_reduce_scatter<16, 32>(colv, lane);
    if (lane < 16) {
        const int z = sel3(st0, st1, st2, pp2) + (lane & 7);
        if (lane < 8) atomicAdd(&P.t1_bar[(long long)r * v + z], cv);
        else atomicAdd(&P.fvo_bar[(long long)z * o + r], cv);
    }
}

// H: 1 fp16 hi/lo, 2 bf16 hi/lo.  DEG 0: i > j > k; 1: i = j > k; 2: i > j = k
// (every work item of a launch).
template <int H, int DEG>
__global__ void __launch_bounds__(F2pSmem::NT, 1)
    k_f2p(const __grid_constant__ F2P<float> P, int nitems) {
    using C = F2pTile;
    constexpr double CF = DEG ? 1.0 : 2.0;   // orbit weight n_ijk n_abc / 18
    constexpr int NREG = DEG ? 18 : 36;      // distinct regions (loaded, written back)
    constexpr int NT = F2pSmem::NT, NW = F2pSmem::NW;
    extern __shared__ __align__(16) uint8_t f2p_smem[];
    float *sWb = reinterpret_cast<float *>(f2p_smem);   // W buffers [2][36 regions]
    float2 *tOT = reinterpret_cast<float2 *>(sWb + 2 * F2pSmem::WTILE);
    float *tT1 = reinterpret_cast<float *>(tOT + C::TAB);
    float *tFV = tT1 + 3 * 24;
    __shared__ long long s_lgb[36];                 // copy descriptors of the next item
    __shared__ int s_lgs[36][2];
    __shared__ F2pRegion s_reg[2][36];              // write-back descriptors per buffer
    __shared__ double s_ev[2][24];
    __shared__ double s_eijk[2];
    __shared__ int s_item[2][5];                     // i, j, k, sub, rep
    __shared__ double s_red[2][NW];
    __shared__ double s_evp[NW][13];

    const Dims &d = P.d;
    const int o = d.o, v = d.v;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x;
    if ((int)blockIdx.x >= nitems) return;
    const float wscf = P.want_grad ? (float)*P.wscale : 1.0f;
    const uint64_t pol = policy_evict_first();

    auto rep_of = [&](int wi) { return P.rep0 + wi / P.nsub_l; };
    auto sub_of = [&](int wi) { return P.sub0 + wi % P.nsub_l; };
    // Set-up of work item wi (occupied indices ijk): write-back descriptors and
    // item scalars into buffer b (wbdesc), copy descriptors into s_lgb (lddesc).
    auto setup = [&](int wi, const int (&ijk)[3], int b, bool wbdesc, bool lddesc) {
        const int sub = sub_of(wi);
        const F2Sub &R = P.sub[sub];
        if (tid < 36) {
            const F2pRegion g = f2p_region_desc(P, ijk[0], ijk[1], ijk[2], R, tid);
            if (lddesc) {
                s_lgb[tid] = g.gb;
                s_lgs[tid][0] = g.gs0;
                s_lgs[tid][1] = g.gs1;
            }
            if (wbdesc) s_reg[b][tid] = g;
        } else if (wbdesc && tid < 60) {
            const int t = tid - 36;
            s_ev[b][t] = P.mo_e[o + R.st[t >> 3] + (t & 7)];
        } else if (wbdesc && tid == 64) {
            s_item[b][0] = ijk[0];
            s_item[b][1] = ijk[1];
            s_item[b][2] = ijk[2];
            s_item[b][3] = sub;
            s_item[b][4] = rep_of(wi);
            s_eijk[b] = P.mo_e[ijk[0]] + P.mo_e[ijk[1]] + P.mo_e[ijk[2]];
        }
    };
    // V-term tables of work item wi into registers (stored to shared at B0)
    constexpr int TU = 5;   // 2304 entries / 512 threads, rounded up
    double ov[TU], tt[TU], t1v = 0.0, fvv = 0.0;
    auto load_tables = [&](int wi, const int (&ijk)[3]) {
        const F2Sub &R = P.sub[sub_of(wi)];
#pragma unroll
        for (int u = 0; u < TU; u++) {
            const int e = tid + u * NT;
            if (e < 2304) {
                const int pair = e / 384, spair = (e >> 6) % 6, hi = (e >> 3) & 7, lo = e & 7;
                const int sp = pair >> 1, sq = (pair & 1) ? ((sp == 2) ? 1 : 2) : ((sp == 0) ? 1 : 0);
                const int cx = spair >> 1, cy = (spair & 1) ? ((cx == 2) ? 1 : 2) : ((cx == 0) ? 1 : 0);
                const int p = sel3(ijk[0], ijk[1], ijk[2], sp), q = sel3(ijk[0], ijk[1], ijk[2], sq);
                const int stx = sel3(R.st[0], R.st[1], R.st[2], cx), sty = sel3(R.st[0], R.st[1], R.st[2], cy);
                ov[u] = __ldg(&P.ovov[(((long long)p * v + stx + hi) * o + q) * v + sty + lo]);
                tt[u] = __ldg(&P.t2[(((long long)q * o + p) * v + sty + hi) * v + stx + lo]);
            }
        }
        if (tid < 72) {
            const int sr = tid / 24, zl = tid % 24;
            const int z = sel3(R.st[0], R.st[1], R.st[2], zl >> 3) + (zl & 7), r = sel3(ijk[0], ijk[1], ijk[2], sr);
            t1v = __ldg(&P.t1[(long long)r * v + z]);
            fvv = __ldg(&P.fvo[(long long)z * o + r]);
        }
    };
    auto store_tables = [&]() {
        float *tf = reinterpret_cast<float *>(tOT);
#pragma unroll
        for (int u = 0; u < TU; u++) {
            const int e = tid + u * NT;
            if (e < 2304) {
                const int blk = e >> 6, hi = (e >> 3) & 7, lo = e & 7;
                tf[2 * (blk * C::TBLK + hi * C::TS + lo)] = (float)ov[u];
                tf[2 * (blk * C::TBLK + lo * C::TS + hi) + 1] = (float)tt[u];
            }
        }
        if (tid < 72) {
            tT1[tid] = (float)t1v;
            tFV[tid] = (float)fvv;
        }
    };
    // 36 regions x 64 runs of 8 z values (s_lgb) into W buffer b: four lanes
    // per 32-byte run, so one warp instruction reads 8 whole sectors
    auto issue_copies = [&](int b) {
        float *sW = sWb + b * F2pSmem::WTILE;
#pragma unroll 2
        for (int e = tid; e < NREG * 64 * 4; e += NT) {
            const int run = e >> 2, c = e & 3;
            const int dreg = run >> 6, yy = (run >> 3) & 7, xx = run & 7;
            const int reg = DEG ? (dreg / 3) * 6 + f2p_act(DEG, dreg % 3) : dreg;
            const float *src =
                P.S + s_lgb[reg] + (long long)yy * s_lgs[reg][0] + (long long)xx * s_lgs[reg][1] + 2 * c;
            cp_async8(sW + reg * C::REG + yy * C::SY + xx * C::SX + 2 * c, src, pol);
        }
    };
    auto load_ijk = [&](int wi, int (&ijk)[3]) {
        const int rep = rep_of(wi);
        ijk[0] = P.ijk[3 * rep];
        ijk[1] = P.ijk[3 * rep + 1];
        ijk[2] = P.ijk[3 * rep + 2];
    };

    // ---- prologue: item 0 in flight, item 1's copy descriptors ready ----
    const int w0 = blockIdx.x;
    {
        int ijk0[3], ijk1[3] = {0, 0, 0};
        load_ijk(w0, ijk0);
        if (w0 + G < nitems) load_ijk(w0 + G, ijk1);
        setup(w0, ijk0, 0, true, true);
        load_tables(w0, ijk0);
        __syncthreads();
        issue_copies(0);
        cp_async_commit();
        __syncthreads();   // s_lgb consumed
        if (w0 + G < nitems) setup(w0 + G, ijk1, 0, false, true);
    }

    const int item = tid;
    const int loc[3] = {item >> 6, (item >> 3) & 7, item & 7};
#pragma unroll 1
    for (int k = 0;; k++) {
        const int wk = w0 + k * G;
        if (wk >= nitems) break;
        const int c = k & 1;
        const int wn = wk + G;
        __syncthreads();   // B0
        store_tables();
        if (wn < nitems) issue_copies(c ^ 1);
        cp_async_commit();
        // occupied indices of the next two items, needed after B3
        int ijkn[3] = {0, 0, 0}, ijknn[3] = {0, 0, 0};
        if (wn < nitems) load_ijk(wn, ijkn);
        if (tid < 36 && wn + G < nitems) load_ijk(wn + G, ijknn);
        cp_async_wait1();
        __syncthreads();   // B1: W buffer c and the tables are complete

        // ---- one orbit item per thread ----
        const float *sW = sWb + c * F2pSmem::WTILE;
        double e_loc = 0.0, dd_loc = 0.0;
        float2 gres[6];
        {
            int woff[6], toff[6];
#pragma unroll
            for (int pi = 0; pi < 6; pi++) {
                int pp[3] = {0, 0, 0};
                perm_of(pi, pp);
                woff[pi] = loc[pp[1]] * C::SY + loc[pp[0]] * C::SX + loc[pp[2]];
                toff[pi] = loc[pp[0]] * C::TS + loc[pp[1]];
            }
            float t1r[3][3], fvr[3][3];
#pragma unroll
            for (int sr = 0; sr < 3; sr++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    t1r[sr][cc] = tT1[sr * 24 + cc * 8 + loc[cc]];
                    fvr[sr][cc] = tFV[sr * 24 + cc * 8 + loc[cc]];
                }
            double WW[6];
            float VV[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                WW[s] = 0.0;
                VV[s] = 0.f;
            }
#pragma unroll
            for (int tau = 0; tau < 6; tau++) {
                int pt[3] = {0, 0, 0};
                perm_of(tau, pt);
                const int pair = pair_index(pt[0], pt[1]);
#pragma unroll
                for (int s = 0; s < 6; s++) {
                    const int pi = perm_compose(s, tau);
                    int pp[3] = {0, 0, 0};
                    perm_of(pi, pp);
                    const int spair = pair_index(pp[0], pp[1]);
                    const int rw = DEG ? f2p_lead(DEG, tau) : tau;   // the loaded region of (pi, tau)
                    const float w = sW[(pi * 6 + rw) * C::REG + woff[pi]];
                    const float2 ot = tOT[(pair * 6 + spair) * C::TBLK + toff[pi]];
                    WW[s] += (double)w;
                    VV[s] = fmaf(ot.x, t1r[pt[2]][pp[2]], fmaf(ot.y, fvr[pt[2]][pp[2]], VV[s]));
                }
            }
            double X[6];
#pragma unroll
            for (int s = 0; s < 6; s++) X[s] = WW[s] + 0.5 * (double)VV[s];
            double Z[6], RW[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                Z[s] = 4.0 * X[s] + X[perm_compose(s, 4)] + X[perm_compose(s, 3)] -
                       2.0 * (X[perm_compose(s, 5)] + X[perm_compose(s, 1)] + X[perm_compose(s, 2)]);
                RW[s] = 4.0 * WW[s] + WW[perm_compose(s, 4)] + WW[perm_compose(s, 3)] -
                        2.0 * (WW[perm_compose(s, 5)] + WW[perm_compose(s, 1)] + WW[perm_compose(s, 2)]);
            }
            const double Dn = s_eijk[c] - s_ev[c][loc[0]] - s_ev[c][8 + loc[1]] - s_ev[c][16 + loc[2]];
            const double rD = 1.0 / Dn;
            double esum = 0.0;
#pragma unroll
            for (int s = 0; s < 6; s++) esum += WW[s] * Z[s];
            e_loc = CF * esum * rD;
            if (P.want_grad) {
                const double g0 = CF * P.ybar * rD;
                const double ddi = -CF * P.ybar * esum * rD * rD;
#pragma unroll
                for (int s = 0; s < 6; s++)
                    gres[s] = make_float2((float)(g0 * (Z[s] + RW[s])), (float)(g0 * 0.5 * RW[s]));
                dd_loc = ddi;
                // d E / d e_abc = -ddi: a-slot uniform over the warp, b-slot fixed in
                // 8-lane groups, c-slot = lane % 8; per-warp partials, no atomics
                const double da = -ddi;
                double db = da;
#pragma unroll
                for (int off = 4; off > 0; off >>= 1) db += __shfl_xor_sync(0xffffffffu, db, off);
                double dc = da;
                dc += __shfl_xor_sync(0xffffffffu, dc, 8);
                dc += __shfl_xor_sync(0xffffffffu, dc, 16);
                double dsum = db;
                dsum += __shfl_xor_sync(0xffffffffu, dsum, 8);
                dsum += __shfl_xor_sync(0xffffffffu, dsum, 16);
                if (lane == 0) s_evp[warp][0] = dsum;
                if ((lane & 7) == 0) s_evp[warp][1 + (lane >> 3)] = db;
                if (lane < 8) s_evp[warp][5 + lane] = dc;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            e_loc += __shfl_down_sync(0xffffffffu, e_loc, off);
            dd_loc += __shfl_down_sync(0xffffffffu, dd_loc, off);
        }
        if (lane == 0) {
            s_red[0][warp] = e_loc;
            s_red[1][warp] = dd_loc;
        }
        __syncthreads();   // B2: W buffer c fully read; partials visible
        const int ik = s_item[c][0], jk = s_item[c][1], kk = s_item[c][2];
        const int subk = s_item[c][3], repk = s_item[c][4];
        const F2Sub &R = P.sub[subk];
        const int st0 = R.st[0], st1 = R.st[1], st2 = R.st[2];
        if (tid == 0) {
            double es = 0.0, ds = 0.0;
            for (int w = 0; w < NW; w++) {
                es += s_red[0][w];
                ds += s_red[1][w];
            }
            P.e_part[(long long)subk * P.n_ijk + repk] = es;
            if (P.want_grad && ds != 0.0) {
                atomicAdd(&P.mo_bar[ik], ds);
                atomicAdd(&P.mo_bar[jk], ds);
                atomicAdd(&P.mo_bar[kk], ds);
            }
        }
        if (P.want_grad) {
            float2 *sG = reinterpret_cast<float2 *>(sWb + c * F2pSmem::WTILE);
            const int gi = loc[0] * C::RA + loc[1] * C::RB + loc[2] * C::RC;
#pragma unroll
            for (int s = 0; s < 6; s++) sG[s * C::PLANE + gi] = gres[s];
            if (tid >= 64 && tid < 88) {
                // orbital-energy gradient of the item's virtual indices from the
                // per-warp partials: a-slot = warp / 2, b-slot = 4 (warp & 1) + group,
                // c-slot = lane % 8
                const int t = tid - 64;
                double acc = 0.0;
                if (t < 8) {
                    acc = s_evp[2 * t][0] + s_evp[2 * t + 1][0];
                } else if (t < 16) {
                    const int lb = t - 8;
                    for (int w = (lb >> 2); w < NW; w += 2) acc += s_evp[w][1 + (lb & 3)];
                } else {
                    for (int w = 0; w < NW; w++) acc += s_evp[w][5 + t - 16];
                }
                if (acc != 0.0) atomicAdd(&P.mo_bar[o + sel3(st0, st1, st2, t >> 3) + (t & 7)], acc);
            }
        }
        __syncthreads();   // B3: item results visible
        // set-up one item ahead (write-back descriptors, tables) and two ahead (copies)
        if (wn < nitems) {
            setup(wn, ijkn, c ^ 1, true, false);
            load_tables(wn, ijkn);
        }
        if (wn + G < nitems) setup(wn + G, ijknn, 0, false, true);
        if (!P.want_grad) continue;

        // ---- write-back: 72 half regions, one z run per lane (warps 0-1 also
        //      did the set-up above, so they take the shorter share) ----
        const float2 *sG = reinterpret_cast<const float2 *>(sWb + c * F2pSmem::WTILE);
#pragma unroll 1
        for (int hr = NW - 1 - warp; hr < 2 * NREG; hr += NW) {
            const int dreg = hr >> 1, part = hr & 1;
            const int pi = DEG ? dreg / 3 : dreg / 6, rho = DEG ? f2p_act(DEG, dreg % 3) : dreg % 6;
            const int reg = pi * 6 + rho;
            const int rho2 = DEG ? f2p_partner(DEG, rho) : rho;
            const int run = (part << 5) + lane;
            const F2pRegion &rg = s_reg[c][reg];
#define F2P_RUN(PIV)                                                                                                \
    f2p_run<H, PIV, DEG>(P, sG, tOT, tT1, tFV, ik, jk, kk, st0, st1, st2, rho, rho2, lane, run, rg.wb, rg.ws0, rg.ws1, \
                         rg.half, wscf)
            switch (pi) {
            case 0: F2P_RUN(0); break;
            case 1: F2P_RUN(1); break;
            case 2: F2P_RUN(2); break;
            case 3: F2P_RUN(3); break;
            case 4: F2P_RUN(4); break;
            default: F2P_RUN(5); break;
            }
#undef F2P_RUN
        }
    }
    cp_async_wait_all();   // nothing in flight when the CTA retires
}

}  // namespace tb

// Chunk epilogue, common case: one occupied representative with i > j > k
// and three distinct, full 8-wide virtual sub-ranges.  Same math and the same
// outputs as k_f2t (f2.cuh), which keeps every other CTA (repeated occupied
// indices, coinciding or short sub-ranges, the FP64 mode):
//
//   WW(s) = sum_tau w(tau(ijk), tau(s abc)),  VV(s) likewise from v,
//   X = WW + VV/2,  Z = r3(X),  E += 2 sum_s WW Z / D,
//   Wbar(s) = c (Z + r3 WW)/D,  Vbar(s) = c r3(WW)/(2D)   (c = 2 ybar)
// (pyscfad/cc/ccsd_t_slow.py:46-124, pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:64-117).
//
// With nothing degenerate, the 36 regions of the CTA are exactly the pairs
// (sub-range ordering pi, occupied ordering rho), region pi*6 + rho, and each
// raw amplitude belongs to one item and one ordering s; every index map below
// is therefore a compile-time constant once the (s, tau) loops are unrolled.
// Data movement:
//  * the 36 regions are read as 32-byte runs of z values (two 16-byte
//    loads, L2 evict-first: the staging is streamed once) and stored with
//    8-byte shared stores (row stride 70 floats keeps the six permuted item
//    gathers within 2-way bank conflicts);
//  * the V-term factors ovov[p,x,q,y] and t2[q,p,y,x] are read coalesced
//    (y-runs for ovov, x-runs for t2) into dense [pair][sub-range pair][8][8]
//    tables; t1 and fvo for the item are kept in registers;
//  * Wbar leaves as 16-byte runs of fp16/bf16 hi and lo halves (evict-first);
//  * V-term gradients are row sums / column sums in registers and shuffles,
//    added to the FP64 gradients once per run / region, as in k_f2t.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "f2.cuh"
#include "tc_ptx.cuh"

namespace tb {

struct F2sSmem {
    static constexpr int SB = 8;
    static constexpr int SX = 8, SY = 70;           // W tile: (y, x, z) at y*SY + x*SX + z (floats)
    static constexpr int REG = SB * SY;             // 560 floats per region
    // item results {Wbar, Vbar} per ordering s: float2 planes, item (la, lb, lc)
    // at la*RA + lb*RB + lc*RC (strides keep the write-back gathers within
    // 2-way bank conflicts per half-warp)
    static constexpr int RA = 70, RB = 9, RC = 2;
    static constexpr int PLANE = 7 * RA + 7 * RB + 7 * RC + 1;   // 568 float2
    static constexpr int TS = 9;                    // V-term table rows: [pair][sub-range pair][x][y] at x*TS + y
    static constexpr int TBLK = 8 * TS;
    static constexpr int TAB = 36 * TBLK;           // float2 {ovov, t2}
    static constexpr int NT = 256;
    static constexpr size_t BYTES = sizeof(float) * (36 * REG + 2 * TAB + 2 * 3 * 24);
    static_assert(2 * 6 * PLANE <= 36 * REG, "item results overlay the W tile");
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
__host__ __device__ constexpr int f2s_sof(int pi, int rho) {
    int r = 0;
    for (int s = 0; s < 6; s++)
        if (perm_compose(s, rho) == pi) r = s;
    return r;
}

template <int H>   // 1: fp16 hi/lo, 2: bf16 hi/lo
__device__ __forceinline__ void f2s_split8(const float (&w)[8], float scale, uint4 &hi, uint4 &lo) {
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

// Write-back of one region (sub-range ordering PI, occupied ordering rho)
// for the two runs (yy, xx) of a lane: Wbar out, V-term gradients in.
template <int H, int PI>
__device__ __forceinline__ void f2s_region(const F2P<float> &P, const float2 *sG, const float2 *tOT,
                                           const float *tT1, const float *tFV, int i0, int i1, int i2,
                                           const F2Sub &R, int rho, int lane, long long wbase, int ws0, int ws1,
                                           long long half, float wscf) {
    using C = F2sSmem;
    constexpr int pp0 = (PI >> 1), pp1 = (PI & 1) ? ((pp0 == 2) ? 1 : 2) : ((pp0 == 0) ? 1 : 0);
    constexpr int pp2 = 3 - pp0 - pp1;
    constexpr int str[3] = {C::RA, C::RB, C::RC};
    constexpr int spair = 2 * pp0 + (pp1 > pp0 ? pp1 - 1 : pp1);
    // occupied ordering rho: slots (pt0, pt1, pt2) of (p, q, r)
    const int pt0 = rho >> 1;
    const int pt1 = (rho & 1) ? ((pt0 == 2) ? 1 : 2) : ((pt0 == 0) ? 1 : 0);
    const int pt2 = 3 - pt0 - pt1;
    const int s = (rho == 0) ? f2s_sof(PI, 0) : (rho == 1) ? f2s_sof(PI, 1) : (rho == 2) ? f2s_sof(PI, 2)
                : (rho == 3) ? f2s_sof(PI, 3) : (rho == 4) ? f2s_sof(PI, 4) : f2s_sof(PI, 5);
    const int p = sel3(i0, i1, i2, pt0), q = sel3(i0, i1, i2, pt1), r = sel3(i0, i1, i2, pt2);
    const int pair = rho;   // pair_index(pt0, pt1) == rho for an ordering
    const int o = P.d.o, v = P.d.v;
    const float2 *g = sG + s * C::PLANE;
    const float2 *tab = tOT + (pair * 6 + spair) * C::TBLK;
    float a1[8], f1[8];
    {
        // rows of 8 floats at 32-byte aligned offsets: two 16-byte loads each
        const float4 *ra = reinterpret_cast<const float4 *>(tT1 + pt2 * 24 + pp2 * 8);
        const float4 *rf = reinterpret_cast<const float4 *>(tFV + pt2 * 24 + pp2 * 8);
        const float4 a_lo = ra[0], a_hi = ra[1], f_lo = rf[0], f_hi = rf[1];
        a1[0] = a_lo.x; a1[1] = a_lo.y; a1[2] = a_lo.z; a1[3] = a_lo.w;
        a1[4] = a_hi.x; a1[5] = a_hi.y; a1[6] = a_hi.z; a1[7] = a_hi.w;
        f1[0] = f_lo.x; f1[1] = f_lo.y; f1[2] = f_lo.z; f1[3] = f_lo.w;
        f1[4] = f_hi.x; f1[5] = f_hi.y; f1[6] = f_hi.z; f1[7] = f_hi.w;
    }
    float colv[16];
#pragma unroll
    for (int c = 0; c < 16; c++) colv[c] = 0.f;
#pragma unroll
    for (int u = 0; u < 2; u++) {
        const int run = lane + 32 * u;
        const int yy = run >> 3, xx = run & 7;
        const int ib = xx * str[pp0] + yy * str[pp1];
        float wb[8], vb[8];
#pragma unroll
        for (int z = 0; z < 8; z++) {
            const float2 gv = g[ib + z * str[pp2]];
            wb[z] = gv.x;
            vb[z] = gv.y;
        }
        uint4 hi, lo;
        f2s_split8<H>(wb, wscf, hi, lo);
        // 16-byte halves of 32-byte sectors: the partner half comes from the
        // block with the other 8-wide half of this z block, scheduled right
        // next to this one, so the sector completes in L2 (default policy)
        const long long wl = wbase + (long long)yy * ws0 + (long long)xx * ws1;
        uint4 *dst = reinterpret_cast<uint4 *>(reinterpret_cast<uint16_t *>(P.SW) + wl);
        uint4 *dlo = reinterpret_cast<uint4 *>(reinterpret_cast<uint16_t *>(P.SW) + wl + half);
        *dst = hi;
        *dlo = lo;
        const float2 ot = tab[xx * C::TS + yy];
        float rs1 = 0.f, rs2 = 0.f;
#pragma unroll
        for (int z = 0; z < 8; z++) {
            rs1 = fmaf(vb[z], a1[z], rs1);
            rs2 = fmaf(vb[z], f1[z], rs2);
            colv[z] = fmaf(vb[z], ot.x, colv[z]);
            colv[8 + z] = fmaf(vb[z], ot.y, colv[8 + z]);
        }
        const int x = R.st[pp0] + xx, y = R.st[pp1] + yy;
        atomicAdd(&P.ovov_bar[(((long long)p * v + x) * o + q) * v + y], (double)rs1);
        atomicAdd(&P.t2_bar[(((long long)q * o + p) * v + y) * v + x], (double)rs2);
    }
    // column sums over the region's 64 runs: t1_bar[r, z], fvo_bar[z, r]
    const double cv = (double)group_reduce_scatter<16, 32>(colv, lane);
    if (lane < 16) {
        const int z = R.st[pp2] + (lane & 7);
        if (lane < 8) atomicAdd(&P.t1_bar[(long long)r * v + z], cv);
        else atomicAdd(&P.fvo_bar[(long long)z * o + r], cv);
    }
}

template <int H>
__global__ void __launch_bounds__(F2sSmem::NT, 2) k_f2s(F2P<float> P) {
    using C = F2sSmem;
    constexpr int NT = C::NT, NW = NT / 32;
    extern __shared__ __align__(16) uint8_t f2s_smem[];
    float *sW = reinterpret_cast<float *>(f2s_smem);
    float2 *sG = reinterpret_cast<float2 *>(f2s_smem);   // item results [6][PLANE] once W is consumed
    float2 *tOT = reinterpret_cast<float2 *>(sW + 36 * C::REG);
    float *tT1 = reinterpret_cast<float *>(tOT + C::TAB);
    float *tFV = tT1 + 3 * 24;
    __shared__ double s_ev[24], s_evbar[24];
    __shared__ double s_red[2][NW];
    __shared__ long long s_gb[36], s_wb[36];
    __shared__ int s_gs[36][2], s_ws[36][2];
    __shared__ long long s_half[36];

    const Dims &d = P.d;
    const int o = d.o, v = d.v;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // linear grid, sub-range triple fastest: the blocks of one representative
    // run together, so the two 16-byte halves of each Wbar sector meet in L2
    const int sub = P.sub0 + (int)(blockIdx.x % (unsigned)P.nsub_l);
    const int rep = P.rep0 + (int)(blockIdx.x / (unsigned)P.nsub_l);
    const F2Sub &R = P.sub[sub];
    const int ijk[3] = {P.ijk[3 * rep], P.ijk[3 * rep + 1], P.ijk[3 * rep + 2]};
    // scalars needed later, fetched while the tiles load
    const double e_ijk = P.mo_e[ijk[0]] + P.mo_e[ijk[1]] + P.mo_e[ijk[2]];
    const float wscf = P.want_grad ? (float)*P.wscale : 1.0f;

    if (tid < 36) {
        // region pi*6 + rho: staging ordering tau holding the sub-range ordering pi
        const int pi = tid / 6, rho = tid % 6;
        int pp[3], pr[3];
        perm_of(pi, pp);
        perm_of(rho, pr);
        int blk[3];
        for (int c = 0; c < 3; c++) {
            blk[c] = -1;
            for (int t = 0; t < 3; t++)
                if (R.st[c] >= P.ch.base[t] && R.st[c] < P.ch.base[t] + P.ch.nabc[t]) blk[c] = P.ch.blk[t];
        }
        int tau = 0;
        for (; tau < P.ch.nperm - 1; tau++)
            if (P.ch.pb[tau].bx == blk[pp[0]] && P.ch.pb[tau].by == blk[pp[1]] && P.ch.pb[tau].bz == blk[pp[2]])
                break;
        const PermBlock &pb = P.ch.pb[tau];
        const int p = ijk[pr[0]], q = ijk[pr[1]], r = ijk[pr[2]];
        const int xs = R.st[pp[0]] - pb.X0, ys = R.st[pp[1]] - pb.Y0, zs = R.st[pp[2]] - pb.Z0;
        const long long gy = (long long)pb.Tx * o * pb.Tz, gx = (long long)o * pb.Tz;
        s_gb[tid] = pb.soff + (long long)(p * o + q) * pb.Ty * gy + ys * gy + xs * gx + (long long)r * pb.Tz + zs;
        s_gs[tid][0] = (int)gy;
        s_gs[tid][1] = (int)gx;
        const long long wx = (long long)o * pb.rzp, wy = (long long)o * pb.Tx * wx;
        s_wb[tid] = 2 * pb.swoff + (long long)ys * wy + (long long)p * pb.Tx * wx + xs * wx + (long long)q * pb.rzp +
                    (long long)r * pb.Tz + zs;
        s_ws[tid][0] = (int)wy;
        s_ws[tid][1] = (int)wx;
        s_half[tid] = (long long)pb.Ty * o * pb.Tx * o * pb.rzp;
    }
    if (tid < 24) {
        s_ev[tid] = P.mo_e[o + R.st[tid >> 3] + (tid & 7)];
        s_evbar[tid] = 0.0;
    }
    __syncthreads();

    // ---- W tile: 36 regions x 64 runs of 8 z values, asynchronous 8-byte copies
    //      (the staging is streamed once: L2 evict-first) ----
    {
        const uint64_t pol = policy_evict_first();
#pragma unroll 3
        for (int e = tid; e < 36 * 64; e += NT) {
            const int reg = e >> 6, yy = (e >> 3) & 7, xx = e & 7;
            const float *src = P.S + s_gb[reg] + (long long)yy * s_gs[reg][0] + (long long)xx * s_gs[reg][1];
            float *dst = sW + reg * C::REG + yy * C::SY + xx * C::SX;
#pragma unroll
            for (int c = 0; c < 4; c++) cp_async8(dst + 2 * c, src + 2 * c, pol);
        }
    }
    // ---- V-term tables {ovov[p,x,q,y], t2[q,p,y,x]} [pair][sub-range pair][xx][yy]
    //      (distinct sub-ranges only), read while the copies are in flight ----
    {
        constexpr int TB = 9;   // 2304 entries / 256 threads
        double ov[TB], tt[TB];
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int e = tid + u * NT;
            const int pair = e / 384, spair = (e >> 6) % 6, hi = (e >> 3) & 7, lo = e & 7;
            const int sp = pair >> 1, sq = (pair & 1) ? ((sp == 2) ? 1 : 2) : ((sp == 0) ? 1 : 0);
            const int cx = spair >> 1, cy = (spair & 1) ? ((cx == 2) ? 1 : 2) : ((cx == 0) ? 1 : 0);
            const int p = ijk[sp], q = ijk[sq];
            // ovov[p, x, q, y]: lanes along y (hi = xx, lo = yy)
            ov[u] = __ldg(&P.ovov[(((long long)p * v + R.st[cx] + hi) * o + q) * v + R.st[cy] + lo]);
            // t2[q, p, y, x]: lanes along x (hi = yy, lo = xx)
            tt[u] = __ldg(&P.t2[(((long long)q * o + p) * v + R.st[cy] + hi) * v + R.st[cx] + lo]);
        }
        float *tf = reinterpret_cast<float *>(tOT);
#pragma unroll
        for (int u = 0; u < TB; u++) {
            const int e = tid + u * NT;
            const int blk = e >> 6, hi = (e >> 3) & 7, lo = e & 7;
            tf[2 * (blk * C::TBLK + hi * C::TS + lo)] = (float)ov[u];
            tf[2 * (blk * C::TBLK + lo * C::TS + hi) + 1] = (float)tt[u];
        }
    }
    if (tid < 72) {
        const int sr = tid / 24, zl = tid % 24;
        const int z = R.st[zl >> 3] + (zl & 7), r = ijk[sr];
        tT1[tid] = (float)P.t1[(long long)r * v + z];
        tFV[tid] = (float)P.fvo[(long long)z * o + r];
    }
    cp_async_wait_all();
    __syncthreads();

    // ---- orbit items: two per thread ----
    double e_loc = 0.0, dd_loc = 0.0;
    float2 gres[2][6];
#pragma unroll
    for (int it = 0; it < 2; it++) {
        const int item = tid + it * NT;
        const int loc[3] = {item >> 6, (item >> 3) & 7, item & 7};
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
            for (int c = 0; c < 3; c++) {
                t1r[sr][c] = tT1[sr * 24 + c * 8 + loc[c]];
                fvr[sr][c] = tFV[sr * 24 + c * 8 + loc[c]];
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
                const float w = sW[(pi * 6 + tau) * C::REG + woff[pi]];
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
        const double Dn = e_ijk - s_ev[loc[0]] - s_ev[8 + loc[1]] - s_ev[16 + loc[2]];
        const double rD = 1.0 / Dn;
        double esum = 0.0;
#pragma unroll
        for (int s = 0; s < 6; s++) esum += WW[s] * Z[s];
        e_loc += 2.0 * esum * rD;      // orbit weight n_ijk n_abc / 18 = 2
        if (P.want_grad) {
            const double g0 = 2.0 * P.ybar * rD;
            const double ddi = -2.0 * P.ybar * esum * rD * rD;
#pragma unroll
            for (int s = 0; s < 6; s++)
                gres[it][s] = make_float2((float)(g0 * (Z[s] + RW[s])), (float)(g0 * 0.5 * RW[s]));
            dd_loc += ddi;
            // d E / d e_abc = -ddi.  Over a warp the a-slot is uniform, the b-slot
            // is fixed within 8-lane groups and the c-slot is lane % 8: reduce
            // with shuffles first, then one shared atomic per distinct slot.
            double da = -ddi;
            double db = da;
#pragma unroll
            for (int off = 4; off > 0; off >>= 1) db += __shfl_xor_sync(0xffffffffu, db, off);
            double dc = da;
            dc += __shfl_xor_sync(0xffffffffu, dc, 8);
            dc += __shfl_xor_sync(0xffffffffu, dc, 16);
            double dsum = db;
            dsum += __shfl_xor_sync(0xffffffffu, dsum, 8);
            dsum += __shfl_xor_sync(0xffffffffu, dsum, 16);
            if (lane == 0) atomicAdd(&s_evbar[loc[0]], dsum);
            if ((lane & 7) == 0) atomicAdd(&s_evbar[8 + loc[1]], db);
            if (lane < 8) atomicAdd(&s_evbar[16 + loc[2]], dc);
        }
    }

    // ---- block reductions: energy partial, occupied-energy gradient ----
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        e_loc += __shfl_down_sync(0xffffffffu, e_loc, off);
        dd_loc += __shfl_down_sync(0xffffffffu, dd_loc, off);
    }
    if (lane == 0) {
        s_red[0][warp] = e_loc;
        s_red[1][warp] = dd_loc;
    }
    __syncthreads();   // every read of the W tile is done: it becomes the item-result buffer
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
    for (int it = 0; it < 2; it++) {
        const int item = tid + it * NT;
        const int gi = (item >> 6) * C::RA + ((item >> 3) & 7) * C::RB + (item & 7) * C::RC;
#pragma unroll
        for (int c = 0; c < 6; c++) sG[c * C::PLANE + gi] = gres[it][c];
    }
    __syncthreads();
    if (tid < 24 && s_evbar[tid] != 0.0) atomicAdd(&P.mo_bar[o + R.st[tid >> 3] + (tid & 7)], s_evbar[tid]);

    // ---- write back Wbar and add the V-term gradients: one region per warp at a time ----
#pragma unroll 1
    for (int reg = warp; reg < 36; reg += NW) {
        const int pi = reg / 6, rho = reg % 6;
        const long long wbase = s_wb[reg];
        const int ws0 = s_ws[reg][0], ws1 = s_ws[reg][1];
        const long long half = s_half[reg];
#define F2S_REGION(PIV) \
    f2s_region<H, PIV>(P, sG, tOT, tT1, tFV, ijk[0], ijk[1], ijk[2], R, rho, lane, wbase, ws0, ws1, half, wscf)
        switch (pi) {
        case 0: F2S_REGION(0); break;
        case 1: F2S_REGION(1); break;
        case 2: F2S_REGION(2); break;
        case 3: F2S_REGION(3); break;
        case 4: F2S_REGION(4); break;
        default: F2S_REGION(5); break;
        }
#undef F2S_REGION
    }
}

}  // namespace tb

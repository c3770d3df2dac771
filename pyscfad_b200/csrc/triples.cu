// (T) energy and adjoint on B200: planner, layout kernels, chunk epilogue,
// FP64 contraction drivers and the C ABI (include/pyscfad_b200.h).
//
// Reference path replaced: pyscfad/cc/ccsd_t.py:28-192 (forward through
// pyscf's ccsd_t.kernel, backward through ccsd_t_energy_vjp,
// pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-497).
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "gemm_fp64.cuh"
#include "tc_f1.cuh"
#include "f2.cuh"
#include "f2p.cuh"
#include "tc_b1.cuh"
#include "lno.cuh"
#include "pyscfad_b200.h"
#include "triples_internal.h"

namespace tb {

// Thread-local error record; every other setting travels with the call
// (Plan, from triples_options), so concurrent calls do not interfere.
static thread_local int g_last_cuda_error = 0;

#define TB_CUDA(call)                                     \
    do {                                                  \
        cudaError_t _e = (call);                          \
        if (_e != cudaSuccess) {                          \
            g_last_cuda_error = (int)_e;                  \
            return TRIPLES_ERR_CUDA;                      \
        }                                                 \
    } while (0)

#define TB_LAUNCH_CHECK() TB_CUDA(cudaGetLastError())

// ---------------------------------------------------------------------------
// optional per-kernel-class timing with CUDA events (on the launch stream)
// ---------------------------------------------------------------------------
enum ProfCat { P_PREP = 0, P_F1, P_F2, P_B1A, P_B1B, P_B1C, P_B1D, P_FOLD, P_LNO, P_LNO_PROJ, P_LNO_ADJ, P_LNO_VG,
               P_NCAT };
static const char *kProfNames[P_NCAT] = {"prep", "f1_contract", "f2_epilogue",
                                         "b1a_ovvv_grad", "b1b_t2_grad", "b1c_ovoo_grad",
                                         "b1d_t2_ooov_grad", "fold", "lno_tile_fwd", "lno_projection",
                                         "lno_tile_adj", "lno_vgrad"};
struct ProfRec {
    int cat;
    cudaEvent_t a, b;
};
// Profiling records belong to the host thread that enabled them: each
// thread sees only the launches of its own calls.
static thread_local bool g_prof = false;
static thread_local std::vector<ProfRec> g_prof_recs;
static thread_local std::vector<cudaEvent_t> g_event_pool;
static thread_local size_t g_pool_used = 0;

static cudaEvent_t prof_event() {
    if (g_pool_used == g_event_pool.size()) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        g_event_pool.push_back(e);
    }
    return g_event_pool[g_pool_used++];
}

template <typename F>
static void prof_wrap(int cat, cudaStream_t st, F &&launch) {
    cudaEvent_t a = nullptr;
    if (g_prof) {
        a = prof_event();
        cudaEventRecord(a, st);
    }
    launch();
    if (g_prof) {
        cudaEvent_t b = prof_event();
        cudaEventRecord(b, st);
        g_prof_recs.push_back({cat, a, b});
    }
}

#define TB_KLAUNCH(cat, ...)                              \
    do {                                                  \
        prof_wrap((cat), st, [&]() { __VA_ARGS__; });     \
        TB_LAUNCH_CHECK();                                \
    } while (0)

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------
static int choose_tv(int o, int tv_request) {
    int tv = tv_request > 0 ? tv_request : 16;
    if (tv > kMaxTv) tv = kMaxTv;
    while (tv > 1 && tv * o > kMaxCols) tv >>= 1;
    int p2 = 1;   // largest power of two <= tv
    while (p2 * 2 <= tv) p2 *= 2;
    return p2;
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static void make_chunk(const Dims &d, int A, int B, int C, ChunkDesc &ch) {
    const int blks[3] = {A, B, C};
    auto bsize = [&](int b) { return block_size(d, b); };
    for (int t = 0; t < 3; t++) {
        ch.blk[t] = blks[t];
        ch.nabc[t] = bsize(blks[t]);
        ch.base[t] = block_start(d, blks[t]);
    }
    ch.nperm = 0;
    long long off = 0, swoff = 0;
    const long long o3 = (long long)d.o * d.o * d.o;
    for (int s = 0; s < 6; s++) {
        int ps[3];
        perm_of(s, ps);
        int bx = blks[ps[0]], by = blks[ps[1]], bz = blks[ps[2]];
        bool dup = false;
        for (int t = 0; t < ch.nperm; t++)
            if (ch.pb[t].bx == bx && ch.pb[t].by == by && ch.pb[t].bz == bz) dup = true;
        if (dup) continue;
        PermBlock &pb = ch.pb[ch.nperm++];
        pb.bx = bx; pb.by = by; pb.bz = bz;
        pb.X0 = block_start(d, bx); pb.Tx = bsize(bx);
        pb.Y0 = block_start(d, by); pb.Ty = bsize(by);
        pb.Z0 = block_start(d, bz); pb.Tz = bsize(bz);
        pb.soff = off;
        off += (o3 * pb.Tx * pb.Ty * pb.Tz + 15) / 16 * 16;   // 64 B aligned sub-buffers
        pb.rzp = (d.o * pb.Tz + 7) / 8 * 8;
        pb.swoff = swoff;
        swoff += ((long long)pb.Ty * d.o * pb.Tx * d.o * pb.rzp + 15) / 16 * 16;
    }
}

static long long chunk_wbar_elems(const ChunkDesc &ch, const Dims &d) {
    long long s = 0;
    for (int t = 0; t < ch.nperm; t++)
        s += ((long long)ch.pb[t].Ty * d.o * ch.pb[t].Tx * d.o * ch.pb[t].rzp + 15) / 16 * 16;
    return s;
}

static long long chunk_stage_elems(const ChunkDesc &ch, const Dims &d) {
    long long o3 = (long long)d.o * d.o * d.o, s = 0;
    for (int t = 0; t < ch.nperm; t++) s += (o3 * ch.pb[t].Tx * ch.pb[t].Ty * ch.pb[t].Tz + 15) / 16 * 16;
    return s;
}

int make_plan(int precision, int nocc, int nvir, int packed, int want_grad, Plan &P, int lno,
              const triples_options *opt) {
    if (nocc < 1 || nvir < 1 || nocc > kMaxCols || nvir > 32767) return TRIPLES_ERR_INVALID_ARGUMENT;
    if (precision < TRIPLES_PRECISION_FP64 || precision > TRIPLES_PRECISION_MIXED_BF16)
        return TRIPLES_ERR_INVALID_ARGUMENT;
    if (lno && nocc > kLnoMaxO) return TRIPLES_ERR_UNSUPPORTED;
    P = Plan{};
    if (opt) {
        if (opt->block_size < 0 || opt->accumulation_segment < 0 || opt->chunk_a0 < 0)
            return TRIPLES_ERR_INVALID_ARGUMENT;
        P.a0 = opt->chunk_a0;
        P.a1 = opt->chunk_a1;
        P.kseg = opt->accumulation_segment > 0 ? opt->accumulation_segment : 1;
        if (opt->tile_n != 0 && opt->tile_n != 128 && opt->tile_n != 256) return TRIPLES_ERR_INVALID_ARGUMENT;
        P.f1_bn = opt->tile_n;
    } else {
        P.kseg = 1;
    }
    // W-contraction N tile: 256 columns (16 r x 16 z) unless padding nocc to
    // 16 wastes more than a quarter of the r values and 8-wide r tiles waste
    // less (measured at nocc = 40: 256 is 3% faster despite 48 padded r)
    if (P.f1_bn == 0) {
        const int p16 = ((nocc + 15) / 16) * 16, p8 = ((nocc + 7) / 8) * 8;
        P.f1_bn = (4 * p16 > 5 * nocc && p8 < p16) ? 128 : 256;
    }
    P.lno = lno ? 1 : 0;
    P.prec = precision;
    P.want_grad = want_grad ? 1 : 0;
    P.packed = packed ? 1 : 0;
    Dims &d = P.d;
    d.o = nocc;
    d.v = nvir;
    d.n = nocc + nvir;
    d.Tv = choose_tv(nocc, opt ? opt->block_size : 0);
    if (lno) {
        // the projected epilogue keeps whole-chunk FP64 work arrays (6 o^3 Tv^3
        // values each at most): halve the block until they fit the budget
        const double o3 = (double)nocc * nocc * nocc;
        while (d.Tv > 4 && kLnoArrays * 6.0 * o3 * d.Tv * d.Tv * d.Tv * sizeof(double) > kLnoBudgetBytes) d.Tv >>= 1;
    }
    d.Kp = nvir;
    P.Kp8 = (nvir + 7) / 8 * 8;
    P.Op8 = (nocc + 7) / 8 * 8;
    P.nb = num_blocks(d);
    P.n_ijk = nocc * (nocc + 1) * (nocc + 2) / 6;
    long long maxst = 0, maxwb = 0;
    int maxitems = 0;
    for (int A = 0; A < P.nb; A++)
        for (int B = 0; B <= A; B++)
            for (int C = 0; C <= B; C++) {
                ChunkDesc ch;
                make_chunk(d, A, B, C, ch);
                long long s = chunk_stage_elems(ch, d);
                if (s > maxst) maxst = s;
                long long w = chunk_wbar_elems(ch, d);
                if (w > maxwb) maxwb = w;
                int it = ch.nabc[0] * ch.nabc[1] * ch.nabc[2];
                if (it > maxitems) maxitems = it;
            }
    P.stage_elems = (size_t)maxst;
    P.wbar_elems = (size_t)maxwb;
    P.max_items = maxitems;
    P.f2_gy = kMaxSub;
    const bool mixed = precision != TRIPLES_PRECISION_FP64;
    P.stage_bytes = mixed ? sizeof(float) : sizeof(double);

    const size_t o = nocc, v = nvir, Kp = d.Kp;
    const size_t el = sizeof(double);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t at = off; off = align256(off + bytes); return at; };
    P.off_ctrl = take(kCtrlBytes);
    // FP64 operand layouts: only the FP64 contractions read them (the split
    // operands of the mixed modes are built straight from the inputs)
    if (!mixed) {
        P.off_A1 = take(v * o * v * Kp * el);
        P.off_B1 = take(o * o * v * Kp * el);
        P.off_A2 = take(o * o * v * o * el);
        P.off_B2 = take(v * o * v * o * el);
    } else {
        P.off_A1 = P.off_B1 = P.off_A2 = P.off_B2 = 0;
    }
    if (mixed) {
        P.off_A1h = take(2 * v * o * v * P.Kp8 * 2);
        P.off_B1h = take(2 * o * o * v * P.Kp8 * 2);
        P.off_A2h = take(2 * o * o * v * P.Op8 * 2);
        P.off_B2h = take(2 * v * o * v * P.Op8 * 2);
    }
    P.off_S = take(P.stage_elems * P.stage_bytes);
    if (want_grad) {
        P.off_SW = take(P.wbar_elems * (mixed ? 4 : 8));
        P.off_GA1 = take(v * o * v * Kp * el);
        P.off_GB1 = take(o * o * v * Kp * el);
        P.off_GA2 = take(o * o * v * o * el);
        P.off_GB2 = take(v * o * v * o * el);
    }
    P.off_ijk = take((size_t)P.n_ijk * 3 * sizeof(int));
    P.off_epart = take((size_t)P.n_ijk * P.f2_gy * el);
    if (P.lno) {
        // whole-chunk FP64 arrays: WW / P^T(Wtbar) / vbar (0), Pt(Q) (1), Q / Dbar (2),
        // Zbar (3); the energy alone needs only 0 and 2
        P.off_L[0] = take(P.stage_elems * el);
        P.off_L[2] = take(P.stage_elems * el);
        if (want_grad) {
            P.off_L[1] = take(P.stage_elems * el);
            P.off_L[3] = take(P.stage_elems * el);
        } else {
            P.off_L[1] = P.off_L[0];
            P.off_L[3] = P.off_L[2];
        }
        P.off_lpart = take((size_t)6 * kLnoGrid * el);
    }
    P.total = off;
    return TRIPLES_OK;
}

// ---------------------------------------------------------------------------
// layout kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long tri_index(int f, int y) {
    return f >= y ? (long long)f * (f + 1) / 2 + y : (long long)y * (y + 1) / 2 + f;
}

// A1[y][p][x][f] = ovvv[p,x,f,y]  (packed: unpacked symmetric [f,y] block)
__global__ void k_prep_A1(const double *__restrict__ ovvv, int packed, Dims d,
                          double *__restrict__ A1) {
    __shared__ double tile[32][33];
    const long long px = blockIdx.z;  // p*v + x
    const int f0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const long long npair = (long long)d.v * (d.v + 1) / 2;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int f = f0 + r, y = y0 + threadIdx.x;
        double val = 0.0;
        if (f < d.v && y < d.v)
            val = packed ? ovvv[px * npair + tri_index(f, y)] : ovvv[(px * d.v + f) * d.v + y];
        tile[r][threadIdx.x] = val;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int y = y0 + r, f = f0 + threadIdx.x;
        if (y < d.v && f < d.Kp)
            A1[((long long)y * d.o * d.v + px) * d.Kp + f] = tile[threadIdx.x][r];
    }
}

// B1[q][r][z][f] = t2[r,q,z,f]
__global__ void k_prep_B1(const double *__restrict__ t2, Dims d, double *__restrict__ B1) {
    const long long row = blockIdx.x;  // (q*o + r)*v + z
    const int z = row % d.v;
    const int qr = row / d.v;
    const int r = qr % d.o, q = qr / d.o;
    const double *src = t2 + (((long long)r * d.o + q) * d.v + z) * d.v;
    for (int f = threadIdx.x; f < d.Kp; f += blockDim.x)
        B1[row * d.Kp + f] = f < d.v ? src[f] : 0.0;
}

// A2[q][p][x][m] = ovoo[p,x,m,q]
__global__ void k_prep_A2(const double *__restrict__ ovoo, Dims d, double *__restrict__ A2) {
    const long long total = (long long)d.o * d.o * d.v * d.o;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = e % d.o;
        long long t = e / d.o;
        int x = t % d.v;
        t /= d.v;
        int p = t % d.o;
        int q = t / d.o;
        A2[e] = ovoo[(((long long)p * d.v + x) * d.o + m) * d.o + q];
    }
}

// B2[y][r][z][m] = t2[r,m,z,y]
__global__ void k_prep_B2(const double *__restrict__ t2, Dims d, double *__restrict__ B2) {
    const long long total = (long long)d.v * d.o * d.v * d.o;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = e % d.o;
        long long t = e / d.o;
        int z = t % d.v;
        t /= d.v;
        int r = t % d.o;
        int y = t / d.o;
        B2[e] = t2[(((long long)r * d.o + m) * d.v + z) * d.v + y];
    }
}

// ---------------------------------------------------------------------------
// 16-bit split operands for the tensor-core path
// ---------------------------------------------------------------------------
// Occupied representatives i >= j >= k: first the o(o-1)(o-2)/6 with
// i > j > k (combinatorial order), then the o(o-1)/2 with i == j > k, as
// many with i > j == k, and the o with i == j == k, so that each pattern the
// persistent epilogue takes (the first three) is one contiguous range.
__host__ __device__ inline int n_distinct_ijk(int o) { return o * (o - 1) * (o - 2) / 6; }

__global__ void k_ijk_table(int o, int *ijk) {
    const int n = o * (o + 1) * (o + 2) / 6, nd = n_distinct_ijk(o), np = o * (o - 1) / 2;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int i, j, k;
        if (r < nd) {
            i = 2;
            while ((i + 1) * i * (i - 1) / 6 <= r) i++;   // largest i with C(i,3) <= r
            int rem = r - i * (i - 1) * (i - 2) / 6;
            j = 1;
            while ((j + 1) * j / 2 <= rem) j++;             // largest j with C(j,2) <= rem
            k = rem - j * (j - 1) / 2;
        } else {
            int t = r - nd;
            const int kind = t < np ? 0 : (t < 2 * np ? 1 : 2);
            t -= kind * np;
            if (kind == 2) {
                i = j = k = t;
            } else {
                int a = 1;
                while ((a + 1) * a / 2 <= t) a++;           // pair a > b, b = t - C(a,2)
                const int b = t - a * (a - 1) / 2;
                i = a;
                j = kind == 0 ? a : b;
                k = b;
            }
        }
        ijk[3 * r] = i;
        ijk[3 * r + 1] = j;
        ijk[3 * r + 2] = k;
    }
}

__global__ void k_absmax(const double *__restrict__ x, long long n, unsigned long long *out) {
    double m = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[e]));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ double pow2_scale(double m) {
    // largest power of two s with m * s < 2^14 (fp16 keeps headroom below 65504)
    if (!(m > 0.0) || !isfinite(m)) return 1.0;
    int e;
    frexp(m, &e);   // m < 2^e
    return ldexp(1.0, 14 - e);
}

__global__ void k_make_scales(Ctrl *ctrl, int scaled) {
    const double a = fmax(__longlong_as_double((long long)ctrl->absmax[0]),
                          __longlong_as_double((long long)ctrl->absmax[1]));
    const double b = __longlong_as_double((long long)ctrl->absmax[2]);
    const double sA = scaled ? pow2_scale(a) : 1.0;
    const double sB = scaled ? pow2_scale(b) : 1.0;
    ctrl->scale[0] = sA;
    ctrl->scale[1] = sB;
    ctrl->out_scale = (float)(1.0 / (sA * sB));
}

// Per-chunk power-of-two scale for the split Wbar, from a bound that needs no
// pass over Wbar:  |Wbar| <= 2|ybar| (144 max|w| + 36 max|v|) / min|D| over the
// chunk (|Z| <= 12 max|X|, |X| <= 6 max|w| + 3 max|v|, |R WW| <= 72 max|w|,
// orbit weight <= 2).  Resets the running max |w| for the next chunk.
__device__ __forceinline__ void chunk_scale_body(Ctrl *ctrl, const double *__restrict__ mo_e, int o, int a0,
                                                 int na, int b0, int nb, int c0, int nc, double ybar, int scaled,
                                                 int lno) {
    __shared__ double s_min[3], s_maxo;
    const double inf = 1e300;
    if (threadIdx.x < 4) {
        double m = (threadIdx.x < 3) ? inf : -inf;
        const int st = threadIdx.x == 0 ? a0 : (threadIdx.x == 1 ? b0 : c0);
        const int n = threadIdx.x == 0 ? na : (threadIdx.x == 1 ? nb : nc);
        if (threadIdx.x < 3) {
            for (int t = 0; t < n; t++) m = fmin(m, mo_e[o + st + t]);
            s_min[threadIdx.x] = m;
        } else {
            for (int t = 0; t < o; t++) m = fmax(m, mo_e[t]);
            s_maxo = m;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double dmin = s_min[0] + s_min[1] + s_min[2] - 3.0 * s_maxo;
        const double mw = (double)__uint_as_float(ctrl->wmax_bits);
        const double mv = __longlong_as_double((long long)ctrl->absmax[3]) * __longlong_as_double((long long)ctrl->absmax[4]) +
                          __longlong_as_double((long long)ctrl->absmax[2]) * __longlong_as_double((long long)ctrl->absmax[5]);
        // |wbar| <= 6 |WWbar|; with the LNO projector (row / column abs sums nr, nc)
        // WWbar = P^T(ybar Q / 3) + r3^T(ybar P(WW) / (3 D)), |Q| <= 12 (6 mw + 3 mv) / dmin;
        // nr = nc = 1 is the canonical bound
        const double nr = lno ? ctrl->lno_norm[0] : 1.0, ncl = lno ? ctrl->lno_norm[1] : 1.0;
        double bound = 2.0 * fabs(ybar) * (72.0 * (nr + ncl) * mw + 36.0 * nr * mv) / (dmin > 1e-300 ? dmin : 1e-300);
        ctrl->wscale = scaled ? pow2_scale(bound) : 1.0;
        ctrl->wmax_bits = 0u;
    }
}

__global__ void k_chunk_scale(Ctrl *ctrl, const double *__restrict__ mo_e, int o, int a0, int na, int b0,
                              int nb, int c0, int nc, double ybar, int scaled, int lno) {
    chunk_scale_body(ctrl, mo_e, o, a0, na, b0, nb, c0, nc, ybar, scaled, lno);
}

// Per problem of a batched chunk step: the chunk's virtual ranges for the
// Wbar scale, and the energy partials of its epilogue.
struct ChunkAux {
    Ctrl *ctrl;
    const double *mo_e;
    const double *e_part;
    double ybar;
    int o, a0, na, b0, nb, c0, nc, n_part;
};

// one 32-thread block per problem
__global__ void k_chunk_scale_batch(const ChunkAux *__restrict__ aux, int scaled) {
    const ChunkAux &A = aux[blockIdx.x];
    chunk_scale_body(A.ctrl, A.mo_e, A.o, A.a0, A.na, A.b0, A.nb, A.c0, A.nc, A.ybar, scaled, 0);
}

// one 256-thread block per problem: the chunk's energy partials, fixed order
__global__ void k_energy_sum_batch(const ChunkAux *__restrict__ aux) {
    const ChunkAux &A = aux[blockIdx.x];
    energy_sum_body(A.e_part, A.n_part, &A.ctrl->e_acc);
}

template <typename H>
__device__ __forceinline__ void split16(double xs, H &hi, H &lo);
template <>
__device__ __forceinline__ void split16<__half>(double xs, __half &hi, __half &lo) {
    hi = __double2half(xs);
    lo = __double2half(xs - (double)__half2float(hi));
}
template <>
__device__ __forceinline__ void split16<__nv_bfloat16>(double xs, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __double2bfloat16(xs);
    lo = __double2bfloat16(xs - (double)__bfloat162float(hi));
}

// A1h[h][y][p][x][f] = split(ovvv[p,x,f,y] * sA), f < Kp8 (zero beyond v)
// max abs row sum and max abs column sum of the LNO projector mat[o,o]
__global__ void k_lno_mat_norms(const double *__restrict__ mat, int o, Ctrl *ctrl) {
    __shared__ double s_r[kLnoMaxO], s_c[kLnoMaxO];
    for (int i = threadIdx.x; i < o; i += blockDim.x) {
        double r = 0.0, c = 0.0;
        for (int k = 0; k < o; k++) {
            r += fabs(mat[i * o + k]);
            c += fabs(mat[k * o + i]);
        }
        s_r[i] = r;
        s_c[i] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mr = 0.0, mc = 0.0;
        for (int i = 0; i < o; i++) {
            mr = fmax(mr, s_r[i]);
            mc = fmax(mc, s_c[i]);
        }
        ctrl->lno_norm[0] = mr;
        ctrl->lno_norm[1] = mc;
    }
}

template <typename H>
__global__ void k_prep_A1h(const double *__restrict__ ovvv, int packed, Dims d, int Kp8,
                           const Ctrl *ctrl, H *__restrict__ out) {
    __shared__ double tile[32][33];
    const long long px = blockIdx.z;
    const int f0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    const long long npair = (long long)d.v * (d.v + 1) / 2;
    const double sA = ctrl->scale[0];
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int f = f0 + r, y = y0 + threadIdx.x;
        double val = 0.0;
        if (f < d.v && y < d.v)
            val = packed ? ovvv[px * npair + tri_index(f, y)] : ovvv[(px * d.v + f) * d.v + y];
        tile[r][threadIdx.x] = val;
    }
    __syncthreads();
    const long long half = (long long)d.v * d.o * d.v * Kp8;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int y = y0 + r, f = f0 + threadIdx.x;
        if (y < d.v && f < Kp8) {
            H hi, lo;
            split16<H>(tile[threadIdx.x][r] * sA, hi, lo);
            const long long e = ((long long)y * d.o * d.v + px) * Kp8 + f;
            out[e] = hi;
            out[half + e] = lo;
        }
    }
}

// B1h[h][q][r][z][f] = split(t2[r,q,z,f] * sB)
template <typename H>
__global__ void k_prep_B1h(const double *__restrict__ t2, Dims d, int Kp8, const Ctrl *ctrl,
                           H *__restrict__ out) {
    const long long row = blockIdx.x;  // (q*o + r)*v + z
    const int z = row % d.v;
    const int qr = row / d.v;
    const int r = qr % d.o, q = qr / d.o;
    const double *src = t2 + (((long long)r * d.o + q) * d.v + z) * d.v;
    const double sB = ctrl->scale[1];
    const long long half = (long long)d.o * d.o * d.v * Kp8;
    for (int f = threadIdx.x; f < Kp8; f += blockDim.x) {
        H hi, lo;
        split16<H>(f < d.v ? src[f] * sB : 0.0, hi, lo);
        out[row * Kp8 + f] = hi;
        out[half + row * Kp8 + f] = lo;
    }
}

// A2h[h][q][p][x][m] = split(-ovoo[p,x,m,q] * sA), m < Op8
template <typename H>
__global__ void k_prep_A2h(const double *__restrict__ ovoo, Dims d, int Op8, const Ctrl *ctrl,
                           H *__restrict__ out) {
    const long long total = (long long)d.o * d.o * d.v * Op8;
    const double sA = ctrl->scale[0];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = e % Op8;
        long long t = e / Op8;
        int x = t % d.v;
        t /= d.v;
        int p = t % d.o;
        int q = t / d.o;
        double val = m < d.o ? -ovoo[(((long long)p * d.v + x) * d.o + m) * d.o + q] * sA : 0.0;
        H hi, lo;
        split16<H>(val, hi, lo);
        out[e] = hi;
        out[total + e] = lo;
    }
}

// B2h[h][y][r][z][m] = split(t2[r,m,z,y] * sB), m < Op8
template <typename H>
__global__ void k_prep_B2h(const double *__restrict__ t2, Dims d, int Op8, const Ctrl *ctrl,
                           H *__restrict__ out) {
    const long long total = (long long)d.v * d.o * d.v * Op8;
    const double sB = ctrl->scale[1];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int m = e % Op8;
        long long t = e / Op8;
        int z = t % d.v;
        t /= d.v;
        int r = t % d.o;
        int y = t / d.o;
        double val = m < d.o ? t2[(((long long)r * d.o + m) * d.v + z) * d.v + y] * sB : 0.0;
        H hi, lo;
        split16<H>(val, hi, lo);
        out[e] = hi;
        out[total + e] = lo;
    }
}

// ---------------------------------------------------------------------------
// FP64 contraction kernels (one GEMM problem per blockIdx.z)
// ---------------------------------------------------------------------------
template <typename StageT>
struct GemmLaunch {
    Dims d;
    ChunkDesc ch;
    int cum[7];      // prefix sums used to decode blockIdx.z
    const double *A1, *B1, *A2, *B2;
    StageT *S;       // staging
    double *G;       // gradient target
};

template <typename StageT>
__device__ __forceinline__ int find_tau(const GemmLaunch<StageT> &L, int b) {
    int t = 0;
    while (t + 1 < L.ch.nperm && b >= L.cum[t + 1]) t++;
    return t;
}

// F1: S_tau[p][q][y][x][r][z] = W for all (tau, y, q)
__global__ void __launch_bounds__(256) k_f1_fp64(GemmLaunch<double> L) {
    __shared__ GemmSmem sm;
    const int b = blockIdx.z;
    const int t = find_tau(L, b);
    const PermBlock &pb = L.ch.pb[t];
    const Dims &d = L.d;
    const int o = d.o, v = d.v, Kp = d.Kp;
    const int rem = b - L.cum[t];
    const int y = rem / o, q = rem % o;
    const long long yg = pb.Y0 + y;
    const long long oTz = (long long)o * pb.Tz;
    GemmArgs g;
    g.M = o * pb.Tx;
    g.N = o * pb.Tz;
    g.K = v;
    g.K2 = o;
    g.A = GOp{L.A1 + (yg * o * v + pb.X0) * Kp, map2(pb.Tx, Kp, (long long)v * Kp), map1(1), 1};
    g.B = GOp{L.B1 + ((long long)q * o * v + pb.Z0) * Kp, map2(pb.Tz, Kp, (long long)v * Kp), map1(1), 1};
    g.A2 = GOp{L.A2 + ((long long)q * o * v + pb.X0) * o, map2(pb.Tx, o, (long long)v * o), map1(1), 1};
    g.B2 = GOp{L.B2 + (yg * o * v + pb.Z0) * o, map2(pb.Tz, o, (long long)v * o), map1(1), 1};
    g.C = L.S + pb.soff + (long long)q * pb.Ty * pb.Tx * oTz + (long long)y * pb.Tx * oTz;
    g.cm = map2(pb.Tx, oTz, (long long)o * pb.Ty * pb.Tx * oTz);
    g.cn = map1(1);
    g.alpha = 1.0;
    g.alpha2 = -1.0;
    g.accumulate = 0;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// ovvv gradient: G_A1[y][p][x][f] += sum_{q,r,z} Wbar * B1[q][r][z][f]; z = (tau, y)
template <typename StageT>
__global__ void __launch_bounds__(256) k_b1a_fp64(GemmLaunch<StageT> L) {
    __shared__ GemmSmem sm;
    const int b = blockIdx.z;
    const int t = find_tau(L, b);
    const PermBlock &pb = L.ch.pb[t];
    const Dims &d = L.d;
    const int o = d.o, v = d.v, Kp = d.Kp;
    const int y = b - L.cum[t];
    const long long oTz = (long long)o * pb.Tz;
    GemmArgsT<StageT> g;
    g.M = o * pb.Tx;
    g.N = v;
    g.K = o * o * pb.Tz;
    g.K2 = 0;
    const long long s_r = pb.Tz, s_q = pb.rzp, s_x = (long long)o * pb.rzp;
    const long long s_p = (long long)pb.Tx * s_x, s_y = (long long)o * s_p;
    (void)s_r;
    g.A = GOpT<StageT>{L.S + pb.swoff + (long long)y * s_y, map2(pb.Tx, s_x, s_p), map2((int)oTz, 1, s_q), 1};
    g.B = GOp{L.B1 + (long long)pb.Z0 * Kp, map1(1),
              map3(pb.Tz, o, Kp, (long long)v * Kp, (long long)o * v * Kp), 0};
    g.C = L.G + (((long long)pb.Y0 + y) * o * v + pb.X0) * Kp;
    g.cm = map2(pb.Tx, Kp, (long long)v * Kp);
    g.cn = map1(1);
    g.alpha = 1.0;
    g.alpha2 = 0.0;
    g.accumulate = 1;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// t2 gradient (ovvv term): G_B1[q][r][z][f] += sum_{y,p,x} Wbar * A1[y][p][x][f]; z = q
template <typename StageT>
__global__ void __launch_bounds__(256) k_b1b_fp64(GemmLaunch<StageT> L) {
    __shared__ GemmSmem sm;
    // grid.z = (ordering, q): all orderings of the chunk in one launch; orderings
    // that share a block write the same gradient rows, hence the atomic adds
    const int q = blockIdx.z % L.d.o;
    const PermBlock &pb = L.ch.pb[blockIdx.z / L.d.o];
    const Dims &d = L.d;
    const int o = d.o, v = d.v, Kp = d.Kp;
    GemmArgsT<StageT> g;
    g.M = o * pb.Tz;
    g.N = v;
    g.K = pb.Ty * o * pb.Tx;
    g.K2 = 0;
    const long long s_r = pb.Tz, s_q = pb.rzp, s_x = (long long)o * pb.rzp;
    const long long s_p = (long long)pb.Tx * s_x, s_y = (long long)o * s_p;
    (void)s_r;
    g.A = GOpT<StageT>{L.S + pb.swoff + (long long)q * s_q, map1(1), map3(pb.Tx, o, s_x, s_p, s_y), 0};
    g.B = GOp{L.A1 + ((long long)pb.Y0 * o * v + pb.X0) * Kp, map1(1),
              map3(pb.Tx, o, Kp, (long long)v * Kp, (long long)o * v * Kp), 0};
    g.C = L.G + ((long long)q * o * v + pb.Z0) * Kp;
    g.cm = map2(pb.Tz, Kp, (long long)v * Kp);
    g.cn = map1(1);
    g.alpha = 1.0;
    g.alpha2 = 0.0;
    g.accumulate = 2;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// ovoo gradient: G_A2[q][p][x][m] -= sum_{y,r,z} Wbar * B2[y][r][z][m]; z = q
template <typename StageT>
__global__ void __launch_bounds__(256) k_b1c_fp64(GemmLaunch<StageT> L) {
    __shared__ GemmSmem sm;
    // grid.z = (ordering, q): all orderings of the chunk in one launch; orderings
    // that share a block write the same gradient rows, hence the atomic adds
    const int q = blockIdx.z % L.d.o;
    const PermBlock &pb = L.ch.pb[blockIdx.z / L.d.o];
    const Dims &d = L.d;
    const int o = d.o, v = d.v;
    const long long oTz = (long long)o * pb.Tz;
    GemmArgsT<StageT> g;
    g.M = o * pb.Tx;
    g.N = o;
    g.K = pb.Ty * o * pb.Tz;
    g.K2 = 0;
    const long long s_r = pb.Tz, s_q = pb.rzp, s_x = (long long)o * pb.rzp;
    const long long s_p = (long long)pb.Tx * s_x, s_y = (long long)o * s_p;
    (void)s_r;
    g.A = GOpT<StageT>{L.S + pb.swoff + (long long)q * s_q, map2(pb.Tx, s_x, s_p), map2((int)oTz, 1, s_y), 1};
    g.B = GOp{L.B2 + ((long long)pb.Y0 * o * v + pb.Z0) * o, map1(1),
              map3(pb.Tz, o, o, (long long)v * o, (long long)o * v * o), 0};
    g.C = L.G + ((long long)q * o * v + pb.X0) * o;
    g.cm = map2(pb.Tx, o, (long long)v * o);
    g.cn = map1(1);
    g.alpha = -1.0;
    g.alpha2 = 0.0;
    g.accumulate = 2;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// t2 gradient (ooov term): G_B2[y][r][z][m] -= sum_{q,p,x} Wbar * A2[q][p][x][m]; z = (tau, y)
template <typename StageT>
__global__ void __launch_bounds__(256) k_b1d_fp64(GemmLaunch<StageT> L) {
    __shared__ GemmSmem sm;
    const int b = blockIdx.z;
    const int t = find_tau(L, b);
    const PermBlock &pb = L.ch.pb[t];
    const Dims &d = L.d;
    const int o = d.o, v = d.v;
    const int y = b - L.cum[t];
    GemmArgsT<StageT> g;
    g.M = o * pb.Tz;
    g.N = o;
    g.K = o * o * pb.Tx;
    g.K2 = 0;
    const long long s_r = pb.Tz, s_q = pb.rzp, s_x = (long long)o * pb.rzp;
    const long long s_p = (long long)pb.Tx * s_x, s_y = (long long)o * s_p;
    (void)s_r;
    g.A = GOpT<StageT>{L.S + pb.swoff + (long long)y * s_y, map1(1), map3(pb.Tx, o, s_x, s_p, s_q), 0};
    g.B = GOp{L.A2 + (long long)pb.X0 * o, map1(1),
              map3(pb.Tx, o, o, (long long)v * o, (long long)o * v * o), 0};
    g.C = L.G + (((long long)pb.Y0 + y) * o * v + pb.Z0) * o;
    g.cm = map2(pb.Tz, o, (long long)v * o);
    g.cn = map1(1);
    g.alpha = -1.0;
    g.alpha2 = 0.0;
    g.accumulate = 1;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// ---------------------------------------------------------------------------
// V-term gradients from Vbar: ovov, t2 (row dots), t1, fvo (column sums)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// gradient fold back to the reference layouts
// ---------------------------------------------------------------------------
// full ovvv_bar[p,x,f,y] = G_A1[y][p][x][f]
__global__ void k_fold_ovvv_full(const double *__restrict__ GA1, Dims d, double *__restrict__ out) {
    __shared__ double tile[32][33];
    const long long px = blockIdx.z;
    const int y0 = blockIdx.x * 32, f0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int y = y0 + r, f = f0 + threadIdx.x;
        tile[r][threadIdx.x] = (y < d.v && f < d.v) ? GA1[((long long)y * d.o * d.v + px) * d.Kp + f] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int f = f0 + r, y = y0 + threadIdx.x;
        if (f < d.v && y < d.v) out[(px * d.v + f) * d.v + y] = tile[threadIdx.x][r];
    }
}

// packed ovvv_bar[p,x,tri(f,y)] = G[f,y] + G[y,f] (f != y), G[f,f]; G[f,y] = G_A1[y][p][x][f]
// (pyscfad/cc/ccsd_t.py:184-191)
__global__ void k_fold_ovvv_packed(const double *__restrict__ GA1, Dims d, double *__restrict__ out) {
    const long long npair = (long long)d.v * (d.v + 1) / 2;
    const long long total = (long long)d.o * d.v * npair;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long px = e / npair;
        const long long ij = e % npair;
        int f = (int)((sqrt(8.0 * (double)ij + 1.0) - 1.0) * 0.5);
        while ((long long)f * (f + 1) / 2 > ij) f--;
        while ((long long)(f + 1) * (f + 2) / 2 <= ij) f++;
        const int y = (int)(ij - (long long)f * (f + 1) / 2);
        const long long sy = (long long)d.o * d.v * d.Kp;
        double val = GA1[y * sy + px * d.Kp + f];
        if (f != y) val += GA1[(long long)f * sy + px * d.Kp + y];
        out[e] = val;
    }
}

// t2_bar[r,q,z,f] += G_B1[q][r][z][f] + G_B2[f][r][z][q]
__global__ void k_fold_t2(const double *__restrict__ GB1, const double *__restrict__ GB2, Dims d,
                          double *__restrict__ t2_bar) {
    const long long total = (long long)d.o * d.o * d.v * d.v;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int f = e % d.v;
        long long t = e / d.v;
        const int z = t % d.v;
        t /= d.v;
        const int q = t % d.o;
        const int r = t / d.o;
        t2_bar[e] += GB1[(((long long)q * d.o + r) * d.v + z) * d.Kp + f] +
                     GB2[(((long long)f * d.o + r) * d.v + z) * d.o + q];
    }
}

// ovoo_bar[p,x,m,q] = G_A2[q][p][x][m]
__global__ void k_fold_ovoo(const double *__restrict__ GA2, Dims d, double *__restrict__ out) {
    const long long total = (long long)d.o * d.v * d.o * d.o;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int q = e % d.o;
        long long t = e / d.o;
        const int m = t % d.o;
        t /= d.o;
        const int x = t % d.v;
        const int p = t / d.v;
        out[e] = GA2[(((long long)q * d.o + p) * d.v + x) * d.o + m];
    }
}

__global__ void k_copy_scalar(const double *src, double *dst) { dst[0] = src[0]; }

// plain FP64 GEMM through the multi-index tile (DF factor products)
__global__ void __launch_bounds__(256) k_gemm_plain(GemmArgs g) {
    __shared__ GemmSmem sm;
    const int m0 = blockIdx.x * kGBM, n0 = blockIdx.y * kGBN;
    if (m0 >= g.M || n0 >= g.N) return;
    gemm_fp64_tile(g, m0, n0, sm);
}

// C[m*cms + n*cns] = sum_k A[m*ams + k*aks] B[n*bms + k*bks]
int gemm_plain(cudaStream_t st, int M, int N, int K, const double *A, long long ams, long long aks,
               const double *B, long long bms, long long bks, double *C, long long cms, long long cns) {
    GemmArgs g;
    g.M = M;
    g.N = N;
    g.K = K;
    g.K2 = 0;
    g.A = GOp{A, map1(ams), map1(aks), aks == 1 ? 1 : 0};
    g.B = GOp{B, map1(bms), map1(bks), bks == 1 ? 1 : 0};
    g.A2 = g.A;
    g.B2 = g.B;
    g.C = C;
    g.cm = map1(cms);
    g.cn = map1(cns);
    g.alpha = 1.0;
    g.alpha2 = 0.0;
    g.accumulate = 0;
    const dim3 grid((unsigned)((M + kGBM - 1) / kGBM), (unsigned)((N + kGBN - 1) / kGBN));
    if (grid.y > 65535) return TRIPLES_ERR_UNSUPPORTED;
    TB_KLAUNCH(P_PREP, k_gemm_plain<<<grid, 256, 0, st>>>(g));
    return TRIPLES_OK;
}

// ---------------------------------------------------------------------------
// driver
// ---------------------------------------------------------------------------
static inline unsigned grid1d(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    if (b > 148 * 64) b = 148 * 64;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// ---- tensor maps (driver entry point fetched through the runtime) ----
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

static EncodeTiledFn lookup_encode_fn() {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        return (EncodeTiledFn)ptr;
    return nullptr;
}

static EncodeTiledFn get_encode_fn() {
    static const EncodeTiledFn fn = lookup_encode_fn();   // initialised once, thread-safe
    return fn;
}

// 5-D map over a [2][d3][d2][d1][d0] 16-bit array (d0 innermost), 128B swizzle.
static int make_tmap5(CUtensorMap *tm, void *base, bool bf16, const uint64_t dims[5], const uint32_t box[5]) {
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return TRIPLES_ERR_UNSUPPORTED;
    cuuint64_t gdim[5], gstr[4];
    uint64_t stride = 2;
    for (int i = 0; i < 5; i++) {
        gdim[i] = dims[i];
        if (i < 4) {
            stride *= dims[i];
            gstr[i] = stride;
        }
    }
    cuuint32_t bx[5], es[5] = {1, 1, 1, 1, 1};
    for (int i = 0; i < 5; i++) bx[i] = box[i];
    CUresult r = enc(tm, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 5, base, gdim,
                     gstr, bx, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? TRIPLES_OK : TRIPLES_ERR_CUDA;
}

// 5-D map over S_tau, an FP32 [p][q][y][x][rz] array (rz innermost, o*16 values),
// used by the W-contraction epilogue to store 32 x 32 pieces; 128B swizzle.
static int make_tmap_stage(CUtensorMap *tm, float *base, int o, int Tx, int Ty) {
    EncodeTiledFn enc = get_encode_fn();
    if (!enc) return TRIPLES_ERR_UNSUPPORTED;
    const cuuint64_t gdim[5] = {(cuuint64_t)o * 16, (cuuint64_t)Tx, (cuuint64_t)Ty, (cuuint64_t)o, (cuuint64_t)o};
    cuuint64_t gstr[4];
    gstr[0] = gdim[0] * sizeof(float);
    for (int i = 1; i < 4; i++) gstr[i] = gstr[i - 1] * gdim[i];
    const cuuint32_t box[5] = {32, 16, 1, 1, 2}, es[5] = {1, 1, 1, 1, 1};
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, gdim, gstr, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? TRIPLES_OK : TRIPLES_ERR_CUDA;
}

// SM count of the current device (cached per device; the first writers
// store the same value, so relaxed atomics suffice).
constexpr int kMaxDev = 64;
static std::atomic<int> g_num_sms[kMaxDev];

static int num_sms() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return 148;
    int n = g_num_sms[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        g_num_sms[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

// One-time set-up per device and kind of work (shared-memory opt-ins and
// constant tables), under a lock so that host threads making their first
// call at the same time do it once.  Assumes the device's primary context
// lives as long as the process (a cudaDeviceReset would need it again).
enum InitKind { INIT_F2_F32 = 0, INIT_F2_F64, INIT_TC, INIT_LNO, INIT_NKINDS };
static std::mutex g_init_mu;
static bool g_init_done[kMaxDev][INIT_NKINDS];

template <typename F>
static int once_per_device(int kind, F &&setup) {
    int dev = 0;
    TB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDev) return TRIPLES_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_init_done[dev][kind]) return TRIPLES_OK;
    const int rc = setup();
    if (rc == TRIPLES_OK) g_init_done[dev][kind] = true;
    return rc;
}

// LNO chunk epilogue (FP64): energy of the projected amplitudes and, with
// want_grad, mat_bar, the D and V-term gradients and the FP64 Wbar staging
// that the adjoint contractions read next (four passes, see lno.cuh).
template <typename StageT>
static int lno_chunk(const Plan &P, const ChunkDesc &ch, cudaStream_t st, const TriplesIO &io, char *ws,
                     Ctrl *ctrl, const StageT *S, void *SW, const int *ijk, int split) {
    {
        const int rc = once_per_device(INIT_LNO, [&]() -> int {
            const int ts = (int)lno_tile_smem();
            TB_CUDA(cudaFuncSetAttribute(k_lno_tile_fwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, ts));
            TB_CUDA(cudaFuncSetAttribute(k_lno_tile_fwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, ts));
            TB_CUDA(cudaFuncSetAttribute(k_lno_tile_adj<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, ts));
            TB_CUDA(cudaFuncSetAttribute(k_lno_tile_adj<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ts));
            TB_CUDA(cudaFuncSetAttribute(k_lno_tile_adj<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ts));
            LnoTables tabs;
            lno_build_tables(tabs);
            TB_CUDA(cudaMemcpyToSymbol(c_lno_tab, &tabs, sizeof(tabs)));
            LnoPattern pats[16];
            lno_build_patterns(pats);
            TB_CUDA(cudaMemcpyToSymbol(c_lno_pat, pats, sizeof(pats)));
            const int ps = (int)lno_proj_smem(kLnoMaxO);
            TB_CUDA(cudaFuncSetAttribute(k_lno_proj, cudaFuncAttributeMaxDynamicSharedMemorySize, ps));
            return TRIPLES_OK;
        });
        if (rc != TRIPLES_OK) return rc;
    }
    const Dims &d = P.d;
    LnoArgs A;
    A.d = d;
    A.ch = ch;
    for (int k = 0; k < 27; k++) A.tau_of[k] = 0;
    for (int sx = 0; sx < 3; sx++)
        for (int sy = 0; sy < 3; sy++)
            for (int sz = 0; sz < 3; sz++)
                for (int t = 0; t < ch.nperm; t++)
                    if (ch.pb[t].bx == ch.blk[sx] && ch.pb[t].by == ch.blk[sy] && ch.pb[t].bz == ch.blk[sz])
                        A.tau_of[(sx * 3 + sy) * 3 + sz] = (signed char)t;
    // virtual sub-block triples, one per orbit of orderings
    A.nsub = 0;
    int nsb[3];
    for (int t = 0; t < 3; t++) nsb[t] = (ch.nabc[t] + kLnoSB - 1) / kLnoSB;
    for (int sa = 0; sa < nsb[0]; sa++)
        for (int sb = 0; sb < nsb[1]; sb++) {
            if (ch.blk[0] == ch.blk[1] && sb > sa) continue;
            for (int sc = 0; sc < nsb[2]; sc++) {
                if (ch.blk[1] == ch.blk[2] && sc > sb) continue;
                if (A.nsub >= kLnoMaxSub) return TRIPLES_ERR_UNSUPPORTED;
                LnoSub &u = A.sub[A.nsub++];
                const int si[3] = {sa, sb, sc};
                for (int t = 0; t < 3; t++) {
                    u.st[t] = ch.base[t] + si[t] * kLnoSB;
                    const int len = ch.nabc[t] - si[t] * kLnoSB;
                    u.len[t] = len < kLnoSB ? len : kLnoSB;
                }
            }
        }
    A.ijk = ijk;
    A.S = S;
    A.B0 = (double *)(ws + P.off_L[0]);
    A.B1 = (double *)(ws + P.off_L[1]);
    A.B2 = (double *)(ws + P.off_L[2]);
    A.B3 = (double *)(ws + P.off_L[3]);
    A.mat = io.mat; A.mo_e = io.mo_energy; A.t1 = io.t1; A.t2 = io.t2; A.ovov = io.ovov; A.fvo = io.fvo;
    A.SW = SW;
    A.wscale = &ctrl->wscale;
    A.mat_bar = io.mat_bar; A.mo_bar = io.mo_energy_bar; A.t1_bar = io.t1_bar; A.t2_bar = io.t2_bar;
    A.ovov_bar = io.ovov_bar; A.fvo_bar = io.fvo_bar;
    A.ybar = io.ybar;
    A.want_grad = P.want_grad;
    A.part = (double *)(ws + P.off_lpart);
    long long maxcols = 0, maxrows = 0;
    for (int t = 0; t < ch.nperm; t++) {
        const long long rows = (long long)d.o * d.o * ch.pb[t].Tx * ch.pb[t].Ty;
        if (rows * d.o * ch.pb[t].Tz > maxcols) maxcols = rows * d.o * ch.pb[t].Tz;
        if (rows > maxrows) maxrows = rows;
    }
    auto clampg = [](long long n) { return (unsigned)(n < kLnoGrid ? (n > 0 ? n : 1) : kLnoGrid); };
    A.n_ijk = P.n_ijk;
    const dim3 gtile((unsigned)A.nsub, (unsigned)((P.n_ijk + kLnoReps - 1) / kLnoReps));
    // streaming passes: a few full waves of two blocks per SM over the chunk's
    // orderings (their per-block reductions end in global atomics on a few
    // hundred entries, so the grid stays small)
    const long long wave = (long long)kLnoWaves * 2 * num_sms() / ch.nperm;
    auto clampw = [&](long long n) { return clampg(n < wave ? n : wave); };
    const dim3 gproj(clampw((maxcols / d.o + kLnoTile - 1) / kLnoTile), (unsigned)ch.nperm);
    TB_KLAUNCH(P_LNO, k_lno_tile_fwd<StageT><<<gtile, kLnoThreads, lno_tile_smem(), st>>>(A));
    TB_KLAUNCH(P_LNO_PROJ, k_lno_proj<<<gproj, kLnoThreads, lno_proj_smem(d.o), st>>>(A));
    TB_KLAUNCH(P_PREP, k_f2_energy_sum<<<1, 256, 0, st>>>(A.part, (int)(gproj.x * gproj.y), &ctrl->e_acc));
    if (!P.want_grad) return TRIPLES_OK;
    if (split != 0)   // fp16: power-of-two scale of the split Wbar; bf16: scale 1 (both read by the contractions)
        TB_KLAUNCH(P_PREP, k_chunk_scale<<<1, 32, 0, st>>>(ctrl, io.mo_energy, d.o, ch.base[0], ch.nabc[0], ch.base[1],
                                                           ch.nabc[1], ch.base[2], ch.nabc[2], io.ybar,
                                                           split == 1 ? 1 : 0, 1));
    if (split == 0)
        TB_KLAUNCH(P_LNO_ADJ, k_lno_tile_adj<0><<<gtile, kLnoThreads, lno_tile_smem(), st>>>(A));
    else if (split == 1)
        TB_KLAUNCH(P_LNO_ADJ, k_lno_tile_adj<1><<<gtile, kLnoThreads, lno_tile_smem(), st>>>(A));
    else
        TB_KLAUNCH(P_LNO_ADJ, k_lno_tile_adj<2><<<gtile, kLnoThreads, lno_tile_smem(), st>>>(A));
    const dim3 gv(clampw((maxrows + kLnoThreads / 32 - 1) / (kLnoThreads / 32)), (unsigned)ch.nperm);
    int maxTz = 0;
    for (int t = 0; t < ch.nperm; t++) maxTz = ch.pb[t].Tz > maxTz ? ch.pb[t].Tz : maxTz;
    const int per_lane = (d.o * maxTz + 31) / 32;
    if (per_lane <= 2)
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<2><<<gv, kLnoThreads, 0, st>>>(A));
    else if (per_lane <= 4)
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<4><<<gv, kLnoThreads, 0, st>>>(A));
    else if (per_lane <= 8)
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<8><<<gv, kLnoThreads, 0, st>>>(A));
    else if (per_lane <= 12)
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<12><<<gv, kLnoThreads, 0, st>>>(A));
    else if (per_lane <= 16)
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<16><<<gv, kLnoThreads, 0, st>>>(A));
    else
        TB_KLAUNCH(P_LNO_VG, k_lno_vgrad<32><<<gv, kLnoThreads, 0, st>>>(A));
    return TRIPLES_OK;
}

// ---------------------------------------------------------------------------
// one-time device set-up and the mixed-precision kernel parameters of a call
// and of one chunk, shared by the single-problem and the batched drivers
// ---------------------------------------------------------------------------
template <typename StageT>
static int setup_epilogue() {
    constexpr int kSB = sizeof(StageT) == 4 ? 8 : 4;
    // once per device and element type: shared-memory opt-in and the
    // constant tables of the epilogue's region patterns
    return once_per_device(sizeof(StageT) == 4 ? INIT_F2_F32 : INIT_F2_F64, [&]() -> int {
        TB_CUDA(cudaFuncSetAttribute(k_f2t<StageT, kSB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)f2_smem_bytes<StageT, kSB>()));
        TB_CUDA(cudaFuncSetAttribute(k_f2t<StageT, kSB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)f2_smem_bytes<StageT, kSB>()));
        if (sizeof(StageT) == 4) {
            TB_CUDA(cudaFuncSetAttribute(k_f2p<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
            TB_CUDA(cudaFuncSetAttribute(k_f2p<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
            TB_CUDA(cudaFuncSetAttribute(k_f2p<1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
            TB_CUDA(cudaFuncSetAttribute(k_f2p<2, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
            TB_CUDA(cudaFuncSetAttribute(k_f2p<1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
            TB_CUDA(cudaFuncSetAttribute(k_f2p<2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)F2pSmem::BYTES));
        }
        F2Pattern pats[kF2Patterns];
        f2_build_patterns(pats);
        TB_CUDA(cudaMemcpyToSymbol(c_f2pat, pats, sizeof(pats)));
        return TRIPLES_OK;
    });
}

static int setup_tensor_cores() {
    return once_per_device(INIT_TC, [&]() -> int {
        TB_CUDA(cudaFuncSetAttribute(k_f1_tc<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcCfg<256>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_f1_tc<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcCfg<128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_f1_tc<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcCfg<256>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_f1_tc<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcCfg<128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<false, 128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<false, 128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<false, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<false, 128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<true, 128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<true, 128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<true, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<true, 128>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<false, 64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<false, 64>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<false, 64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<false, 64>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<true, 64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<true, 64>::SMEM));
        TB_CUDA(cudaFuncSetAttribute(k_b1_tc<true, 64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TcB1Cfg<true, 64>::SMEM));
        return TRIPLES_OK;
    });
}

// Tensor maps over one call's 16-bit operands (built on the host).
struct OperandMaps {
    CUtensorMap tmA1, tmB1, tmA2, tmB2;             // W contraction, K-major boxes
    CUtensorMap tmA1m, tmA2m, tmB1z[5], tmB2z[5];   // adjoint contractions, MN-major boxes
};

// The W contraction's N tile is BN = 16 * RT columns (RT occupied r values x
// 16 z), P.f1_bn.
static int build_operand_maps(const Plan &P, char *ws, OperandMaps &M) {
    const uint64_t o = P.d.o, v = P.d.v;
    const bool bf16 = P.prec == TRIPLES_PRECISION_MIXED_BF16;
    const uint64_t dA1[5] = {(uint64_t)P.Kp8, v, o, v, 2};
    const uint32_t bA[5] = {64, 16, 8, 1, 1};
    const uint64_t dB1[5] = {(uint64_t)P.Kp8, v, o, o, 2};
    const uint32_t bB[5] = {64, 16, (uint32_t)(P.f1_bn / 16), 1, 1};
    const uint64_t dA2[5] = {(uint64_t)P.Op8, v, o, o, 2};
    const uint64_t dB2[5] = {(uint64_t)P.Op8, v, o, v, 2};
    int rc;
    if ((rc = make_tmap5(&M.tmA1, ws + P.off_A1h, bf16, dA1, bA)) != TRIPLES_OK) return rc;
    if ((rc = make_tmap5(&M.tmB1, ws + P.off_B1h, bf16, dB1, bB)) != TRIPLES_OK) return rc;
    if ((rc = make_tmap5(&M.tmA2, ws + P.off_A2h, bf16, dA2, bA)) != TRIPLES_OK) return rc;
    if ((rc = make_tmap5(&M.tmB2, ws + P.off_B2h, bf16, dB2, bB)) != TRIPLES_OK) return rc;
    if (P.want_grad) {
        const uint64_t dA1mn[5] = {(uint64_t)P.Kp8, v, o, v, 2};
        const uint64_t dA2mn[5] = {(uint64_t)P.Op8, v, o, o, 2};
        const uint64_t dB1mn[5] = {(uint64_t)P.Kp8, v, o, o, 2};
        const uint64_t dB2mn[5] = {(uint64_t)P.Op8, v, o, v, 2};
        const uint32_t bX[5] = {64, 16, 4, 1, 1};
        if ((rc = make_tmap5(&M.tmA1m, ws + P.off_A1h, bf16, dA1mn, bX)) != TRIPLES_OK) return rc;
        if ((rc = make_tmap5(&M.tmA2m, ws + P.off_A2h, bf16, dA2mn, bX)) != TRIPLES_OK) return rc;
        for (int lt = 0; lt < 5; lt++) {
            const uint32_t tz = 1u << lt;
            const uint32_t bZ[5] = {64, tz, 64 / tz, 1, 1};
            if ((rc = make_tmap5(&M.tmB1z[lt], ws + P.off_B1h, bf16, dB1mn, bZ)) != TRIPLES_OK) return rc;
            if ((rc = make_tmap5(&M.tmB2z[lt], ws + P.off_B2h, bf16, dB2mn, bZ)) != TRIPLES_OK) return rc;
        }
    }
    return TRIPLES_OK;
}

// W-contraction parameters of one chunk (tiles ordering by ordering).
static int f1_params(const Plan &P, const ChunkDesc &ch, char *ws, TcF1Params &T) {
    const Dims &d = P.d;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    float *S = (float *)(ws + P.off_S);
    T.d = d;
    T.ch = ch;
    T.mt_count = (d.o + 7) / 8;
    const int rt = P.f1_bn / 16;
    T.nt_count = (d.o + rt - 1) / rt;
    T.cum[0] = 0;
    for (int t = 0; t < ch.nperm; t++) T.cum[t + 1] = T.cum[t] + ch.pb[t].Ty * d.o * T.mt_count * T.nt_count;
    T.nkb1 = (P.Kp8 + kTcBK - 1) / kTcBK;
    T.nkb2 = (P.Op8 + kTcBK - 1) / kTcBK;
    T.S = S;
    T.out_scale = &ctrl->out_scale;
    T.wmax_bits = &ctrl->wmax_bits;
    T.err = &ctrl->err;
    T.bf16 = P.prec == TRIPLES_PRECISION_MIXED_BF16 ? 1 : 0;
    T.kseg = P.kseg;
    for (int t = 0; t < 6; t++) T.tmS_ok[t] = 0;
    for (int t = 0; t < ch.nperm; t++) {
        const PermBlock &pb = ch.pb[t];
        if (pb.Tx == 16 && pb.Tz == 16 && d.o >= 2) {
            const int trc = make_tmap_stage(&T.tmS[t], S + pb.soff, d.o, pb.Tx, pb.Ty);
            if (trc != TRIPLES_OK) return trc;
            T.tmS_ok[t] = 1;
        }
    }
    return TRIPLES_OK;
}

// Epilogue parameters of one chunk: every sub-range triple, those of three
// distinct full 8-wide sub-ranges first (mixed precision; the persistent
// kernel k_f2p takes them with every occupied representative but i == j == k).
// Returns the number of those leading sub-range triples.
template <typename StageT>
static int f2_params(const Plan &P, const ChunkDesc &ch, char *ws, const TriplesIO &io, F2P<StageT> &F) {
    constexpr int kSB = sizeof(StageT) == 4 ? 8 : 4;
    const bool mixed = P.prec != TRIPLES_PRECISION_FP64;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    F.d = P.d;
    F.ch = ch;
    F.nsub = 0;
    int nsb[3];
    for (int t = 0; t < 3; t++) nsb[t] = (ch.nabc[t] + kSB - 1) / kSB;
    F2Sub rest[kMaxSub];
    int nrest = 0;
    for (int sa = 0; sa < nsb[0]; sa++)
        for (int sb = 0; sb < nsb[1]; sb++) {
            if (ch.blk[0] == ch.blk[1] && sb > sa) continue;
            for (int sc = 0; sc < nsb[2]; sc++) {
                if (ch.blk[1] == ch.blk[2] && sc > sb) continue;
                F2Sub u;
                const int si[3] = {sa, sb, sc};
                for (int t = 0; t < 3; t++) {
                    u.st[t] = ch.base[t] + si[t] * kSB;
                    int len = ch.nabc[t] - si[t] * kSB;
                    u.len[t] = len < kSB ? len : kSB;
                }
                const bool simple = mixed && u.len[0] == 8 && u.len[1] == 8 && u.len[2] == 8 &&
                                    u.st[0] != u.st[1] && u.st[1] != u.st[2] && u.st[0] != u.st[2];
                if (simple) F.sub[F.nsub++] = u;
                else rest[nrest++] = u;
            }
        }
    const int n_simple_sub = F.nsub;
    for (int t = 0; t < nrest; t++) F.sub[F.nsub++] = rest[t];
    F.ijk = (int *)(ws + P.off_ijk);
    F.mo_e = io.mo_energy; F.t1 = io.t1; F.t2 = io.t2; F.ovov = io.ovov; F.fvo = io.fvo;
    F.S = (StageT *)(ws + P.off_S);
    F.SW = P.want_grad ? (void *)(ws + P.off_SW) : nullptr;
    F.split = mixed ? (P.prec == TRIPLES_PRECISION_MIXED_BF16 ? 2 : 1) : 0;
    F.wscale = &ctrl->wscale;
    F.ybar = io.ybar;
    F.want_grad = P.want_grad;
    F.e_part = (double *)(ws + P.off_epart);
    F.n_ijk = P.n_ijk;
    F.mo_bar = io.mo_energy_bar;
    F.t1_bar = io.t1_bar; F.fvo_bar = io.fvo_bar; F.ovov_bar = io.ovov_bar; F.t2_bar = io.t2_bar;
    F.rep0 = 0;
    F.sub0 = 0;
    F.nsub_l = F.nsub;
    return n_simple_sub;
}

// Adjoint-contraction parameters of one chunk and kind (0: ovvv_bar, 1: t2_bar
// ovvv term, 2: ovoo_bar, 3: t2_bar ooov term), tiles ordering by ordering.
static int b1_params(const Plan &P, const ChunkDesc &ch, char *ws, const OperandMaps &M, int kind, TcB1Params &B) {
    const Dims &d = P.d;
    const uint64_t o = d.o;
    const bool bf16 = P.prec == TRIPLES_PRECISION_MIXED_BF16;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    char *SW = ws + P.off_SW;
    const uint32_t bK[5] = {64, 1, 16, 8, 1};   // Wbar K-major (kinds 0, 2)
    const uint32_t bM[5] = {64, 1, 16, 4, 1};   // Wbar MN-major (kinds 1, 3)
    B.d = d;
    B.nperm = ch.nperm;
    for (int t = 0; t < ch.nperm; t++) B.pb[t] = ch.pb[t];
    B.wscale = &ctrl->wscale;
    B.err = &ctrl->err;
    B.bf16 = bf16 ? 1 : 0;
    B.kseg = P.kseg;
    B.kind = kind;
    B.ntile_n = kind <= 1 ? (d.v + 127) / 128 : (d.o + 63) / 64;
    B.G = (double *)(ws + (kind == 0 ? P.off_GA1 : kind == 1 ? P.off_GB1 : kind == 2 ? P.off_GA2 : P.off_GB2));
    B.oscale = &ctrl->scale[(kind == 0 || kind == 2) ? 1 : 0];
    B.sign = kind == 2 ? -1.0 : 1.0;
    for (int t = 0; t < ch.nperm; t++) {
        const PermBlock &pb = ch.pb[t];
        const uint64_t dW[5] = {(uint64_t)pb.rzp, o, (uint64_t)pb.Tx, o, (uint64_t)(2 * pb.Ty)};
        const int rc = make_tmap5(&B.tmA[t], SW + 2 * pb.swoff * 2, bf16, dW, (kind == 0 || kind == 2) ? bK : bM);
        if (rc != TRIPLES_OK) return rc;
        int lz = 0;
        while ((1 << lz) < pb.Tz) lz++;
        switch (kind) {
        case 0:
            B.tmB[t] = M.tmB1z[lz];
            B.nbatch[t] = pb.Ty; B.ntile_m[t] = (d.o + 7) / 8;
            B.nk_outer[t] = d.o; B.nk_inner[t] = (d.o * pb.Tz + 63) / 64;
            break;
        case 1:
            B.tmB[t] = M.tmA1m;
            B.nbatch[t] = d.o; B.ntile_m[t] = (d.o * pb.Tz + 127) / 128;
            B.nk_outer[t] = pb.Ty; B.nk_inner[t] = (d.o + 3) / 4;
            break;
        case 2:
            B.tmB[t] = M.tmB2z[lz];
            B.nbatch[t] = d.o; B.ntile_m[t] = (d.o + 7) / 8;
            B.nk_outer[t] = pb.Ty; B.nk_inner[t] = (d.o * pb.Tz + 63) / 64;
            break;
        default:
            B.tmB[t] = M.tmA2m;
            B.nbatch[t] = pb.Ty; B.ntile_m[t] = (d.o * pb.Tz + 127) / 128;
            B.nk_outer[t] = d.o; B.nk_inner[t] = (d.o + 3) / 4;
            break;
        }
    }
    B.cum[0] = 0;
    for (int t = 0; t < ch.nperm; t++) B.cum[t + 1] = B.cum[t] + B.nbatch[t] * B.ntile_m[t] * B.ntile_n;
    return TRIPLES_OK;
}

// Per-call preparation: control block, occupied table, zeroed gradients, and
// the operand layouts (FP64 copies, or 16-bit splits with their scales).
template <typename StageT>
static int prep_launches(const Plan &P, cudaStream_t st, const TriplesIO &io) {
    const Dims d = P.d;
    const bool mixed = P.prec != TRIPLES_PRECISION_FP64;
    const bool bf16 = P.prec == TRIPLES_PRECISION_MIXED_BF16;
    char *ws = (char *)io.workspace;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    double *A1 = (double *)(ws + P.off_A1);
    double *B1 = (double *)(ws + P.off_B1);
    double *A2 = (double *)(ws + P.off_A2);
    double *B2 = (double *)(ws + P.off_B2);
    void *SW = P.want_grad ? (void *)(ws + P.off_SW) : nullptr;
    double *GA1 = P.want_grad ? (double *)(ws + P.off_GA1) : nullptr;
    double *GB1 = P.want_grad ? (double *)(ws + P.off_GB1) : nullptr;
    double *GA2 = P.want_grad ? (double *)(ws + P.off_GA2) : nullptr;
    double *GB2 = P.want_grad ? (double *)(ws + P.off_GB2) : nullptr;
    int *ijk = (int *)(ws + P.off_ijk);
    const size_t o = d.o, v = d.v, n = d.n;

    TB_CUDA(cudaMemsetAsync(ctrl, 0, kCtrlBytes, st));
    TB_KLAUNCH(P_PREP, k_ijk_table<<<grid1d(P.n_ijk, 128), 128, 0, st>>>(d.o, ijk));
    if (P.want_grad) {
        TB_CUDA(cudaMemsetAsync(GA1, 0, v * o * v * d.Kp * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(GB1, 0, o * o * v * d.Kp * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(GA2, 0, o * o * v * o * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(GB2, 0, v * o * v * o * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(io.mo_energy_bar, 0, n * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(io.t1_bar, 0, o * v * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(io.t2_bar, 0, o * o * v * v * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(io.ovov_bar, 0, o * v * o * v * sizeof(double), st));
        TB_CUDA(cudaMemsetAsync(io.fvo_bar, 0, v * o * sizeof(double), st));
        if (P.lno) {
            TB_CUDA(cudaMemsetAsync(io.mat_bar, 0, o * o * sizeof(double), st));
            if (mixed) TB_KLAUNCH(P_PREP, k_lno_mat_norms<<<1, 64, 0, st>>>(io.mat, d.o, ctrl));
        }
    }

    // FP64 operand layouts (used by the FP64 contractions only)
    if (!mixed) {
        TB_KLAUNCH(P_PREP, k_prep_A1<<<dim3((d.Kp + 31) / 32, (d.v + 31) / 32, (unsigned)(o * v)), dim3(32, 8), 0, st>>>(
            io.ovvv, P.packed, d, A1));
        TB_KLAUNCH(P_PREP, k_prep_B1<<<(unsigned)(o * o * v), 128, 0, st>>>(io.t2, d, B1));
        TB_KLAUNCH(P_PREP, k_prep_A2<<<grid1d((long long)o * o * v * o, 256), 256, 0, st>>>(io.ovoo, d, A2));
        TB_KLAUNCH(P_PREP, k_prep_B2<<<grid1d((long long)v * o * v * o, 256), 256, 0, st>>>(io.t2, d, B2));
    }

    // 16-bit split operands (tensor-core path)
    if (mixed) {
        const long long npair = (long long)v * (v + 1) / 2;
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * v * (P.packed ? npair : (long long)v * v), 256), 256, 0, st>>>(
            io.ovvv, (long long)o * v * (P.packed ? npair : (long long)v * v), &ctrl->absmax[0]));
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * v * o * o, 256), 256, 0, st>>>(io.ovoo, (long long)o * v * o * o,
                                                                         &ctrl->absmax[1]));
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * o * v * v, 256), 256, 0, st>>>(io.t2, (long long)o * o * v * v,
                                                                         &ctrl->absmax[2]));
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * v * o * v, 256), 256, 0, st>>>(io.ovov, (long long)o * v * o * v, &ctrl->absmax[3]));
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * v, 256), 256, 0, st>>>(io.t1, (long long)o * v, &ctrl->absmax[4]));
        TB_KLAUNCH(P_PREP, k_absmax<<<grid1d((long long)o * v, 256), 256, 0, st>>>(io.fvo, (long long)o * v, &ctrl->absmax[5]));
        TB_KLAUNCH(P_PREP, k_make_scales<<<1, 1, 0, st>>>(ctrl, bf16 ? 0 : 1));
        if (bf16) {
            TB_KLAUNCH(P_PREP, k_prep_A1h<__nv_bfloat16><<<dim3((P.Kp8 + 31) / 32, (d.v + 31) / 32, (unsigned)(o * v)), dim3(32, 8), 0, st>>>(
                io.ovvv, P.packed, d, P.Kp8, ctrl, (__nv_bfloat16 *)(ws + P.off_A1h)));
            TB_KLAUNCH(P_PREP, k_prep_B1h<__nv_bfloat16><<<(unsigned)(o * o * v), 128, 0, st>>>(io.t2, d, P.Kp8, ctrl,
                                                                            (__nv_bfloat16 *)(ws + P.off_B1h)));
            TB_KLAUNCH(P_PREP, k_prep_A2h<__nv_bfloat16><<<grid1d((long long)o * o * v * P.Op8, 256), 256, 0, st>>>(
                io.ovoo, d, P.Op8, ctrl, (__nv_bfloat16 *)(ws + P.off_A2h)));
            TB_KLAUNCH(P_PREP, k_prep_B2h<__nv_bfloat16><<<grid1d((long long)v * o * v * P.Op8, 256), 256, 0, st>>>(
                io.t2, d, P.Op8, ctrl, (__nv_bfloat16 *)(ws + P.off_B2h)));
        } else {
            TB_KLAUNCH(P_PREP, k_prep_A1h<__half><<<dim3((P.Kp8 + 31) / 32, (d.v + 31) / 32, (unsigned)(o * v)), dim3(32, 8), 0, st>>>(
                io.ovvv, P.packed, d, P.Kp8, ctrl, (__half *)(ws + P.off_A1h)));
            TB_KLAUNCH(P_PREP, k_prep_B1h<__half><<<(unsigned)(o * o * v), 128, 0, st>>>(io.t2, d, P.Kp8, ctrl,
                                                                     (__half *)(ws + P.off_B1h)));
            TB_KLAUNCH(P_PREP, k_prep_A2h<__half><<<grid1d((long long)o * o * v * P.Op8, 256), 256, 0, st>>>(
                io.ovoo, d, P.Op8, ctrl, (__half *)(ws + P.off_A2h)));
            TB_KLAUNCH(P_PREP, k_prep_B2h<__half><<<grid1d((long long)v * o * v * P.Op8, 256), 256, 0, st>>>(
                io.t2, d, P.Op8, ctrl, (__half *)(ws + P.off_B2h)));
        }
        TB_LAUNCH_CHECK();
        if (P.want_grad) TB_CUDA(cudaMemsetAsync(SW, 0, P.wbar_elems * 4, st));
    }
    return TRIPLES_OK;

}

// Gradients back to the reference layouts, and the energy out.
static int fold_launches(const Plan &P, cudaStream_t st, const TriplesIO &io) {
    const Dims d = P.d;
    char *ws = (char *)io.workspace;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    const double *GA1 = (const double *)(ws + P.off_GA1), *GB1 = (const double *)(ws + P.off_GB1);
    const double *GA2 = (const double *)(ws + P.off_GA2), *GB2 = (const double *)(ws + P.off_GB2);
    const size_t o = d.o, v = d.v;
    if (P.want_grad) {
        if (P.packed) {
            TB_KLAUNCH(P_FOLD, k_fold_ovvv_packed<<<grid1d((long long)o * v * (v * (v + 1) / 2), 256), 256, 0, st>>>(
                GA1, d, io.ovvv_bar));
        } else {
            TB_KLAUNCH(P_FOLD, k_fold_ovvv_full<<<dim3((d.v + 31) / 32, (d.v + 31) / 32, (unsigned)(o * v)), dim3(32, 8), 0, st>>>(
                GA1, d, io.ovvv_bar));
        }
        TB_LAUNCH_CHECK();
        TB_KLAUNCH(P_FOLD, k_fold_t2<<<grid1d((long long)o * o * v * v, 256), 256, 0, st>>>(GB1, GB2, d, io.t2_bar));
        TB_KLAUNCH(P_FOLD, k_fold_ovoo<<<grid1d((long long)o * v * o * o, 256), 256, 0, st>>>(GA2, d, io.ovoo_bar));
    }
    TB_KLAUNCH(P_FOLD, k_copy_scalar<<<1, 1, 0, st>>>(&ctrl->e_acc, io.e_out));
    return TRIPLES_OK;
}

template <typename StageT>
static int run_impl(const Plan &P, cudaStream_t st, const TriplesIO &io) {
    constexpr int kSB = sizeof(StageT) == 4 ? 8 : 4;   // epilogue sub-block edge
    {
        const int rc = setup_epilogue<StageT>();
        if (rc != TRIPLES_OK) return rc;
    }
    int prc = prep_launches<StageT>(P, st, io);
    if (prc != TRIPLES_OK) return prc;
    const Dims d = P.d;
    const bool mixed = P.prec != TRIPLES_PRECISION_FP64;
    const bool bf16 = P.prec == TRIPLES_PRECISION_MIXED_BF16;
    char *ws = (char *)io.workspace;
    Ctrl *ctrl = (Ctrl *)(ws + P.off_ctrl);
    double *A1 = (double *)(ws + P.off_A1);
    double *B1 = (double *)(ws + P.off_B1);
    double *A2 = (double *)(ws + P.off_A2);
    double *B2 = (double *)(ws + P.off_B2);
    StageT *S = (StageT *)(ws + P.off_S);
    void *SW = P.want_grad ? (void *)(ws + P.off_SW) : nullptr;
    double *GA1 = P.want_grad ? (double *)(ws + P.off_GA1) : nullptr;
    double *GB1 = P.want_grad ? (double *)(ws + P.off_GB1) : nullptr;
    double *GA2 = P.want_grad ? (double *)(ws + P.off_GA2) : nullptr;
    double *GB2 = P.want_grad ? (double *)(ws + P.off_GB2) : nullptr;
    int *ijk = (int *)(ws + P.off_ijk);
    double *e_part = (double *)(ws + P.off_epart);
    const int f1_bn = P.f1_bn;
    OperandMaps M;
    if (mixed) {
        if ((prc = build_operand_maps(P, ws, M)) != TRIPLES_OK) return prc;
        if ((prc = setup_tensor_cores()) != TRIPLES_OK) return prc;
    }

    for (int A = 0; A < P.nb; A++) {
        if (A < P.a0 || (P.a1 > 0 && A >= P.a1)) continue;
        for (int B = 0; B <= A; B++)
            for (int C = 0; C <= B; C++) {
                ChunkDesc ch;
                make_chunk(d, A, B, C, ch);
                int maxTx = 0, maxTz = 0;
                for (int t = 0; t < ch.nperm; t++) {
                    if (ch.pb[t].Tx > maxTx) maxTx = ch.pb[t].Tx;
                    if (ch.pb[t].Tz > maxTz) maxTz = ch.pb[t].Tz;
                }
                // F1: raw amplitudes
                if (mixed) {
                    TcF1Params T;
                    const int frc = f1_params(P, ch, ws, T);
                    if (frc != TRIPLES_OK) return frc;
                    const int tiles = T.cum[ch.nperm];
                    const int grid = tiles < num_sms() ? tiles : num_sms();
                    const F1Maps Mf1{M.tmA1, M.tmB1, M.tmA2, M.tmB2};
                    if (f1_bn == 128)
                        TB_KLAUNCH(P_F1, (k_f1_tc<128, false><<<grid, kF1Threads, TcCfg<128>::SMEM, st>>>(
                                             Mf1, T, nullptr, nullptr, 0)));
                    else
                        TB_KLAUNCH(P_F1, (k_f1_tc<256, false><<<grid, kF1Threads, TcCfg<256>::SMEM, st>>>(
                                             Mf1, T, nullptr, nullptr, 0)));
                } else {
                    GemmLaunch<double> L;
                    L.d = d;
                    L.ch = ch;
                    L.A1 = A1; L.B1 = B1; L.A2 = A2; L.B2 = B2;
                    L.S = (double *)S;
                    L.G = nullptr;
                    L.cum[0] = 0;
                    for (int t = 0; t < ch.nperm; t++) L.cum[t + 1] = L.cum[t] + ch.pb[t].Ty * d.o;
                    TB_KLAUNCH(P_F1, k_f1_fp64<<<dim3((d.o * maxTx + kGBM - 1) / kGBM, (d.o * maxTz + kGBN - 1) / kGBN,
                                     L.cum[ch.nperm]),
                                256, 0, st>>>(L));
                }
                if (P.lno) {
                    // projected energy: whole-chunk epilogue instead of the orbit tiles
                    const int rc = lno_chunk<StageT>(P, ch, st, io, ws, ctrl, S, SW, ijk, mixed ? (bf16 ? 2 : 1) : 0);
                    if (rc != TRIPLES_OK) return rc;
                } else {
                    // F2: energy (+ adjoint of the raw amplitudes).  Sub-range
                    // triples of three distinct full 8-wide sub-ranges come first;
                    // in the mixed modes they go to the persistent kernel k_f2p with
                    // the all-distinct occupied representatives (the first
                    // n_distinct_ijk of the table) and, in a second launch, with the
                    // representatives i = j > k and i > j = k that follow them; every
                    // other item (i = j = k, the remaining sub-range triples) to k_f2t.
                    F2P<StageT> F;
                    const int n_simple_sub = f2_params<StageT>(P, ch, ws, io, F);
                    if (mixed && P.want_grad)
                        TB_KLAUNCH(P_PREP, k_chunk_scale<<<1, 32, 0, st>>>(ctrl, io.mo_energy, d.o, ch.base[0], ch.nabc[0],
                                                                           ch.base[1], ch.nabc[1], ch.base[2], ch.nabc[2],
                                                                           io.ybar, bf16 ? 0 : 1, 0));
                    const int nd = mixed ? n_distinct_ijk(d.o) : 0;
                    const int np = mixed ? d.o * (d.o - 1) / 2 : 0;   // i = j > k, then as many i > j = k
                    auto f2t = [&](int rep0, int nrep, int sub0, int nsub_l) -> int {
                        if (nrep <= 0 || nsub_l <= 0) return TRIPLES_OK;
                        F.rep0 = rep0;
                        F.sub0 = sub0;
                        F.nsub_l = nsub_l;
                        TB_KLAUNCH(P_F2, (k_f2t<StageT, kSB, false><<<(unsigned)(nrep * nsub_l), F2Smem<kSB>::NT,
                                                                      f2_smem_bytes<StageT, kSB>(), st>>>(
                                             F, nullptr, nullptr, 0)));
                        return TRIPLES_OK;
                    };
                    // k_f2p over the representatives [rep0, rep0 + nrep) and the
                    // leading n_simple_sub sub-range triples
                    auto f2p = [&](int rep0, int nrep, int deg) -> int {
                        if (nrep <= 0 || n_simple_sub <= 0) return TRIPLES_OK;
                        F.rep0 = rep0;
                        F.sub0 = 0;
                        F.nsub_l = n_simple_sub;
                        F2P<float> Ff;
                        std::memcpy(&Ff, &F, sizeof(F));   // StageT = float in the mixed modes
                        const int nitems = nrep * n_simple_sub;
                        const unsigned nb = (unsigned)(nitems < num_sms() ? nitems : num_sms());
#define TB_F2P(HV, DV) TB_KLAUNCH(P_F2, (k_f2p<HV, DV><<<nb, F2pSmem::NT, F2pSmem::BYTES, st>>>(Ff, nitems)))
                        if (deg == 1) {
                            if (bf16) TB_F2P(2, 1);
                            else TB_F2P(1, 1);
                        } else if (deg == 2) {
                            if (bf16) TB_F2P(2, 2);
                            else TB_F2P(1, 2);
                        } else {
                            if (bf16) TB_F2P(2, 0);
                            else TB_F2P(1, 0);
                        }
#undef TB_F2P
                        return TRIPLES_OK;
                    };
                    int frc;
                    if ((frc = f2p(0, nd, 0)) != TRIPLES_OK) return frc;
                    if ((frc = f2p(nd, np, 1)) != TRIPLES_OK) return frc;
                    if ((frc = f2p(nd + np, np, 2)) != TRIPLES_OK) return frc;
                    if ((frc = f2t(0, nd + 2 * np, n_simple_sub, F.nsub - n_simple_sub)) != TRIPLES_OK) return frc;
                    if ((frc = f2t(nd + 2 * np, P.n_ijk - nd - 2 * np, 0, F.nsub)) != TRIPLES_OK) return frc;
                    TB_KLAUNCH(P_F2, k_f2_energy_sum<<<1, 256, 0, st>>>(e_part, P.n_ijk * F.nsub, &ctrl->e_acc));
                }
                if (!P.want_grad) continue;
                // W-term gradients
                if (mixed) {
                    // one launch per kind over all orderings of the chunk
                    TcB1Params B;
                    auto launch_b1 = [&](int kind) -> int {
                        const int brc = b1_params(P, ch, ws, M, kind, B);
                        if (brc != TRIPLES_OK) return brc;
                        const int tiles = B.cum[ch.nperm];
                        const int grid = tiles < num_sms() ? tiles : num_sms();
                        switch (kind) {
                        case 0:
                            TB_KLAUNCH(P_B1A, (k_b1_tc<false, 128, false><<<grid, kB1Threads, TcB1Cfg<false, 128>::SMEM, st>>>(
                                                  B, nullptr, nullptr, 0)));
                            break;
                        case 1:
                            TB_KLAUNCH(P_B1B, (k_b1_tc<true, 128, false><<<grid, kB1Threads, TcB1Cfg<true, 128>::SMEM, st>>>(
                                                  B, nullptr, nullptr, 0)));
                            break;
                        case 2:
                            TB_KLAUNCH(P_B1C, (k_b1_tc<false, 64, false><<<grid, kB1Threads, TcB1Cfg<false, 64>::SMEM, st>>>(
                                                  B, nullptr, nullptr, 0)));
                            break;
                        default:
                            TB_KLAUNCH(P_B1D, (k_b1_tc<true, 64, false><<<grid, kB1Threads, TcB1Cfg<true, 64>::SMEM, st>>>(
                                                  B, nullptr, nullptr, 0)));
                            break;
                        }
                        return TRIPLES_OK;
                    };
                    for (int kind = 0; kind < 4; kind++) {
                        const int brc = launch_b1(kind);
                        if (brc != TRIPLES_OK) return brc;
                    }
                } else {
                GemmLaunch<StageT> L;
                L.d = d;
                L.ch = ch;
                L.A1 = A1; L.B1 = B1; L.A2 = A2; L.B2 = B2;
                L.S = reinterpret_cast<StageT *>(SW);
                L.cum[0] = 0;
                for (int t = 0; t < ch.nperm; t++) L.cum[t + 1] = L.cum[t] + ch.pb[t].Ty;
                L.G = GA1;
                TB_KLAUNCH(P_B1A, k_b1a_fp64<StageT><<<dim3((d.o * maxTx + kGBM - 1) / kGBM, (d.v + kGBN - 1) / kGBN, L.cum[ch.nperm]),
                                     256, 0, st>>>(L));
                L.G = GB2;
                TB_KLAUNCH(P_B1D, k_b1d_fp64<StageT><<<dim3((d.o * maxTz + kGBM - 1) / kGBM, (d.o + kGBN - 1) / kGBN, L.cum[ch.nperm]),
                                     256, 0, st>>>(L));
                L.G = GB1;
                TB_KLAUNCH(P_B1B, k_b1b_fp64<StageT><<<dim3((d.o * maxTz + kGBM - 1) / kGBM, (d.v + kGBN - 1) / kGBN,
                                                             (unsigned)(d.o * ch.nperm)),
                                     256, 0, st>>>(L));
                L.G = GA2;
                TB_KLAUNCH(P_B1C, k_b1c_fp64<StageT><<<dim3((d.o * maxTx + kGBM - 1) / kGBM, (d.o + kGBN - 1) / kGBN,
                                                             (unsigned)(d.o * ch.nperm)),
                                     256, 0, st>>>(L));
                }
            }
    }

    return fold_launches(P, st, io);
}

int run_triples(const Plan &P, cudaStream_t st, const TriplesIO &io) {
    if (P.prec == TRIPLES_PRECISION_FP64) return run_impl<double>(P, st, io);
    return run_impl<float>(P, st, io);
}

// ---------------------------------------------------------------------------
// batched calls: many problems of uneven size.  Every problem keeps its own
// workspace (operands, one chunk's staging, gradient accumulators); chunk
// step c launches each kernel kind ONCE over the c-th chunk of every problem
// that has one (tiles / CTAs numbered problem after problem, parameters in
// job tables built on the host when the batch is created and stored after
// the problems' workspaces).  Mixed precision only; an FP64 batch runs the
// problems one after another.
// ---------------------------------------------------------------------------
struct BatchStep {
    size_t f1_jobs[2], f1_start[2];   // [0]: W-contraction N tile 256, [1]: 128
    int f1_n[2], f1_tiles[2];
    size_t aux;                       // ChunkAux per problem of the step
    int naux;
    size_t f2_jobs, f2_start;
    int f2_ctas;
    size_t b1_jobs[4], b1_start[4];   // per adjoint kind
    int b1_tiles[4];
};

struct Batch {
    int prec = 0, nprob = 0;
    char *ws = nullptr;
    std::vector<Plan> plans;
    std::vector<TriplesIO> ios;
    std::vector<size_t> ws_off;
    std::vector<BatchStep> steps;
    size_t tables_off = 0, total = 0;
};

static void batch_chunks(const Plan &P, std::vector<ChunkDesc> &out) {
    out.clear();
    for (int A = 0; A < P.nb; A++)
        for (int B = 0; B <= A; B++)
            for (int C = 0; C <= B; C++) {
                ChunkDesc ch;
                make_chunk(P.d, A, B, C, ch);
                out.push_back(ch);
            }
}

// Plans, workspace offsets and (with image != nullptr) the job tables of a
// batch; B.ws must then be the device workspace the tables point into.
static int batch_build(Batch &B, int prec, int nprob, const triples_problem *probs, double ybar,
                       std::vector<char> *image) {
    if (nprob < 1 || !probs) return TRIPLES_ERR_INVALID_ARGUMENT;
    B.prec = prec;
    B.nprob = nprob;
    B.plans.assign(nprob, Plan{});
    B.ios.assign(nprob, TriplesIO{});
    B.ws_off.assign(nprob, 0);
    size_t off = 0;
    for (int p = 0; p < nprob; p++) {
        const triples_problem &q = probs[p];
        triples_options opt{};
        opt.block_size = q.block_size;
        opt.tile_n = q.tile_n;
        const int rc = make_plan(prec, q.nocc, q.nvir, q.ovvv_packed, 1, B.plans[p], 0, &opt);
        if (rc != TRIPLES_OK) return rc;
        B.ws_off[p] = off;
        off = align256(off + B.plans[p].total);
        TriplesIO &io = B.ios[p];
        io.mo_energy = q.mo_energy; io.t1 = q.t1; io.t2 = q.t2; io.ovoo = q.ovoo; io.ovov = q.ovov;
        io.ovvv = q.ovvv; io.fvo = q.fvo; io.ybar = ybar; io.e_out = q.e_out;
        io.mo_energy_bar = q.mo_energy_bar; io.t1_bar = q.t1_bar; io.t2_bar = q.t2_bar; io.ovoo_bar = q.ovoo_bar;
        io.ovov_bar = q.ovov_bar; io.ovvv_bar = q.ovvv_bar; io.fvo_bar = q.fvo_bar;
        io.workspace = B.ws ? B.ws + B.ws_off[p] : nullptr;
        if (image && (!io.mo_energy || !io.t1 || !io.t2 || !io.ovoo || !io.ovov || !io.ovvv || !io.fvo || !io.e_out ||
                      !io.mo_energy_bar || !io.t1_bar || !io.t2_bar || !io.ovoo_bar || !io.ovov_bar ||
                      !io.ovvv_bar || !io.fvo_bar))
            return TRIPLES_ERR_INVALID_ARGUMENT;
    }
    B.tables_off = off;
    B.steps.clear();
    if (prec == TRIPLES_PRECISION_FP64) {
        B.total = off;
        return TRIPLES_OK;
    }
    std::vector<std::vector<ChunkDesc>> chunks(nprob);
    std::vector<OperandMaps> maps(image ? nprob : 0);
    size_t nsteps = 0;
    for (int p = 0; p < nprob; p++) {
        batch_chunks(B.plans[p], chunks[p]);
        if (chunks[p].size() > nsteps) nsteps = chunks[p].size();
        if (image) {
            const int rc = build_operand_maps(B.plans[p], B.ws + B.ws_off[p], maps[p]);
            if (rc != TRIPLES_OK) return rc;
        }
    }
    // table layout: per step, 256-byte aligned arrays
    size_t t = 0;
    auto take = [&](size_t bytes) {
        const size_t at = t;
        t = align256(t + bytes);
        return at;
    };
    B.steps.resize(nsteps);
    for (size_t c = 0; c < nsteps; c++) {
        BatchStep &S = B.steps[c];
        std::vector<int> who, who_bn[2];
        for (int p = 0; p < nprob; p++)
            if (c < chunks[p].size()) {
                who.push_back(p);
                who_bn[B.plans[p].f1_bn == 256 ? 0 : 1].push_back(p);
            }
        const int n = (int)who.size();
        for (int g = 0; g < 2; g++) {
            S.f1_n[g] = (int)who_bn[g].size();
            S.f1_jobs[g] = take(sizeof(F1Job) * S.f1_n[g]);
            S.f1_start[g] = take(sizeof(int) * (S.f1_n[g] + 1));
        }
        S.naux = n;
        S.aux = take(sizeof(ChunkAux) * n);
        S.f2_jobs = take(sizeof(F2P<float>) * n);
        S.f2_start = take(sizeof(int) * (n + 1));
        for (int k = 0; k < 4; k++) {
            S.b1_jobs[k] = take(sizeof(TcB1Params) * n);
            S.b1_start[k] = take(sizeof(int) * (n + 1));
        }
        if (!image) continue;
        if (image->size() < t) image->resize(t);
        char *img = image->data();
        for (int g = 0; g < 2; g++) {
            int *start = (int *)(img + S.f1_start[g]);
            start[0] = 0;
            for (int j = 0; j < S.f1_n[g]; j++) {
                const int p = who_bn[g][j];
                F1Job job;
                std::memset(&job, 0, sizeof(job));
                const OperandMaps &M = maps[p];
                job.m = F1Maps{M.tmA1, M.tmB1, M.tmA2, M.tmB2};
                const int rc = f1_params(B.plans[p], chunks[p][c], B.ws + B.ws_off[p], job.P);
                if (rc != TRIPLES_OK) return rc;
                std::memcpy(img + S.f1_jobs[g] + sizeof(F1Job) * j, &job, sizeof(job));
                start[j + 1] = start[j] + job.P.cum[job.P.ch.nperm];
            }
            S.f1_tiles[g] = start[S.f1_n[g]];
        }
        int *f2s = (int *)(img + S.f2_start);
        f2s[0] = 0;
        int *b1s[4];
        for (int k = 0; k < 4; k++) {
            b1s[k] = (int *)(img + S.b1_start[k]);
            b1s[k][0] = 0;
        }
        for (int j = 0; j < n; j++) {
            const int p = who[j];
            const Plan &P = B.plans[p];
            const ChunkDesc &ch = chunks[p][c];
            char *wsp = B.ws + B.ws_off[p];
            F2P<float> F;
            std::memset(&F, 0, sizeof(F));
            f2_params<float>(P, ch, wsp, B.ios[p], F);   // one segment: every representative, every sub-range triple
            std::memcpy(img + S.f2_jobs + sizeof(F) * j, &F, sizeof(F));
            f2s[j + 1] = f2s[j] + P.n_ijk * F.nsub;
            ChunkAux A;
            std::memset(&A, 0, sizeof(A));
            A.ctrl = (Ctrl *)(wsp + P.off_ctrl);
            A.mo_e = B.ios[p].mo_energy;
            A.e_part = (const double *)(wsp + P.off_epart);
            A.ybar = ybar;
            A.o = P.d.o;
            A.a0 = ch.base[0]; A.na = ch.nabc[0];
            A.b0 = ch.base[1]; A.nb = ch.nabc[1];
            A.c0 = ch.base[2]; A.nc = ch.nabc[2];
            A.n_part = P.n_ijk * F.nsub;
            std::memcpy(img + S.aux + sizeof(A) * j, &A, sizeof(A));
            for (int k = 0; k < 4; k++) {
                TcB1Params Bp;
                std::memset(&Bp, 0, sizeof(Bp));
                const int rc = b1_params(P, ch, wsp, maps[p], k, Bp);
                if (rc != TRIPLES_OK) return rc;
                std::memcpy(img + S.b1_jobs[k] + sizeof(Bp) * j, &Bp, sizeof(Bp));
                b1s[k][j + 1] = b1s[k][j] + Bp.cum[ch.nperm];
            }
        }
        S.f2_ctas = f2s[n];
        for (int k = 0; k < 4; k++) S.b1_tiles[k] = b1s[k][n];
    }
    if (image) image->resize(t);
    B.total = B.tables_off + t;
    return TRIPLES_OK;
}

static int run_batch(const Batch &B, cudaStream_t st) {
    if (B.prec == TRIPLES_PRECISION_FP64) {
        for (int p = 0; p < B.nprob; p++) {
            const int rc = run_impl<double>(B.plans[p], st, B.ios[p]);
            if (rc != TRIPLES_OK) return rc;
        }
        return TRIPLES_OK;
    }
    int rc;
    if ((rc = setup_epilogue<float>()) != TRIPLES_OK) return rc;
    if ((rc = setup_tensor_cores()) != TRIPLES_OK) return rc;
    for (int p = 0; p < B.nprob; p++)
        if ((rc = prep_launches<float>(B.plans[p], st, B.ios[p])) != TRIPLES_OK) return rc;
    const char *tab = B.ws + B.tables_off;
    const int nsm = num_sms();
    const int scaled = B.prec == TRIPLES_PRECISION_MIXED_BF16 ? 0 : 1;
    const F1Maps M0{};
    const TcF1Params T0{};
    const TcB1Params B0{};
    const F2P<float> F0{};
    auto cap = [&](int n) { return n < nsm ? n : nsm; };
    for (const BatchStep &S : B.steps) {
        const F1Job *f1j[2] = {(const F1Job *)(tab + S.f1_jobs[0]), (const F1Job *)(tab + S.f1_jobs[1])};
        const int *f1s[2] = {(const int *)(tab + S.f1_start[0]), (const int *)(tab + S.f1_start[1])};
        if (S.f1_n[0] > 0)
            TB_KLAUNCH(P_F1, (k_f1_tc<256, true><<<cap(S.f1_tiles[0]), kF1Threads, TcCfg<256>::SMEM, st>>>(
                                 M0, T0, f1j[0], f1s[0], S.f1_n[0])));
        if (S.f1_n[1] > 0)
            TB_KLAUNCH(P_F1, (k_f1_tc<128, true><<<cap(S.f1_tiles[1]), kF1Threads, TcCfg<128>::SMEM, st>>>(
                                 M0, T0, f1j[1], f1s[1], S.f1_n[1])));
        const ChunkAux *aux = (const ChunkAux *)(tab + S.aux);
        TB_KLAUNCH(P_PREP, k_chunk_scale_batch<<<S.naux, 32, 0, st>>>(aux, scaled));
        TB_KLAUNCH(P_F2, (k_f2t<float, 8, true><<<S.f2_ctas, F2Smem<8>::NT, f2_smem_bytes<float, 8>(), st>>>(
                             F0, (const F2P<float> *)(tab + S.f2_jobs), (const int *)(tab + S.f2_start), S.naux)));
        TB_KLAUNCH(P_F2, k_energy_sum_batch<<<S.naux, 256, 0, st>>>(aux));
        const TcB1Params *bj[4];
        const int *bs[4];
        for (int k = 0; k < 4; k++) {
            bj[k] = (const TcB1Params *)(tab + S.b1_jobs[k]);
            bs[k] = (const int *)(tab + S.b1_start[k]);
        }
        TB_KLAUNCH(P_B1A, (k_b1_tc<false, 128, true><<<cap(S.b1_tiles[0]), kB1Threads, TcB1Cfg<false, 128>::SMEM, st>>>(
                              B0, bj[0], bs[0], S.naux)));
        TB_KLAUNCH(P_B1B, (k_b1_tc<true, 128, true><<<cap(S.b1_tiles[1]), kB1Threads, TcB1Cfg<true, 128>::SMEM, st>>>(
                              B0, bj[1], bs[1], S.naux)));
        TB_KLAUNCH(P_B1C, (k_b1_tc<false, 64, true><<<cap(S.b1_tiles[2]), kB1Threads, TcB1Cfg<false, 64>::SMEM, st>>>(
                              B0, bj[2], bs[2], S.naux)));
        TB_KLAUNCH(P_B1D, (k_b1_tc<true, 64, true><<<cap(S.b1_tiles[3]), kB1Threads, TcB1Cfg<true, 64>::SMEM, st>>>(
                              B0, bj[3], bs[3], S.naux)));
    }
    for (int p = 0; p < B.nprob; p++)
        if ((rc = fold_launches(B.plans[p], st, B.ios[p])) != TRIPLES_OK) return rc;
    return TRIPLES_OK;
}

void profile_enable(int on) {
    g_prof = on != 0;
    g_prof_recs.clear();
    g_pool_used = 0;
}

int profile_read(int max_cats, double *ms, int *launches) {
    for (int c = 0; c < max_cats && c < P_NCAT; c++) {
        ms[c] = 0.0;
        launches[c] = 0;
    }
    for (const ProfRec &r : g_prof_recs) {
        float t = 0.f;
        if (cudaEventSynchronize(r.b) != cudaSuccess) return -1;
        cudaEventElapsedTime(&t, r.a, r.b);
        if (r.cat < max_cats) {
            ms[r.cat] += t;
            launches[r.cat] += 1;
        }
    }
    return P_NCAT;
}

const char *profile_name(int cat) { return (cat >= 0 && cat < P_NCAT) ? kProfNames[cat] : ""; }
int last_cuda_error() { return g_last_cuda_error; }
void set_last_cuda_error(int e) { g_last_cuda_error = e; }

}  // namespace tb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

size_t triples_workspace_size(int precision, int nocc, int nvir, int ovvv_packed, int want_grad) {
    return triples_workspace_size_ex(precision, nocc, nvir, ovvv_packed, want_grad, nullptr);
}

size_t triples_workspace_size_ex(int precision, int nocc, int nvir, int ovvv_packed, int want_grad,
                                 const triples_options *opt) {
    tb::Plan P;
    if (tb::make_plan(precision, nocc, nvir, ovvv_packed, want_grad, P, 0, opt) != TRIPLES_OK) return 0;
    return P.total;
}

static int triples_call(void *stream, int precision, int nocc, int nvir, int ovvv_packed, int want_grad,
                        const triples_options *opt, const tb::TriplesIO &io, size_t workspace_bytes) {
    tb::Plan P;
    int rc = tb::make_plan(precision, nocc, nvir, ovvv_packed, want_grad, P, 0, opt);
    if (rc != TRIPLES_OK) return rc;
    if (!io.workspace || workspace_bytes < P.total) return TRIPLES_ERR_WORKSPACE;
    if (!io.mo_energy || !io.t1 || !io.t2 || !io.ovoo || !io.ovov || !io.ovvv || !io.fvo || !io.e_out)
        return TRIPLES_ERR_INVALID_ARGUMENT;
    if (want_grad && (!io.mo_energy_bar || !io.t1_bar || !io.t2_bar || !io.ovoo_bar || !io.ovov_bar ||
                      !io.ovvv_bar || !io.fvo_bar))
        return TRIPLES_ERR_INVALID_ARGUMENT;
    return tb::run_triples(P, (cudaStream_t)stream, io);
}

int triples_energy(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                   const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                   const double *ovov, const double *ovvv, const double *fvo, void *workspace,
                   size_t workspace_bytes, double *e_out) {
    tb::TriplesIO io{};
    io.mo_energy = mo_energy; io.t1 = t1; io.t2 = t2; io.ovoo = ovoo; io.ovov = ovov;
    io.ovvv = ovvv; io.fvo = fvo; io.ybar = 1.0; io.workspace = workspace; io.e_out = e_out;
    return triples_call(stream, precision, nocc, nvir, ovvv_packed, 0, nullptr, io, workspace_bytes);
}

int triples_energy_vjp(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                       const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                       const double *ovov, const double *ovvv, const double *fvo, double ybar,
                       void *workspace, size_t workspace_bytes, double *e_out, double *mo_energy_bar,
                       double *t1_bar, double *t2_bar, double *ovoo_bar, double *ovov_bar,
                       double *ovvv_bar, double *fvo_bar) {
    return triples_energy_vjp_ex(stream, precision, nocc, nvir, ovvv_packed, mo_energy, t1, t2, ovoo, ovov,
                                 ovvv, fvo, ybar, 1, nullptr, workspace, workspace_bytes, e_out, mo_energy_bar,
                                 t1_bar, t2_bar, ovoo_bar, ovov_bar, ovvv_bar, fvo_bar);
}

int triples_energy_vjp_ex(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                          const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                          const double *ovov, const double *ovvv, const double *fvo, double ybar,
                          int want_grad, const triples_options *opt, void *workspace, size_t workspace_bytes,
                          double *e_out, double *mo_energy_bar, double *t1_bar, double *t2_bar,
                          double *ovoo_bar, double *ovov_bar, double *ovvv_bar, double *fvo_bar) {
    tb::TriplesIO io{};
    io.mo_energy = mo_energy; io.t1 = t1; io.t2 = t2; io.ovoo = ovoo; io.ovov = ovov;
    io.ovvv = ovvv; io.fvo = fvo; io.ybar = want_grad ? ybar : 1.0; io.workspace = workspace; io.e_out = e_out;
    if (want_grad) {
        io.mo_energy_bar = mo_energy_bar; io.t1_bar = t1_bar; io.t2_bar = t2_bar; io.ovoo_bar = ovoo_bar;
        io.ovov_bar = ovov_bar; io.ovvv_bar = ovvv_bar; io.fvo_bar = fvo_bar;
    }
    return triples_call(stream, precision, nocc, nvir, ovvv_packed, want_grad ? 1 : 0, opt, io, workspace_bytes);
}

// ---- LNO (projected) energy ----
size_t triples_lno_workspace_size(int precision, int nocc, int nvir, int ovvv_packed, int want_grad) {
    return triples_lno_workspace_size_ex(precision, nocc, nvir, ovvv_packed, want_grad, nullptr);
}

size_t triples_lno_workspace_size_ex(int precision, int nocc, int nvir, int ovvv_packed, int want_grad,
                                     const triples_options *opt) {
    tb::Plan P;
    if (tb::make_plan(precision, nocc, nvir, ovvv_packed, want_grad, P, 1, opt) != TRIPLES_OK) return 0;
    return P.total;
}

static int triples_lno_call(void *stream, int precision, int nocc, int nvir, int ovvv_packed, int want_grad,
                            const triples_options *opt, const tb::TriplesIO &io, size_t workspace_bytes) {
    tb::Plan P;
    int rc = tb::make_plan(precision, nocc, nvir, ovvv_packed, want_grad, P, 1, opt);
    if (rc != TRIPLES_OK) return rc;
    if (!io.workspace || workspace_bytes < P.total) return TRIPLES_ERR_WORKSPACE;
    if (!io.mat || !io.mo_energy || !io.t1 || !io.t2 || !io.ovoo || !io.ovov || !io.ovvv || !io.fvo || !io.e_out)
        return TRIPLES_ERR_INVALID_ARGUMENT;
    if (want_grad && (!io.mat_bar || !io.mo_energy_bar || !io.t1_bar || !io.t2_bar || !io.ovoo_bar ||
                      !io.ovov_bar || !io.ovvv_bar || !io.fvo_bar))
        return TRIPLES_ERR_INVALID_ARGUMENT;
    return tb::run_triples(P, (cudaStream_t)stream, io);
}

int triples_lno_energy(void *stream, int precision, int nocc, int nvir, int ovvv_packed, const double *mat,
                       const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                       const double *ovov, const double *ovvv, const double *fvo, void *workspace,
                       size_t workspace_bytes, double *e_out) {
    return triples_lno_energy_vjp_ex(stream, precision, nocc, nvir, ovvv_packed, mat, mo_energy, t1, t2, ovoo, ovov,
                                     ovvv, fvo, 1.0, 0, nullptr, workspace, workspace_bytes, e_out, nullptr,
                                     nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
}

int triples_lno_energy_vjp(void *stream, int precision, int nocc, int nvir, int ovvv_packed, const double *mat,
                           const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                           const double *ovov, const double *ovvv, const double *fvo, double ybar,
                           void *workspace, size_t workspace_bytes, double *e_out, double *mat_bar,
                           double *mo_energy_bar, double *t1_bar, double *t2_bar, double *ovoo_bar,
                           double *ovov_bar, double *ovvv_bar, double *fvo_bar) {
    return triples_lno_energy_vjp_ex(stream, precision, nocc, nvir, ovvv_packed, mat, mo_energy, t1, t2, ovoo, ovov,
                                     ovvv, fvo, ybar, 1, nullptr, workspace, workspace_bytes, e_out, mat_bar,
                                     mo_energy_bar, t1_bar, t2_bar, ovoo_bar, ovov_bar, ovvv_bar, fvo_bar);
}

int triples_lno_energy_vjp_ex(void *stream, int precision, int nocc, int nvir, int ovvv_packed, const double *mat,
                              const double *mo_energy, const double *t1, const double *t2, const double *ovoo,
                              const double *ovov, const double *ovvv, const double *fvo, double ybar,
                              int want_grad, const triples_options *opt, void *workspace, size_t workspace_bytes,
                              double *e_out, double *mat_bar, double *mo_energy_bar, double *t1_bar,
                              double *t2_bar, double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                              double *fvo_bar) {
    tb::TriplesIO io{};
    io.mat = mat;
    io.mo_energy = mo_energy; io.t1 = t1; io.t2 = t2; io.ovoo = ovoo; io.ovov = ovov;
    io.ovvv = ovvv; io.fvo = fvo; io.ybar = want_grad ? ybar : 1.0; io.workspace = workspace; io.e_out = e_out;
    if (want_grad) {
        io.mat_bar = mat_bar;
        io.mo_energy_bar = mo_energy_bar; io.t1_bar = t1_bar; io.t2_bar = t2_bar; io.ovoo_bar = ovoo_bar;
        io.ovov_bar = ovov_bar; io.ovvv_bar = ovvv_bar; io.fvo_bar = fvo_bar;
    }
    return triples_lno_call(stream, precision, nocc, nvir, ovvv_packed, want_grad ? 1 : 0, opt, io,
                            workspace_bytes);
}

// ---- LNO host tables (introspection) ----
size_t triples_lno_tables(void *out, size_t bytes) {
    const size_t need = sizeof(tb::LnoTables) + 16 * sizeof(tb::LnoPattern);
    if (out && bytes >= need) {
        tb::LnoTables t;
        tb::LnoPattern pats[16];
        tb::lno_build_tables(t);
        tb::lno_build_patterns(pats);
        std::memcpy(out, &t, sizeof(t));
        std::memcpy((char *)out + sizeof(t), pats, sizeof(pats));
    }
    return need;
}

// ---- density-fitted ERI producer ----
// ovvv[(p,x), pair] = sum_P Lov[P,(p,x)] Lvv[P,pair]  (pyscfad/cc/dfccsd.py:77-88), packed
// pairs f >= y at f(f+1)/2 + y, built on the device by one FP64 GEMM; the (T)
// path then runs on it with packed ovvv, and the packed ovvv cotangent maps
// back to
//   Lov_bar[P,(p,x)] = sum_pair ovvv_bar[(p,x),pair] Lvv[P,pair]
//   Lvv_bar[P,pair]  = sum_(p,x) ovvv_bar[(p,x),pair] Lov[P,(p,x)]
// (two more GEMMs, the same FP64 tile as the FP64 contractions).
struct DfLayout {
    tb::Plan P;
    size_t off_ovvv, off_gvvv, total;
};

static int df_layout(int precision, int nocc, int nvir, int naux, int want_grad, DfLayout &L) {
    if (naux < 1) return TRIPLES_ERR_INVALID_ARGUMENT;
    int rc = tb::make_plan(precision, nocc, nvir, 1, want_grad, L.P);
    if (rc != TRIPLES_OK) return rc;
    const size_t nov = (size_t)nocc * nvir, npair = (size_t)nvir * (nvir + 1) / 2;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t off = al(L.P.total);
    L.off_ovvv = off;
    off = al(off + nov * npair * sizeof(double));
    L.off_gvvv = off;
    if (want_grad) off = al(off + nov * npair * sizeof(double));
    L.total = off;
    return TRIPLES_OK;
}

size_t triples_df_workspace_size(int precision, int nocc, int nvir, int naux, int want_grad) {
    DfLayout L;
    if (df_layout(precision, nocc, nvir, naux, want_grad, L) != TRIPLES_OK) return 0;
    return L.total;
}

static int triples_df_call(void *stream, int precision, int nocc, int nvir, int naux, int want_grad,
                           const double *Lov, const double *Lvv, tb::TriplesIO io, size_t workspace_bytes,
                           double *Lov_bar, double *Lvv_bar) {
    DfLayout L;
    int rc = df_layout(precision, nocc, nvir, naux, want_grad, L);
    if (rc != TRIPLES_OK) return rc;
    if (!io.workspace || workspace_bytes < L.total) return TRIPLES_ERR_WORKSPACE;
    if (!Lov || !Lvv || !io.mo_energy || !io.t1 || !io.t2 || !io.ovoo || !io.ovov || !io.fvo || !io.e_out)
        return TRIPLES_ERR_INVALID_ARGUMENT;
    if (want_grad && (!Lov_bar || !Lvv_bar || !io.mo_energy_bar || !io.t1_bar || !io.t2_bar || !io.ovoo_bar ||
                      !io.ovov_bar || !io.fvo_bar))
        return TRIPLES_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    char *ws = (char *)io.workspace;
    double *ovvv = (double *)(ws + L.off_ovvv), *gvvv = (double *)(ws + L.off_gvvv);
    const long long nov = (long long)nocc * nvir, npair = (long long)nvir * (nvir + 1) / 2;
    // ovvv[px][pair] = sum_P Lov[P][px] Lvv[P][pair]
    if ((rc = tb::gemm_plain(st, (int)nov, (int)npair, naux, Lov, 1, nov, Lvv, 1, npair, ovvv, npair, 1)) !=
        TRIPLES_OK)
        return rc;
    io.ovvv = ovvv;
    io.ovvv_bar = want_grad ? gvvv : nullptr;
    if ((rc = tb::run_triples(L.P, st, io)) != TRIPLES_OK) return rc;
    if (!want_grad) return TRIPLES_OK;
    // Lov_bar[P][px] = sum_pair G[px][pair] Lvv[P][pair]
    if ((rc = tb::gemm_plain(st, (int)nov, naux, (int)npair, gvvv, npair, 1, Lvv, npair, 1, Lov_bar, 1, nov)) !=
        TRIPLES_OK)
        return rc;
    // Lvv_bar[P][pair] = sum_px G[px][pair] Lov[P][px]
    return tb::gemm_plain(st, (int)npair, naux, (int)nov, gvvv, 1, npair, Lov, nov, 1, Lvv_bar, 1, npair);
}

int triples_energy_df(void *stream, int precision, int nocc, int nvir, int naux, const double *mo_energy,
                      const double *t1, const double *t2, const double *ovoo, const double *ovov, const double *Lov,
                      const double *Lvv, const double *fvo, void *workspace, size_t workspace_bytes, double *e_out) {
    tb::TriplesIO io{};
    io.mo_energy = mo_energy; io.t1 = t1; io.t2 = t2; io.ovoo = ovoo; io.ovov = ovov;
    io.fvo = fvo; io.ybar = 1.0; io.workspace = workspace; io.e_out = e_out;
    return triples_df_call(stream, precision, nocc, nvir, naux, 0, Lov, Lvv, io, workspace_bytes, nullptr, nullptr);
}

int triples_energy_vjp_df(void *stream, int precision, int nocc, int nvir, int naux, const double *mo_energy,
                          const double *t1, const double *t2, const double *ovoo, const double *ovov,
                          const double *Lov, const double *Lvv, const double *fvo, double ybar, void *workspace,
                          size_t workspace_bytes, double *e_out, double *mo_energy_bar, double *t1_bar,
                          double *t2_bar, double *ovoo_bar, double *ovov_bar, double *Lov_bar, double *Lvv_bar,
                          double *fvo_bar) {
    tb::TriplesIO io{};
    io.mo_energy = mo_energy; io.t1 = t1; io.t2 = t2; io.ovoo = ovoo; io.ovov = ovov;
    io.fvo = fvo; io.ybar = ybar; io.workspace = workspace; io.e_out = e_out;
    io.mo_energy_bar = mo_energy_bar; io.t1_bar = t1_bar; io.t2_bar = t2_bar; io.ovoo_bar = ovoo_bar;
    io.ovov_bar = ovov_bar; io.fvo_bar = fvo_bar;
    return triples_df_call(stream, precision, nocc, nvir, naux, 1, Lov, Lvv, io, workspace_bytes, Lov_bar, Lvv_bar);
}

// Fixed scratch for callers that may not allocate device memory themselves
// (for example code running inside another framework's memory pool or a
// host program that must keep its device footprint fixed).  Every device
// that loads this library holds the array until the process exits.  The
// call clears what must start at zero (its control block and gradient
// accumulators) on each use, so the last call's leftovers do no harm; two
// calls whose GPU work overlaps share the array and race.
static constexpr size_t kStaticScratchBytes = TRIPLES_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];
static constexpr int kStaticMaxDevices = 64;
// Device address of the array per device, looked up once with that device
// current.  Host threads making their first call on a device at the same
// time both store the same address; the cache assumes the device's primary
// context lives as long as the process.
static std::atomic<void *> g_static_scratch_addr[kStaticMaxDevices];

static int static_scratch_address(void **addr_out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        tb::set_last_cuda_error((int)e);
        return TRIPLES_ERR_CUDA;
    }
    if (dev < 0 || dev >= kStaticMaxDevices) return TRIPLES_ERR_UNSUPPORTED;
    void *addr = g_static_scratch_addr[dev].load(std::memory_order_acquire);
    if (addr == nullptr) {
        // the array's host-side name is only a stand-in for the symbol
        e = cudaGetSymbolAddress(&addr, g_static_scratch);
        if (e != cudaSuccess || addr == nullptr) {
            tb::set_last_cuda_error((int)e);
            return TRIPLES_ERR_CUDA;
        }
        g_static_scratch_addr[dev].store(addr, std::memory_order_release);
    }
    *addr_out = addr;
    return TRIPLES_OK;
}

int triples_energy_vjp_static(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                              const double *mo_energy, const double *t1, const double *t2,
                              const double *ovoo, const double *ovov, const double *ovvv,
                              const double *fvo, double ybar, double *e_out, double *mo_energy_bar,
                              double *t1_bar, double *t2_bar, double *ovoo_bar, double *ovov_bar,
                              double *ovvv_bar, double *fvo_bar) {
    const size_t need = triples_workspace_size(precision, nocc, nvir, ovvv_packed, 1);
    if (need == 0) return TRIPLES_ERR_INVALID_ARGUMENT;
    if (need > kStaticScratchBytes) return TRIPLES_ERR_WORKSPACE;   // problem too large for the fixed scratch
    void *scratch = nullptr;
    const int rc = static_scratch_address(&scratch);
    if (rc != TRIPLES_OK) return rc;
    return triples_energy_vjp(stream, precision, nocc, nvir, ovvv_packed, mo_energy, t1, t2, ovoo, ovov, ovvv,
                              fvo, ybar, scratch, kStaticScratchBytes, e_out, mo_energy_bar, t1_bar, t2_bar,
                              ovoo_bar, ovov_bar, ovvv_bar, fvo_bar);
}

int triples_static_scratch(void **ptr, size_t *bytes) {
    if (!ptr) return TRIPLES_ERR_INVALID_ARGUMENT;
    const int rc = static_scratch_address(ptr);
    if (rc == TRIPLES_OK && bytes) *bytes = kStaticScratchBytes;
    return rc;
}

int triples_static_check_device_status(void *stream) {
    void *scratch = nullptr;
    const int rc = static_scratch_address(&scratch);
    if (rc != TRIPLES_OK) return rc;
    return triples_check_device_status(stream, scratch);
}

int triples_check_device_status(void *stream, const void *workspace) {
    if (!workspace) return TRIPLES_ERR_INVALID_ARGUMENT;
    tb::Ctrl c;
    cudaError_t e = cudaMemcpyAsync(&c, workspace, sizeof(c), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) {
        tb::set_last_cuda_error((int)e);
        return TRIPLES_ERR_CUDA;
    }
    return c.err ? TRIPLES_ERR_DEVICE_TIMEOUT : TRIPLES_OK;
}

// ---- batched calls ----
struct triples_batch {
    tb::Batch b;
};

size_t triples_batch_workspace_size(int precision, int nprob, const triples_problem *probs) {
    tb::Batch B;
    if (tb::batch_build(B, precision, nprob, probs, 1.0, nullptr) != TRIPLES_OK) return 0;
    return B.total;
}

int triples_batch_create(int precision, int nprob, const triples_problem *probs, double ybar, void *workspace,
                         size_t workspace_bytes, triples_batch **batch) {
    if (!batch) return TRIPLES_ERR_INVALID_ARGUMENT;
    *batch = nullptr;
    if (!workspace) return TRIPLES_ERR_WORKSPACE;
    {
        // the workspace must hold the batch before any table points into it
        tb::Batch sizing;
        const int rc = tb::batch_build(sizing, precision, nprob, probs, ybar, nullptr);
        if (rc != TRIPLES_OK) return rc;
        if (workspace_bytes < sizing.total) return TRIPLES_ERR_WORKSPACE;
    }
    triples_batch *h = new (std::nothrow) triples_batch;
    if (!h) return TRIPLES_ERR_INVALID_ARGUMENT;
    h->b.ws = (char *)workspace;
    std::vector<char> image;
    int rc = tb::batch_build(h->b, precision, nprob, probs, ybar, &image);
    if (rc == TRIPLES_OK && !image.empty()) {
        const cudaError_t e = cudaMemcpy(h->b.ws + h->b.tables_off, image.data(), image.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            tb::set_last_cuda_error((int)e);
            rc = TRIPLES_ERR_CUDA;
        }
    }
    if (rc != TRIPLES_OK) {
        delete h;
        return rc;
    }
    *batch = h;
    return TRIPLES_OK;
}

int triples_batch_run(triples_batch *batch, void *stream) {
    if (!batch) return TRIPLES_ERR_INVALID_ARGUMENT;
    return tb::run_batch(batch->b, (cudaStream_t)stream);
}

int triples_batch_check_device_status(triples_batch *batch, void *stream) {
    if (!batch) return TRIPLES_ERR_INVALID_ARGUMENT;
    int status = TRIPLES_OK;
    for (int p = 0; p < batch->b.nprob; p++) {
        const int rc = triples_check_device_status(stream, batch->b.ws + batch->b.ws_off[p]);
        if (rc == TRIPLES_ERR_CUDA) return rc;
        if (rc != TRIPLES_OK) status = rc;
    }
    return status;
}

void triples_batch_destroy(triples_batch *batch) { delete batch; }

const char *triples_status_string(int status) {
    switch (status) {
    case TRIPLES_OK: return "ok";
    case TRIPLES_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TRIPLES_ERR_WORKSPACE: return "workspace too small";
    case TRIPLES_ERR_CUDA: return "CUDA error";
    case TRIPLES_ERR_UNSUPPORTED: return "unsupported precision or device";
    case TRIPLES_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
    }
}

int triples_last_cuda_error(void) { return tb::last_cuda_error(); }

const char *triples_version(void) { return "0.1.0"; }

void triples_profile_enable(int on) { tb::profile_enable(on); }

int triples_profile_read(int max_categories, double *ms, int *launches) {
    if (max_categories < 0 || (max_categories > 0 && (!ms || !launches))) return -1;
    return tb::profile_read(max_categories, ms, launches);
}

const char *triples_profile_name(int category) { return tb::profile_name(category); }

}  // extern "C"

// Internal planning structures shared by the (T) drivers.
#pragma once
#include <cstddef>

#include "common.cuh"
#include "f2.cuh"
#include "pyscfad_b200.h"

namespace tb {

constexpr int kF2Threads = 256;   // chunk-epilogue block size
constexpr int kMaxTv = 16;        // largest virtual block
constexpr int kMaxCols = 1024;    // largest nocc * Tv (one staged (r, z) row)
constexpr int kCtrlBytes = 256;   // control block at workspace offset 0
constexpr int kLnoGrid = 1184;    // LNO streaming kernels: most blocks per ordering (energy partials)
constexpr int kLnoArrays = 4;     // LNO whole-chunk FP64 work arrays (with the adjoint)
constexpr double kLnoBudgetBytes = 96e9;   // their largest total before the block size is halved

// Control block (workspace offset 0)
struct Ctrl {
    int err;                      // device-side error bits (bounded waits that gave up)
    double e_acc;                 // E(T) accumulator
    double scale[2];              // operand scales (A: ovvv/ovoo, B: t2), powers of two
    float out_scale;              // 1 / (scale[0] * scale[1])
    float pad_;
    double wscale;                // per-chunk power-of-two scale of the split Wbar
    unsigned long long absmax[6]; // bit patterns of max |ovvv|, |ovoo|, |t2|, |ovov|, |t1|, |fvo|
    unsigned wmax_bits;           // bit pattern of max |W| of the current chunk (F1)
    double lno_norm[2];           // LNO projector: max abs row sum, max abs column sum
};

static_assert(sizeof(Ctrl) <= kCtrlBytes, "control block too large");

struct Plan {
    Dims d;
    int a0, a1;      // chunk slice by largest virtual block (a1 <= 0: no upper bound)
    int kseg;        // 64-wide K blocks per FP32 accumulation segment (mixed precision)
    int f1_bn;       // N tile of the tensor-core W contraction (128 or 256)
    int prec, want_grad, packed;
    int lno;         // projected (LNO) energy: whole-chunk work arrays off_L
    int nb;          // number of virtual blocks
    int n_ijk;       // occupied triplet representatives i >= j >= k
    int max_items;   // largest |A||B||C| over chunks
    int f2_gy;       // epilogue grid.y upper bound
    int Kp8, Op8;    // 16-byte padded contraction lengths of the 16-bit operands
    size_t stage_elems, stage_bytes, wbar_elems;
    size_t off_ctrl;
    size_t off_A1, off_B1, off_A2, off_B2, off_S, off_SW;
    size_t off_A1h, off_B1h, off_A2h, off_B2h;
    size_t off_GA1, off_GB1, off_GA2, off_GB2;
    size_t off_ijk, off_epart;
    size_t off_L[4], off_lpart;
    size_t total;
};

struct TriplesIO {
    const double *mo_energy, *t1, *t2, *ovoo, *ovov, *ovvv, *fvo;
    const double *mat;             // LNO projector [o,o] (lno plans only)
    double ybar;
    void *workspace;
    double *e_out;
    double *mo_energy_bar, *t1_bar, *t2_bar, *ovoo_bar, *ovov_bar, *ovvv_bar, *fvo_bar;
    double *mat_bar;
};

int make_plan(int precision, int nocc, int nvir, int packed, int want_grad, Plan &P, int lno = 0,
              const triples_options *opt = nullptr);
int run_triples(const Plan &P, cudaStream_t st, const TriplesIO &io);
int gemm_plain(cudaStream_t st, int M, int N, int K, const double *A, long long ams, long long aks,
               const double *B, long long bms, long long bks, double *C, long long cms, long long cns);

}  // namespace tb

/*
 * pyscfad_b200 -- C ABI of the B200 (sm_100a) CCSD(T) perturbative-triples
 * energy and its adjoint.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * (passed as void*), allocates nothing itself unless stated, never
 * synchronises the stream, and returns a triples_status (0 = success).
 * The library keeps no settings between calls: everything that shapes a
 * call arrives with it (arguments, triples_options), so host threads may
 * call it concurrently on different streams and workspaces (the reference's
 * C kernels are likewise re-entrant).  The first call on a device does a
 * one-time set-up (kernel attributes, constant tables) under a lock; make it
 * before any stream capture.
 *
 * Array layouts are the reference's canonical ones (C order, FP64), i.e. the
 * leaves of pyscfad's ERI pytree and the CCSD amplitudes:
 *   mo_energy[n]          n = nocc + nvir      (eris.mo_energy)
 *   t1[o,v], t2[o,o,v,v]                       (mycc.t1, mycc.t2)
 *   ovoo[o,v,o,o]                              (eris.ovoo)
 *   ovov[o,v,o,v]                              (eris.ovov)
 *   ovvv[o,v,v(v+1)/2]  when ovvv_packed != 0  (eris.ovvv of DF ERIs,
 *                                               pyscfad/cc/dfccsd.py:88)
 *   ovvv[o,v,v,v]       when ovvv_packed == 0
 *   fvo[v,o]            = fock[o:,:o]          (pyscfad/cc/ccsd_t.py:93)
 *
 * Reference interfaces replaced (pyscfadlib, ctypes-bound through
 * pyscfadlib/pyscfadlib/lib.py:3-12):
 *   - the forward, pyscf.cc.ccsd_t.kernel called at pyscfad/cc/ccsd_t.py:41
 *     (and lnoccsdt_contract, pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c:96-100,
 *     with mat = identity);
 *   - the adjoint, ccsd_t_energy_vjp
 *     (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-346) together with the
 *     host-side preparation and fold of _ccsd_t_energy_vjp
 *     (pyscfad/cc/ccsd_t.py:82-192).
 */
#ifndef PYSCFAD_B200_H
#define PYSCFAD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum triples_status {
    TRIPLES_OK = 0,
    TRIPLES_ERR_INVALID_ARGUMENT = 1,  /* bad size, null pointer, bad enum */
    TRIPLES_ERR_WORKSPACE = 2,         /* workspace smaller than triples_workspace_size() */
    TRIPLES_ERR_CUDA = 3,              /* a CUDA call failed; see triples_last_cuda_error() */
    TRIPLES_ERR_UNSUPPORTED = 4,       /* precision / device not supported */
    TRIPLES_ERR_DEVICE_TIMEOUT = 5     /* a bounded device-side wait gave up */
};

enum triples_precision {
    TRIPLES_PRECISION_FP64 = 0,       /* all contractions in FP64 */
    TRIPLES_PRECISION_MIXED = 1,      /* tcgen05 contractions on fp16 hi/lo splits with
                                         power-of-two scaling (3 products, ~22-bit
                                         operands), FP32 accumulate; FP64 denominators
                                         and energy sums */
    TRIPLES_PRECISION_MIXED_BF16 = 2  /* same with unscaled bf16 hi/lo splits (~16-bit) */
};

/* Per-call settings of triples_energy_vjp_ex / triples_workspace_size_ex.
 * All zero (or a NULL pointer) gives the defaults the plain entry points use. */
typedef struct triples_options {
    /* virtual block size Tv of the chunk decomposition: 0 = default (16);
     * rounded down to a power of two, clamped to [1,16] and to nocc*Tv <= 1024.
     * Changes the workspace size and the FP64 summation order, nothing else. */
    int block_size;
    /* only the chunks whose largest virtual block index lies in
     * [chunk_a0, chunk_a1) (chunk_a1 <= 0: no upper bound); (0, 0) = the whole
     * problem.  The energy and gradients are then the partial sums over those
     * chunks, which add up exactly over a partition of the blocks.  With
     * Tv = 16, block A holds the virtual indices [16A, 16A+16), so slice
     * [A, A+1) is the reference's job range a in [16A, 16A+16), b0 = 0,
     * b1 = a1 of ccsd_t_energy_vjp (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-346). */
    int chunk_a0, chunk_a1;
    /* mixed precision: 64-wide K blocks the tensor cores accumulate in FP32
     * before the partial result is added in higher precision; 0 = default (1). */
    int accumulation_segment;
    /* mixed precision: N tile of the W contraction, 128 or 256 columns
     * (8 or 16 occupied indices x 16 virtuals); 0 = 256 unless padding nocc
     * to 16 wastes over a quarter of it.  Performance only. */
    int tile_n;
} triples_options;

/* Bytes of device workspace the calls below need for this problem.
 * want_grad = 0 sizes triples_energy, 1 sizes triples_energy_vjp. */
size_t triples_workspace_size(int precision, int nocc, int nvir, int ovvv_packed,
                              int want_grad);
size_t triples_workspace_size_ex(int precision, int nocc, int nvir, int ovvv_packed,
                                 int want_grad, const triples_options *opt);

/* E(T) into *e_out (device FP64 scalar).
 * Replaces the forward of pyscfad/cc/ccsd_t.py:37-42 (pyscf's ccsd_t.kernel). */
int triples_energy(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                   const double *mo_energy, const double *t1, const double *t2,
                   const double *ovoo, const double *ovov, const double *ovvv,
                   const double *fvo,
                   void *workspace, size_t workspace_bytes,
                   double *e_out);

/* E(T) and its vector-Jacobian product for adjoint seed ybar.
 * Gradient outputs are OVERWRITTEN (the reference accumulates into
 * caller-zeroed buffers, ccsd_t.py:89-106; the result is the same).
 * Each gradient has the layout of its input; ovvv_bar is packed
 * [o,v,v(v+1)/2] exactly as pyscfad/cc/ccsd_t.py:184-191 folds it when
 * ovvv_packed != 0, and the unsymmetrised [o,v,v,v] gradient otherwise.
 * fvo_bar is the vo block of fock_bar (ccsd_t.py:181-182).
 * Replaces ccsd_t_energy_vjp (pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332)
 * plus _ccsd_t_energy_vjp's blocking and fold (pyscfad/cc/ccsd_t.py:82-192). */
int triples_energy_vjp(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                       const double *mo_energy, const double *t1, const double *t2,
                       const double *ovoo, const double *ovov, const double *ovvv,
                       const double *fvo, double ybar,
                       void *workspace, size_t workspace_bytes,
                       double *e_out,
                       double *mo_energy_bar, double *t1_bar, double *t2_bar,
                       double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                       double *fvo_bar);

/* triples_energy (want_grad = 0; gradient pointers may be NULL) or
 * triples_energy_vjp (want_grad = 1) with per-call settings `opt` (NULL =
 * defaults); the workspace is sized by triples_workspace_size_ex with the
 * same `opt`. */
int triples_energy_vjp_ex(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                          const double *mo_energy, const double *t1, const double *t2,
                          const double *ovoo, const double *ovov, const double *ovvv,
                          const double *fvo, double ybar, int want_grad,
                          const triples_options *opt,
                          void *workspace, size_t workspace_bytes,
                          double *e_out,
                          double *mo_energy_bar, double *t1_bar, double *t2_bar,
                          double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                          double *fvo_bar);

/* LNO (T): the triples energy of a local-natural-orbital fragment, in which
 * the first occupied index of the projected amplitude runs through the
 * projector mat[o,o] (pyscfad/lno/ccsd_t.py:42, mat = ulo^T ulo):
 *   E = (1/3) sum_{ijk,abc} (sum_l mat[l,i] W[l,j,k]) Z[i,j,k] / D[i,j,k]
 * in the index convention of triples_energy (mat = identity gives E(T)).
 * nocc <= 64 (TRIPLES_ERR_UNSUPPORTED otherwise); every precision: the
 * mixed ones run the W contraction and the adjoint contractions on the tensor
 * cores as triples_energy does and the projected epilogue in FP64.  Other
 * arguments, layouts and
 * workspace rules are those of triples_energy / triples_energy_vjp;
 * triples_lno_workspace_size sizes the workspace of these two calls.
 * Replaces lnoccsdt_contract (pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t.c:96)
 * with the 2/3 of pyscfad/lno/ccsd_t.py:111, and lnoccsdt_energy_vjp
 * (pyscfadlib/pyscfadlib/vjp/cc/lno_ccsd_t_vjp.c:400) with the host-side
 * preparation and fold of _ccsd_t_energy_bwd (pyscfad/lno/ccsd_t.py:121-235).
 * mat_bar[o,o] is the cotangent of mat (overwritten, like every gradient). */
size_t triples_lno_workspace_size(int precision, int nocc, int nvir, int ovvv_packed, int want_grad);

int triples_lno_energy(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                       const double *mat, const double *mo_energy, const double *t1,
                       const double *t2, const double *ovoo, const double *ovov,
                       const double *ovvv, const double *fvo,
                       void *workspace, size_t workspace_bytes, double *e_out);

int triples_lno_energy_vjp(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                           const double *mat, const double *mo_energy, const double *t1,
                           const double *t2, const double *ovoo, const double *ovov,
                           const double *ovvv, const double *fvo, double ybar,
                           void *workspace, size_t workspace_bytes,
                           double *e_out, double *mat_bar,
                           double *mo_energy_bar, double *t1_bar, double *t2_bar,
                           double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                           double *fvo_bar);

/* Introspection (host only, no GPU): the gather tables and de-duplication
 * patterns of the LNO orbit tiles, as the library builds them, copied into
 * `out` when `bytes` suffices; returns the size needed.  Layout: six
 * sigma-permuted slot maps [6][64], two r3 slot maps [2][6][64] (slots padded
 * as s + 3 (s / 16)), candidate maps [36][6] and [2][36][6] (a 16-byte aligned
 * block of 1808 bytes), then 16 patterns of {nslab, cand[36], prim[36]}. */
size_t triples_lno_tables(void *out, size_t bytes);

/* The LNO calls with per-call settings (triples_options; NULL = defaults;
 * want_grad = 0 computes the energy alone and ignores the gradient
 * pointers). */
size_t triples_lno_workspace_size_ex(int precision, int nocc, int nvir, int ovvv_packed,
                                     int want_grad, const triples_options *opt);

int triples_lno_energy_vjp_ex(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                              const double *mat, const double *mo_energy, const double *t1,
                              const double *t2, const double *ovoo, const double *ovov,
                              const double *ovvv, const double *fvo, double ybar, int want_grad,
                              const triples_options *opt,
                              void *workspace, size_t workspace_bytes,
                              double *e_out, double *mat_bar,
                              double *mo_energy_bar, double *t1_bar, double *t2_bar,
                              double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                              double *fvo_bar);

/* Density-fitted inputs: the ovvv operand comes from the DF factors as the
 * reference's DF ERIs build it (pyscfad/cc/dfccsd.py:77-88):
 *   Lov[naux, o*v]          = Lpq[:, :o, o:]
 *   Lvv[naux, v(v+1)/2]     = pack_tril(Lpq[:, o:, o:])   (pair f >= y at f(f+1)/2 + y)
 *   ovvv[o*v, v(v+1)/2]     = Lov^T Lvv
 * built on the device, so the caller never holds or transfers the
 * o*v*v(v+1)/2 ovvv array.  Gradients are returned for the factors instead of
 * ovvv: Lov_bar[naux, o*v], Lvv_bar[naux, v(v+1)/2] (the packed convention of
 * Lvv: one entry per pair).  Everything else is exactly triples_energy[_vjp]
 * with ovvv_packed = 1 (the three factor products are FP64 GEMMs in the
 * library). */
size_t triples_df_workspace_size(int precision, int nocc, int nvir, int naux, int want_grad);

int triples_energy_df(void *stream, int precision, int nocc, int nvir, int naux,
                      const double *mo_energy, const double *t1, const double *t2,
                      const double *ovoo, const double *ovov,
                      const double *Lov, const double *Lvv, const double *fvo,
                      void *workspace, size_t workspace_bytes, double *e_out);

int triples_energy_vjp_df(void *stream, int precision, int nocc, int nvir, int naux,
                          const double *mo_energy, const double *t1, const double *t2,
                          const double *ovoo, const double *ovov,
                          const double *Lov, const double *Lvv, const double *fvo, double ybar,
                          void *workspace, size_t workspace_bytes, double *e_out,
                          double *mo_energy_bar, double *t1_bar, double *t2_bar,
                          double *ovoo_bar, double *ovov_bar,
                          double *Lov_bar, double *Lvv_bar, double *fvo_bar);

/* Size of the fixed device scratch behind triples_energy_vjp_static. */
#define TRIPLES_STATIC_SCRATCH_BYTES ((size_t)64 << 20)

/* triples_energy_vjp without a workspace argument and without any device
 * allocation, for callers that may not allocate device memory (code that runs
 * inside another framework's memory pool, or a host program that must keep
 * its device footprint fixed).  No counterpart in the reference, which
 * allocates its own scratch with malloc.
 * The scratch is a fixed array of TRIPLES_STATIC_SCRATCH_BYTES (64 MiB) in
 * the library, held by every device that loads it until the process exits.
 * Problems with triples_workspace_size(precision, nocc, nvir, ovvv_packed, 1)
 * above that limit are rejected with TRIPLES_ERR_WORKSPACE before any GPU
 * work (for example FP64 fits nocc = 5 with nvir up to 57, mixed nocc = 8 with
 * nvir up to 41).
 * The first call on a device looks up the array's device address and does the
 * library's one-time kernel set-up; make that first call before any stream
 * capture.  The address is cached per device for the life of the process
 * (it assumes the device's primary context is not reset).  Each call clears
 * the parts of the scratch that must start at zero.  All calls share the one
 * array: calls whose GPU work overlaps (other streams, other host threads)
 * race and must be serialised by the caller.  Inputs, outputs and results are
 * exactly those of triples_energy_vjp; triples_static_check_device_status
 * reports device-side failures of the last static call. */
int triples_energy_vjp_static(void *stream, int precision, int nocc, int nvir, int ovvv_packed,
                              const double *mo_energy, const double *t1, const double *t2,
                              const double *ovoo, const double *ovov, const double *ovvv,
                              const double *fvo, double ybar,
                              double *e_out,
                              double *mo_energy_bar, double *t1_bar, double *t2_bar,
                              double *ovoo_bar, double *ovov_bar, double *ovvv_bar,
                              double *fvo_bar);

/* Synchronises `stream` and reports device-side failures of the last call
 * that used `workspace` (bounded waits that gave up): TRIPLES_OK or
 * TRIPLES_ERR_DEVICE_TIMEOUT. */
int triples_check_device_status(void *stream, const void *workspace);

/* triples_check_device_status for the fixed scratch of
 * triples_energy_vjp_static on the current device. */
int triples_static_check_device_status(void *stream);

/* Device address and size of that fixed scratch on the current device (the
 * workspace a static call used; its control block, with the device-side
 * error bits, sits at offset 0). */
int triples_static_scratch(void **ptr, size_t *bytes);

/* ---- batched calls: many (T) problems of uneven size -------------------------
 *
 * The reference evaluates one molecule per call (pyscfad/cc/ccsd_t.py:28-192,
 * ccsd_t_energy_vjp at pyscfadlib/pyscfadlib/vjp/cc/ccsd_t_vjp.c:332-346);
 * these entry points run E(T) and its VJP (one adjoint seed for all) for a
 * list of problems, each with the layouts and outputs of
 * triples_energy_vjp.  In the mixed modes every kernel kind is launched once
 * per chunk step over the corresponding chunk of every problem, instead of
 * once per chunk per problem; an FP64 batch runs its problems one after
 * another. */
typedef struct triples_problem {
    int nocc, nvir, ovvv_packed;
    int block_size;   /* virtual block size, 0 = default (triples_options.block_size) */
    int tile_n;       /* W-contraction N tile, 0 = default (triples_options.tile_n) */
    const double *mo_energy, *t1, *t2, *ovoo, *ovov, *ovvv, *fvo;
    double *e_out;
    double *mo_energy_bar, *t1_bar, *t2_bar, *ovoo_bar, *ovov_bar, *ovvv_bar, *fvo_bar;
} triples_problem;

typedef struct triples_batch triples_batch;   /* opaque */

/* Bytes of device workspace a batch of these problems needs (0 on invalid
 * arguments): every problem's workspace plus the batch's job tables. */
size_t triples_batch_workspace_size(int precision, int nprob, const triples_problem *probs);

/* Plans the batch over `workspace` and writes its job tables there (a
 * blocking host-to-device copy: not for stream capture).  The problems'
 * buffers and the workspace must stay allocated, at the same addresses, for
 * as long as the batch is used; their values may change between runs.
 * *batch receives a handle for triples_batch_run / _destroy. */
int triples_batch_create(int precision, int nprob, const triples_problem *probs, double ybar, void *workspace,
                         size_t workspace_bytes, triples_batch **batch);

/* Runs the whole batch on `stream` (asynchronous; no host allocation and no
 * synchronisation, so it can be captured into a CUDA graph after a first
 * eager run has done the library's one-time device set-up).  Runs of the
 * same batch on different streams race on its workspace. */
int triples_batch_run(triples_batch *batch, void *stream);

/* Synchronises `stream` and reports device-side failures of the last run
 * (TRIPLES_ERR_DEVICE_TIMEOUT if any problem's bounded waits gave up). */
int triples_batch_check_device_status(triples_batch *batch, void *stream);

/* Frees the handle (not the workspace). */
void triples_batch_destroy(triples_batch *batch);

/* Human-readable text for a triples_status value. */
const char *triples_status_string(int status);

/* The cudaError_t of the most recent failing CUDA call on this thread. */
int triples_last_cuda_error(void);

/* Measurement: when enabled, every kernel launched by the calls the calling
 * host thread makes is bracketed by CUDA events on the caller's stream
 * (enabling clears earlier records; other threads are not affected).
 * triples_profile_read() synchronises on this thread's events and fills
 * per-category totals (milliseconds, launch counts) for up to max_categories
 * categories; it returns the number of categories, or -1 on error. */
void triples_profile_enable(int on);
int triples_profile_read(int max_categories, double *ms, int *launches);
const char *triples_profile_name(int category);

/* Version of this library, e.g. "0.1.0". */
const char *triples_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PYSCFAD_B200_H */

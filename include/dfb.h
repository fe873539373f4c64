/*
 * libdfb -- B200-native density-fitted two-electron engine, C ABI.
 *
 * Every entry point takes plain device pointers, sizes and a cudaStream_t
 * passed as void*.  All calls are asynchronous on that stream, allocate no
 * device memory of their own (scratch is passed in), and return 0 on success
 * or a negative error code; dfb_last_error() returns the message of the last
 * failure on the calling thread.
 *
 * Index conventions follow the reference engine (ASUKA cuERI):
 *   - Cartesian components x-major: for x=l..0, for y=l-x..0, z=l-x-y
 *     (asuka/cueri/cuda/ext/src/cueri_cuda_kernels_rys_generic.cu:38-50);
 *   - primitive pairs of shell pair (A,B) stored ia*nprimB+ib
 *     (asuka/cueri/cuda/ext/src/cueri_cuda_kernels.cu:61-123);
 *   - DF "pairs" of the metric are (P, dummy) with the dummy an s shell of
 *     exponent 0, coefficient 1 at the origin (asuka/cueri/gpu.py:511-558).
 */
#ifndef DFB_H
#define DFB_H

#ifdef __cplusplus
extern "C" {
#endif

#include "dfb_types.h"

/* Library version (major*10000+minor*100+patch). */
int dfb_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char *dfb_last_error(void);

/*
 * Upload the Rys node/weight table for the current device (once per device).
 * coef: concatenated (nint, 2n, deg+1) blocks for n=1..nmax, offs[n] = start
 * of block n; herm: concatenated (2, n) Gauss-Hermite limits, hoffs[n].
 * Replaces the reference's per-call root solver
 * (asuka/cueri/cuda/ext/src/cueri_cuda_rys_device.cuh:231-529).
 */
int dfb_rys_table_init(const double *coef, const int *offs, long ncoef, const double *herm, const int *hoffs,
                       long nherm, int nmax, int nint, int deg, double tmax);

/*
 * Primitive-pair tables: eta = a+b, P = (aA+bB)/eta, cK = ca cb exp(-ab/eta |AB|^2),
 * plus the exponents a and b.  One entry per primitive pair, pp_sp[i] = owning
 * shell pair, ordered ia*nprimB+ib inside each pair.  pp_local (optional, may be
 * NULL) gives entry i's index ia*nprimB+ib inside its shell pair when the table
 * holds only a subset of the pairs (screened tables); NULL means entries are
 * dense from sp_pstart[sp].  b_dummy=1 builds the metric's (P, dummy) tables
 * (eta=a, P=A, cK=ca, eb=0).
 * Replaces KernelBuildPairTables_ss (asuka/cueri/cuda/ext/src/cueri_cuda_kernels.cu:61-123).
 */
int dfb_pair_tables(const double *cxyz, const int *shell_pstart, const int *shell_nprim, const double *pexp,
                    const double *pcoef, const int *sp_A, const int *sp_B, const int *sp_pstart, const int *pp_sp,
                    const int *pp_local, long npp, int b_dummy, double *eta, double *Px, double *Py, double *Pz, double *cK, double *ea,
                    double *eb, void *stream);

/*
 * Rys integrals for one angular class (la, lb, lc) over ntask tasks, written
 * straight into the output.  Tasks are (task_pair[t], task_aux[t]) when
 * naux_grid == 0, the pair-major grid (task_pair[t / naux_grid], task_aux[t %
 * naux_grid]) when naux_grid > 0 (ntask = npairs * naux_grid), or the aux-major
 * grid (task_pair[t % n], task_aux[t / n]), n = -naux_grid, when naux_grid < 0.  Output (the
 * reference's tile kernel plus scatter, K3+K7, in one pass):
 *   mode 0: 3c, out[(P0+c)*sP + mu*sM + nu*sN] and the (nu, mu) mirror;
 *   mode 1: metric, out[(Q0+c)*sP + (P0+a)*sM] and out[(P0+a)*sP + (Q0+c)*sM].
 * scratch: device buffer of at least dfb_rys_scratch_doubles(...) doubles.
 * Replaces df_int3c2e_rys_device_block / df_metric_2c2e_rys_device
 * (asuka/cueri/gpu.py:2742, :2104) with its launch path
 * (asuka/cueri/eri_dispatch.py:399 run_kernel_batch_spd).
 */
int dfb_rys_int(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux, const int *task_pair,
                const int *task_aux, long ntask, long naux_grid, int mode, double *out, long sP, long sM, long sN, double *scratch,
                long scratch_doubles, void *stream);

/*
 * Derivative contraction for one class: grad[atom, xyz] +=
 *   fac * sum_{abc} bar[abc] * d(ab|c)/dR,  fac = 2 for off-diagonal tasks,
 * bar read as bar[(P0+c)*sbP + mu*sbM + nu*sbN] (mode 0, (mu,nu)-symmetric)
 * or bar[(P0+a)*sbP + (Q0+c)*sbM] (mode 1).  Centre C by translational
 * invariance.  grad is (natm, 3), accumulated.
 * Replaces df_int3c2e_deriv_contracted_cart_allsp_atomgrad_inplace_device and
 * the metric analogue (asuka/integrals/grad.py:537-565, :659-687).
 */
int dfb_rys_deriv(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux,
                  const int *task_pair, const int *task_aux, long ntask, long naux_grid, int mode, const double *bar, long sbP,
                  long sbM, long sbN, double *grad, int natm, double *scratch, long scratch_doubles, void *stream);

/*
 * FP64 FMA throughput probe: blocks x threads threads each run iters x 64
 * dependent-chain FMAs (8 chains); out holds blocks*threads doubles.  Used to
 * measure the FP64 peak that bounds the Rys kernels (no reference counterpart).
 */
int dfb_fp64_fma_probe(double *out, int blocks, int threads, int iters, void *stream);

/* FP32 FMA throughput probe (the roofline denominator of the FP32 recurrences of the
 * mixed-precision Rys kernels): blocks x threads threads each run iters x 64 FMAs in
 * 16 independent chains; out holds blocks*threads floats.  No reference counterpart. */
int dfb_fp32_fma_probe(float *out, int blocks, int threads, int iters, void *stream);

/* Number of kernels the library has launched in this process (all entry points). */
long dfb_launch_count(void);

/*
 * Allocation-free variant of dfb_rys_int for callers that cannot allocate
 * device memory (frameworks that hand over only input/output buffers, code
 * under an allocator that forbids new device allocations).  No counterpart in
 * the reference.  Same arguments and output as dfb_rys_int without the
 * scratch buffer: the generic warp kernel uses a fixed 8 MiB scratch array
 * (2^20 doubles) in the library's device image (held by every GPU that loads the
 * library), and the class's tasks run in batches of floor(2^20 / slot) tasks per
 * pair of launches, slot being one task's contracted intermediate; a class fails
 * with DFB_ERR_UNSUPPORTED only if a single task's slot exceeds the array (none
 * with l <= 8 does).  The first call on a device looks up
 * the array's address and should come before any stream capture; calls share
 * the array, so calls that overlap on the GPU race.  dfb_rys_table_init must
 * have run on the device.
 */
int dfb_rys_int_noalloc(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux,
                        const int *task_pair, const int *task_aux, long ntask, long naux_grid, int mode, double *out,
                        long sP, long sM, long sN, void *stream);

/* Precision of the Rys kernels (dfb_rys_int_prec, dfb_rys_deriv_prec). */
#define DFB_PREC_FP64 0  /* every step in FP64 (the reference's arithmetic) */
#define DFB_PREC_MIXED 1 /* FP64 roots, weights, prefactors, horizontal recurrence, adjoint contraction and
                            gradient accumulation; FP32 2D recurrence tables and per-task accumulation */

/*
 * dfb_rys_int / dfb_rys_deriv with a precision argument.  DFB_PREC_MIXED runs
 * the class-specialised kernels with FP32 recurrence tables and accumulators
 * (about 1e-7 relative per integral); classes that have no specialised
 * kernel run in FP64 either way.  The reference's counterpart is its
 * mixed-precision Rys tile kernels (kMixedPrec,
 * asuka/cueri/cuda/ext/src/generated/cueri_cuda_kernels_wave1_generated.cu:1536)
 * switched on by CuERIDFConfig.mixed_precision (asuka/integrals/cueri_df.py:61-65).
 */
int dfb_rys_int_prec(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux,
                     const int *task_pair, const int *task_aux, long ntask, long naux_grid, int mode, int precision,
                     double *out, long sP, long sM, long sN, double *scratch, long scratch_doubles, void *stream);
int dfb_rys_deriv_prec(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux,
                       const int *task_pair, const int *task_aux, long ntask, long naux_grid, int mode, int precision,
                       const double *bar, long sbP, long sbM, long sbN, double *grad, int natm, double *scratch,
                       long scratch_doubles, void *stream);

/*
 * One operand of dfb_tc_gemm.  Element (row, k) of batch entry b is
 *   ptr[b*s_batch + row*s_row + (k / nk1)*s_kq + (k % nk1)*s_k1],
 * so strided views need no copy (the exchange update's W[Q, mu, i] with k = (Q, i):
 * s_row = nocc, s_kq = nao*nocc, s_k1 = 1, nk1 = nocc).
 */
typedef struct {
    const double *ptr;
    long s_row, s_kq, s_k1, nk1, s_batch;
} dfb_tc_operand_t;

/*
 * Split-BF16 tensor-core GEMM (tcgen05, sm_100a):
 *   C[b][m*ldc + n] (+)= sum_k A(m, k) B(n, k),  b < batch, C at C + b*s_cbatch.
 * Each FP64 element is split into nterms (2 or 3) bfloat16 terms; the products of
 * order <= 2^-8 (nterms 2) or 2^-16 (nterms 3) run on the tensor cores with FP32
 * accumulation over k spans of kspan (<= 0: all of K), and the spans are combined
 * in FP64.  accumulate=0 stores C (needs one span, kspan >= K); accumulate=1 adds
 * with FP64 atomics (C must hold the start value).  symmetric=1 (A == B, M == N)
 * computes the tiles on and above the diagonal and mirrors them.  About 1e-7
 * relative (nterms 3).  Replaces the reference's cuBLAS DGEMM calls of the DF J/K
 * workspace (asuka/hf/cuda/ext/src/hf_df_jk_cuda_ext.cpp:231-598) in mixed mode.
 */
int dfb_tc_gemm(long M, long N, long K, long batch, const dfb_tc_operand_t *A, const dfb_tc_operand_t *B, double *C,
                long ldc, long s_cbatch, int accumulate, int symmetric, int nterms, long kspan, void *stream);

/* First error code recorded by a bounded wait inside the tensor-core kernels since the
 * last reset (0 = none; 1, 2 = an mbarrier wait gave up).  Synchronous. */
int dfb_tc_error(int reset);

/*
 * Error word of the class-specialised Rys kernels on the current device: 0, or the code of the
 * first bounded wait on a shared-memory copy of the Rys table that gave up (1: the block fell
 * back to the global table; 2: its copy was still in flight at exit).  reset != 0 clears it.
 * Returns a negative DFB_ERR_* code when the table is not uploaded.  No reference counterpart.
 */
int dfb_rys_error(int reset);

/*
 * 3c adjoint of the DF gradient: out[P] = U_P Cw^T for P < nP, written (nP, nao, nao)
 * contiguous and exactly symmetric, where U_P = Cw A_P with A_P symmetric (so U_P Cw^T =
 * Cw A_P Cw^T).  U element (P, mu, j) at U[mu * sU_mu + P * sU_P + j], j < nocc; Cw is
 * (nao, nocc) contiguous.  FP64.  Replaces the adjoint GEMMs of the whitened-factor route
 * (asuka/integrals/df_adjoint.py:172-235); no counterpart of its own in the reference.
 */
int dfb_gamma_sym(long nP, int nao, int nocc, const double *U, long sU_mu, long sU_P, const double *Cw,
                  double *out, void *stream);

/* Scratch doubles dfb_rys_int / dfb_rys_deriv need for this class and task count. */
long dfb_rys_scratch_doubles(int la, int lb, int lc, long ntask, int deriv);

#ifdef __cplusplus
}
#endif
#endif /* DFB_H */

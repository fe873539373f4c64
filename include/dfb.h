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

#define DFB_OK 0
#define DFB_ERR_INVALID (-1)
#define DFB_ERR_CUDA (-2)
#define DFB_ERR_UNSUPPORTED (-3)
#define DFB_ERR_NOT_INITIALISED (-4)

/* AB side of a Rys task: AO shell pairs (A,B), or aux self-pairs (P, dummy). */
typedef struct {
    const int *shA, *shB;          /* per pair: shell indices in the AB basis (shB unused if b_dummy) */
    const int *pstart, *npair;     /* per pair: primitive-pair range in the tables below */
    const double *eta, *Px, *Py, *Pz, *cK;  /* per primitive pair */
    const double *ea, *eb;         /* per primitive pair: exponents of the A and B primitives */
    const double *cxyz;            /* AB basis shell centres (nshell, 3) */
    const int *aostart;            /* AB basis first function of each shell */
    const int *atom;               /* AB basis shell -> atom */
    int b_dummy;                   /* 1: B is the dummy s shell (metric) */
} dfb_pair_side_t;

/* C side of a Rys task: one aux shell (the dummy D is implicit). */
typedef struct {
    const double *cxyz;
    const int *pstart, *nprim;
    const double *pexp, *pcoef;
    const int *aostart;
    const int *atom;
} dfb_aux_side_t;

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

/*
 * Allocation-free variant of dfb_rys_int for callers that cannot allocate
 * device memory (frameworks that hand over only input/output buffers, code
 * under an allocator that forbids new device allocations).  No counterpart in
 * the reference.  Same arguments and output as dfb_rys_int without the
 * scratch buffer: the generic warp kernel uses a fixed 8 MiB scratch array in
 * the library's device image (held by every GPU that loads the library), the
 * persistent grid is shrunk to fit it, and classes that need more than it holds
 * per block fail with DFB_ERR_UNSUPPORTED.  The first call on a device looks up
 * the array's address and should come before any stream capture; calls share
 * the array, so calls that overlap on the GPU race.  dfb_rys_table_init must
 * have run on the device.
 */
int dfb_rys_int_noalloc(int la, int lb, int lc, const dfb_pair_side_t *ps, const dfb_aux_side_t *aux,
                        const int *task_pair, const int *task_aux, long ntask, long naux_grid, int mode, double *out,
                        long sP, long sM, long sN, void *stream);

/* Scratch doubles dfb_rys_int / dfb_rys_deriv need for this class and task count. */
long dfb_rys_scratch_doubles(int la, int lb, int lc, long ntask, int deriv);

#ifdef __cplusplus
}
#endif
#endif /* DFB_H */

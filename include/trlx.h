/*
 * trlx.h -- extensions of the B200 Lanczos engine that have no counterpart
 * in the reference API.  The reference's own entry points (trlan.h,
 * ztrlan.h) are unchanged; everything new lives in trlx_* functions so that
 * trl_info keeps its layout.
 */
#ifndef TRLAN_B200_TRLX_H
#define TRLAN_B200_TRLX_H

#include "trlan.h"
#include "ztrlan.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------
 * Built-in device operators.  Passing trlx_matvec (or trlx_zmatvec) as `op`
 * with info->mvparam pointing at a trlx_operator lets the engine run its
 * fused kernel (sparse product + alpha dot in one pass) instead of a
 * callback; called directly they behave like any trl_matvec on device
 * pointers.  Matrices are square, rows/columns 0-based, CSR row pointers
 * 64-bit.
 * ------------------------------------------------------------------------- */
typedef struct trlx_operator trlx_operator;

#define TRLX_HOST_ARRAYS 0   /* input arrays live in host memory   */
#define TRLX_DEVICE_ARRAYS 1 /* input arrays are device pointers   */

/* Real CSR (values FP64).  Returns 0 or a negative error code. */
int trlx_csr_create(int nrow, const long long *row_ptr, const int *col_idx,
                    const double *val, int where, trlx_operator **out);

/* Real SELL-C-sigma (C = 32) built from CSR input; sigma >= 1 is the
   row-sorting window (1 keeps the natural order).  The layout is built on
   the device (the row order of sigma > 1 on the host, from the row
   pointers); host input arrays are copied to the device first. */
int trlx_sell_create(int nrow, const long long *row_ptr, const int *col_idx,
                     const double *val, int sigma, int where,
                     trlx_operator **out);

/* Complex CSR (values complex128). */
int trlx_zcsr_create(int nrow, const long long *row_ptr, const int *col_idx,
                     const trl_dcomplex *val, int where,
                     trlx_operator **out);

/* Complex SELL-C-sigma (C = 32, values complex128), built like
   trlx_sell_create. */
int trlx_zsell_create(int nrow, const long long *row_ptr, const int *col_idx,
                      const trl_dcomplex *val, int sigma, int where,
                      trlx_operator **out);

/* Waits for the device (like cudaFree), then returns the operator's memory
   to the library's device pool. */
void trlx_operator_destroy(trlx_operator *op);

/* Number of stored entries (including SELL padding) and rows. */
long long trlx_operator_nnz(const trlx_operator *op);
int trlx_operator_nrow(const trlx_operator *op);

/* Single-solve autotuner (no counterpart in the reference, whose operator
   is an opaque callback).  For an operator created with trlx_csr_create or
   trlx_zcsr_create (not distributed) it times, on the current GPU, one
   fused product y = A x + alpha in the CSR form and in the SELL-C-32 form
   built from the same device arrays, and Gram-Schmidt projections over
   maxlan / 4, maxlan / 2 and 3 maxlan / 4 columns (at most 32, 64 and 96)
   of the operator's row count in each of the projection kernel's forms
   (median of 5 launches each, summed over the three widths), over 64-bit
   columns and again
   over 32-bit columns (the two basis storage widths of
   trlx_options.basis_bits); complex operators have the projection forms 3,
   4 and 5 only (the others report -1 ms).  It keeps the faster operator
   form (storage switched in place, the handle stays valid) and the faster
   projection form for each basis width for every later solve with this
   operator (call it before, not during, solves that use the operator).
   Temporary device memory: two vectors and the projection's columns (at
   most a quarter of the free memory).  Returns 0, -1 for an operator it
   does not tune (SELL-created or distributed), -2 if the temporary memory
   cannot be allocated, -3 on a CUDA error. */
typedef struct {
    int format;            /* kept operator form: 0 CSR, 1 SELL-C-32        */
    int project_form;      /* kept projection form: 1, 2, 3: 8, 12, 16
                              columns per warp; 4: 16 columns with the
                              column-pointer table in shared memory; 5: 8
                              columns per warp, 16 warps, the basis staged
                              through shared memory by cp.async, one
                              block per SM                                 */
    double spmv_ms[2];     /* one product: CSR, SELL-C-32 (-1: not built)  */
    double project_ms[5];  /* projections at the three widths, forms 1 .. 5 */
    int columns;           /* middle projection width timed                 */
    double seconds;        /* wall time of the tuning                       */
    int project_form32;    /* kept form for a 32-bit basis (same values)    */
    double project32_ms[5];/* the same over 32-bit columns, forms 1..5     */
} trlx_tune_result;
int trlx_operator_autotune(trlx_operator *op, int maxlan, trlx_tune_result *out);
/* Sets the projection form of later solves with this operator (a
   trlx_tune_result.project_form value, 0 for the default), for example to
   reuse a tuning result on an operator created again from the same matrix.
   Returns 0, or -1 for a null operator or an unknown form. */
int trlx_operator_set_project_form(trlx_operator *op, int project_form);
/* The same for solves over a 32-bit basis (trlx_options.basis_bits = 32; a
   trlx_tune_result.project_form32 value). */
int trlx_operator_set_project_form32(trlx_operator *op, int project_form);

/* trl_matvec / ztrl_matvec compatible appliers (device x, y). */
void trlx_matvec(const int nrow, const int ncol, const double *x,
                 const int ldx, double *y, const int ldy, void *mvparam);
void trlx_zmatvec(const int nrow, const int ncol, const trl_dcomplex *x,
                  const int ldx, trl_dcomplex *y, const int ldy,
                  void *mvparam);

/* ---------------------------------------------------------------------------
 * Kernel-level entry points (device pointers, column-major blocks).
 * ------------------------------------------------------------------------- */
/* Gram-Schmidt projection wrk = [v1 v2]^T rr over two blocks of basis
   columns (v1: m1 columns, leading dimension ld1; v2: m2 columns, ld2):
   the counterpart of the reference's trl_g_dot_ (SRC/trl_comm_none.c:238),
   which the MPI build also uses as the allreduce point.  All pointers are
   device memory; the work is queued on `stream` (a cudaStream_t, NULL for
   the legacy default stream) and wrk is valid once that stream reaches it.
   Deterministic (fixed summation order).  Returns 0, -201 if ld1 or ld2 is
   smaller than nrow (the reference aborts there), -1 on invalid arguments,
   -5 if the reduction scratch cannot be allocated.  nrow = 0 (a rank with
   no local rows) writes zeros. */
int trlx_g_dot(int nrow, const double *v1, int ld1, int m1, const double *v2,
               int ld2, int m2, const double *rr, double *wrk, void *stream);
/* Complex twin: wrk = [v1 v2]^H rr (ztrl_g_dot_, SRC/ztrl_comm_none.c:16). */
int trlx_zg_dot(int nrow, const trl_dcomplex *v1, int ld1, int m1,
                const trl_dcomplex *v2, int ld2, int m2,
                const trl_dcomplex *rr, trl_dcomplex *wrk, void *stream);

/* Allocation-free variant of trlx_g_dot, for callers that must not allocate
   device memory (an application-wide memory budget or caching allocator
   owns the GPU, or the call happens inside an operator callback or another
   hot loop where cudaMalloc could synchronize the device).  No counterpart
   in the reference.  Same arguments, result and error codes as trlx_g_dot;
   it calls no cudaMalloc/cudaFree.  Its reduction scratch is a fixed
   592 KiB array inside the library, held by every GPU that loads the library
   until the process exits; at most TRLX_G_DOT_NOALLOC_MAX_COLS columns
   (m1 + m2), larger requests return -7.  The first call on a device looks
   up that array's device address (cudaGetSymbolAddress) and caches it; under
   CUDA's lazy module loading that lookup also loads the array onto the
   device, so the first call may allocate and synchronize.  Make it once per
   device as a warm-up, outside any memory budget, hot loop or stream
   capture; later calls allocate nothing.  All calls
   share the array: calls whose work overlaps on the GPU (different streams
   or threads on one device) race and must be serialised. */
#define TRLX_G_DOT_NOALLOC_MAX_COLS 512
int trlx_g_dot_noalloc(int nrow, const double *v1, int ld1, int m1,
                       const double *v2, int ld2, int m2, const double *rr,
                       double *wrk, void *stream);

/* ---------------------------------------------------------------------------
 * Solver options.
 * ------------------------------------------------------------------------- */
typedef struct {
    int basis_bits;          /* 64: FP64 (c128) basis; 32: FP32 (c64)     */
    unsigned long long seed; /* seed of the counter-based random restarts */
    void *stream;            /* cudaStream_t to run on; NULL: own stream  */
    int refine;              /* 1: FP64 Rayleigh-Ritz refinement of the
                                returned pairs (default 1 for 32-bit)      */
    int profile;             /* 1: time every kernel class with CUDA events
                                (fills trlx_stats.kernel_*)                */
} trlx_options;

void trlx_default_options(trlx_options *opts);

/* trlan()/ztrlan() with explicit options (NULL = defaults). */
void trlx_trlan(trl_matvec op, trl_uo user_ortho, trl_info *info, int nrow,
                int mev, double *eval, double *evec, int lde, int lwrk,
                double *wrk, const trlx_options *opts);
void trlx_ztrlan(ztrl_matvec op, trl_info *info, int nrow, int mev,
                 double *eval, trl_dcomplex *evec, int lde,
                 trl_dcomplex *misc, int nmis, double *dwrk, int ldwrk,
                 const trlx_options *opts);

/* ---------------------------------------------------------------------------
 * Several GPUs, block rows (the reference's parallel model, SRC/trl_comm_mpi.c):
 * every rank owns nloc contiguous rows of every vector (rank r's rows follow
 * rank r-1's) and calls trlan/trlx_trlan with its own nloc and evec rows.
 * The dot products, norms and Gram-Schmidt projections are summed over the
 * ranks of the communicator that trlx_init_info_comm stores in
 * info->mpicomp (the reference keeps its MPI communicator there); the small
 * projected problem is solved on every rank from identical sums, so every
 * rank takes the same decisions.  The operator sees this rank's rows: a
 * user `op` exchanges what it needs itself (as in the reference); the
 * distributed built-in operators below do it for CSR input.
 * ------------------------------------------------------------------------- */
typedef struct trlx_comm trlx_comm;

#define TRLX_SUM 0
#define TRLX_MAX 1
#define TRLX_MIN 2

/* Host-callback communicator: fn must replace buf[0:count] (host memory) by
   its elementwise sum / max / min (TRLX_SUM/MAX/MIN) over all ranks, with
   the same result on every rank, and return 0 (MPI_Allreduce, a gloo
   process group, ...).  Device values are staged through pinned host memory
   around each call; halo exchanges travel as one sum over a board of all
   ranks' messages. */
typedef int (*trlx_allreduce_fn)(double *buf, long long count, int op, void *ctx);
int trlx_comm_create_host(int nranks, int rank, trlx_allreduce_fn fn, void *ctx,
                          trlx_comm **out);

/* NCCL communicator (libnccl.so.2, or $TRLX_NCCL_LIB, loaded at run time;
   -1011 when it cannot be loaded): rank 0 calls trlx_comm_nccl_id, the 128
   bytes reach every rank by any channel, and every rank calls
   trlx_comm_create_nccl with its device current.  Sums are queued on the
   solver's stream; halo exchanges are grouped point-to-point messages. */
int trlx_comm_nccl_id(unsigned char id[128]);
int trlx_comm_create_nccl(int nranks, int rank, const unsigned char id[128],
                          trlx_comm **out);

int trlx_comm_rank(const trlx_comm *comm);
int trlx_comm_size(const trlx_comm *comm);
/* Sum / max / min of host doubles over the ranks. */
int trlx_comm_allreduce(trlx_comm *comm, double *buf, long long count, int op);
/* Destroy after every solve and operator using the communicator. */
void trlx_comm_destroy(trlx_comm *comm);

/* trl_init_info for this rank's nloc rows, then ntot = sum of nloc over the
   ranks, my_pe / npes from the communicator and info->mpicomp = comm
   (reference trl_init_info, SRC/trl_comm_mpi.c).  maxmv <= 0 takes the
   reference default from the global ntot.  Returns 0 or an error code. */
int trlx_init_info_comm(trl_info *info, trlx_comm *comm, int nloc, int mxlan,
                        int lohi, int ned, double tol, int restart, int maxmv);

/* This rank's block of a distributed matrix: nloc rows (row_ptr has nloc+1
   entries, starting at 0) whose column indices are GLOBAL.  Rank r's rows
   start after the rows of ranks 0..r-1 (sizes gathered over comm).  Columns
   owned by other ranks become a halo received before every product; the
   local part is stored as CSR or SELL-C-sigma.  Collective: every rank
   calls it. */
int trlx_dist_csr_create(trlx_comm *comm, int nloc, const long long *row_ptr,
                         const int *col_idx, const double *val, int where,
                         trlx_operator **out);
int trlx_dist_sell_create(trlx_comm *comm, int nloc, const long long *row_ptr,
                          const int *col_idx, const double *val, int sigma,
                          int where, trlx_operator **out);
/* Halo entries this rank receives per product (0 for other operators). */
long long trlx_operator_halo(const trlx_operator *op);

/* ---------------------------------------------------------------------------
 * Batched solver: many independent real symmetric problems of uneven size,
 * smallest (lohi < 0) eigenpairs of each, solved by ONE persistent kernel
 * launch.  Each problem is solved by a group of threads of a CTA (the
 * CTA's 1024 or 512 threads, or a half or quarter of them) running the same
 * thick-restart algorithm as trlan() (FP64 basis); problems are taken
 * largest first from a device work queue.  The CTA size, the group size
 * and the operator format (stencil or CSR) per size bucket (n > 32768,
 * 8192 < n <= 32768, n <= 8192) are chosen by an autotuner that times a
 * sample of each bucket.  No counterpart in the reference.
 * ------------------------------------------------------------------------- */
typedef struct trlx_batch trlx_batch;

/* Problems A_p = 5-point Dirichlet Laplacian on an L[p] x L[p] grid
   (4 on the diagonal, -1 couplings) + diag(d_p), d_p = diag[p] (host,
   L[p]^2 doubles, site (i, j) at i + L*j).  L[p] >= 4. */
int trlx_batch_create_stencil5(int nprob, const int *L,
                               const double *const *diag, trlx_batch **out);
/* Optional start vectors (host, n doubles each; NULL entries keep the
   seeded uniform[-1, 1] start). */
int trlx_batch_set_start(trlx_batch *b, const double *const *start);

typedef struct {
    int ned, maxlan, lohi, restart, maxmv; /* as in trl_info; maxlan <= 64 */
    double tol;
    unsigned long long seed; /* start vectors / random restarts          */
    int threads;             /* 0: autotuned per bucket; else the group
                                size: cta_threads, 1/2 or 1/4 of it (-1 if
                                that split's shared memory does not fit for
                                this maxlan)                                */
    int format;              /* -1: autotuned; 0 stencil, 1 CSR           */
    int cta_threads;         /* 0: autotuned; 1024 (64 registers/thread,
                                8-column projection passes) or 512 (up to
                                128 registers, 16-column passes)           */
} trlx_batch_options;

typedef struct {
    int bucket_threads[3];
    int bucket_format[3];
    double tune_seconds;
    int cta_threads;         /* threads per CTA of the launch              */
    int graph_replays;       /* the solve's launch sequence (queue reset +
                                persistent kernel) is a CUDA graph captured
                                once per launch configuration: how many
                                solves have replayed it, this one included */
} trlx_batch_config;

void trlx_batch_default_options(trlx_batch_options *o);
int trlx_batch_autotune(trlx_batch *b, const trlx_batch_options *o,
                        trlx_batch_config *best);
/* eval/res: nprob * ned (res = residual estimates), info: nprob * 4
   (stat, nec, matvec, restarts); any may be NULL. */
int trlx_batch_solve(trlx_batch *b, const trlx_batch_options *o, double *eval,
                     double *res, int *info, trlx_batch_config *used);
/* The ned eigenvectors of problem prob (ned * n doubles, host or device). */
int trlx_batch_eigenvectors(trlx_batch *b, int prob, double *out);
int trlx_batch_size(const trlx_batch *b, int prob);
void trlx_batch_destroy(trlx_batch *b);

/* ---------------------------------------------------------------------------
 * Seed network: a 5-layer convolutional network (3x3 kernels, dilations
 * 1, 2, 4, 8, 1; channels 1 -> 32 -> 32 -> 32 -> 32 -> 16; ReLU after the
 * first four layers; zero "same" padding) mapping a potential V on an
 * H x W grid to 16 vectors whose span approximates the lowest eigenvectors
 * of -Laplacian + V.  The input is (V - min V) / 50 per sample.  BF16
 * activations and weights, FP32 accumulation on the
 * tensor cores, FP32 master weights updated by Adam.  Training minimises
 * per sample  sum_k (1 - |U^T y_k|^2 / |y_k|^2)
 *           + lam * sum_{j != k} (y_j . y_k)^2 / (|y_j|^2 |y_k|^2)
 * against orthonormal reference eigenvectors U.  No counterpart in the
 * reference.  Arrays (host or device): V is B * H * W floats (sample-major,
 * site x + W * y), U and network outputs are B * H * W * 16 floats laid out
 * [sample][site][vector].  Weights are exchanged as, per layer,
 * [tap][c_in][c_out] (9 * 32 * 32 floats, tap = 3 * (dy + 1) + (dx + 1),
 * unused channels zero) followed by 32 biases: trlx_seednet_num_params()
 * floats in total.
 * Returns 0, -1 (bad arguments), -5 (device allocation), -1001 (CUDA).
 * ------------------------------------------------------------------------- */
typedef struct trlx_seednet trlx_seednet;

/* H >= 8, W >= 64 and a multiple of 64; max_batch samples per call. */
int trlx_seednet_create(int H, int W, int max_batch, unsigned long long seed,
                        trlx_seednet **out);
void trlx_seednet_destroy(trlx_seednet *net);
int trlx_seednet_forward(trlx_seednet *net, int B, const float *V, float *out);
/* Loss per sample (loss_out, B floats) and, when grads != NULL, the
   gradient of the batch-mean loss in the weight layout above. */
int trlx_seednet_gradients(trlx_seednet *net, int B, const float *V,
                           const float *U, float lam, float *loss_out,
                           float *grads);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch-mean loss. */
int trlx_seednet_train_step(trlx_seednet *net, int B, const float *V,
                            const float *U, float lam, float lr,
                            float *loss_out);
int trlx_seednet_get_weights(trlx_seednet *net, float *out);
/* Also resets the Adam state. */
int trlx_seednet_set_weights(trlx_seednet *net, const float *in);
int trlx_seednet_num_params(void);

/* Start vector from a predicted subspace Y (nrow x k FP32, [site][vector],
   host or device, 1 <= k <= 32).  project = 1: Rayleigh-Ritz -- Y is
   orthonormalised in FP64 (numerically dependent directions dropped) and
   projected on the built-in operator op (k applications); start (nrow
   doubles, host or device) receives the sum of the Ritz vectors, theta and
   res (k doubles, host, optional) the Ritz values (ascending) and residual
   norms |A x - theta x| (-1 for dropped directions).  project = 0: start =
   sum of the normalised columns of Y, no operator application (theta 0,
   res -1).  Pass start to trlan() with trl_set_iguess(info, 0, 1, 0, NULL)
   and start in the first column of evec.  Returns the number of vectors
   used (>= 1) or -1 (bad arguments), -5 (device allocation), -234 (Y
   numerically zero), -1001 (CUDA).  No counterpart in the reference. */
int trlx_seed_start(void *op, int nrow, int k, const float *Y, int project,
                    double *start, double *theta, double *res);

/* Statistics of the last solve issued from the calling thread. */
typedef struct {
    double seconds_total;     /* wall time of the solve                    */
    double seconds_op;        /* device time in the operator               */
    double seconds_orth;      /* device time in Gram-Schmidt               */
    double seconds_restart;   /* restart (host small dense + V*Y)          */
    double basis_bytes;       /* algorithmic bytes moved by Gram-Schmidt
                                 and restart kernels                        */
    double op_bytes;          /* algorithmic bytes of built-in operators   */
    long long kernel_launches;/* kernels launched by the engine            */
    int cgs_passes;           /* Gram-Schmidt passes (== info->north)      */
    int host_syncs;           /* host/device synchronisations              */
    double max_true_residual; /* refinement: max ||Az - theta z||, or -1   */
    /* Per kernel class (TRLX_K_*), filled when trlx_options.profile is set:
       device seconds (CUDA events on the solver's stream), algorithmic
       bytes moved, and launches. */
    double kernel_seconds[8];
    double kernel_bytes[8];
    long long kernel_count[8];
    double seconds_setup;     /* workspace acquisition and initialisation  */
    long long speculative_steps;     /* Lanczos steps issued ahead of the
                                        host decisions and accepted         */
    long long speculative_discarded; /* speculative steps rerun (their
                                        operator applications are not in
                                        info->matvec)                       */
} trlx_stats;

#define TRLX_K_SPMV 0      /* built-in operator (+ fused alpha)          */
#define TRLX_K_PROJECT 1   /* Gram-Schmidt projection h = V^H r          */
#define TRLX_K_UPDATE 2    /* Gram-Schmidt update r - V h                */
#define TRLX_K_NORMALIZE 3 /* scaling / storing the new basis vector     */
#define TRLX_K_RITZ 4      /* restart recombination V Y                  */
#define TRLX_K_DOT 5       /* standalone dot products                    */
#define TRLX_K_OTHER 6

void trlx_get_last_stats(trlx_stats *stats);

/* Device workspace (basis pool, reduction scratch) is kept per thread
   between solves and reused when large enough; this frees it, together with
   the pinned host buffers of the staged host<->device copies and the device
   memory that destroyed operators left in the library's allocation pool
   (trlx_operator_destroy keeps it there for the next operator). */
void trlx_release_workspace(void);

/* Version string of the library. */
const char *trlx_version(void);

/* ---------------------------------------------------------------------------
 * Host-side building blocks, exported for inspection and CPU tests.  They
 * are the engine's own FP64 routines for the projected problem.
 * ------------------------------------------------------------------------- */
/* Ritz values (ascending) and residual estimates of the tridiagonal
   (alpha, beta) with the first `locked` values treated as locked. */
int trlx_host_get_eval(int nd, int locked, const double *alpha,
                       const double *beta, double *lambda, double *res);
/* Eigenvalues (ascending) and last eigenvector components of a symmetric
   tridiagonal matrix (diag d[n], off-diagonal e[n-1]). */
int trlx_host_tridiag_eig_last(int n, const double *d, const double *e,
                               double *lambda, double *zlast);
/* Arrow matrix -> tridiagonal with rotation (nd x nd, column-major). */
int trlx_host_arrow_to_tridiag(int nd, const double *alpha,
                               const double *beta, double *rot,
                               double *alfrot, double *betrot);
/* Symmetric eigen-decomposition in place (A n x n column-major). */
int trlx_host_sym_eig(int n, double *A, int lda, double *w);
int trlx_host_herm_eig(int n, const trl_dcomplex *A, int lda, double *w,
                       trl_dcomplex *Z, int ldz);
/* Restart decision: kept pairs (and info->klan for schemes 7/8). */
void trlx_host_shuffle_eig(int nd, int mnd, double *lambda, double *res,
                           trl_info *info, int *kept, int locked);
void trlx_host_convergence_test(int nd, double *lambda, double *res,
                                trl_info *info, double *wrk);
void trlx_host_sort_eig(int nd, int lohi, int nec, double ref,
                        double *lambda, double *res);
void trlx_host_set_locking(int jnd, int nlam, double *lambda, double *res,
                           double *yy, double anrm, int *locked);
/* Paired shell sort, ascending in key. */
void trlx_host_sort2(int n, double *key, double *other);

#ifdef __cplusplus
}
#endif

#endif /* TRLAN_B200_TRLX_H */

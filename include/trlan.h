/*
 * trlan.h -- public C interface of the B200 thick-restart Lanczos engine.
 *
 * Drop-in replacement for nuTRLan's public header (reference INC/trlan.h).
 * The trl_info structure below keeps the reference's field names, order and
 * types so that it has the same size (800 bytes on LP64) and the same field
 * offsets: programs and bindings compiled against the reference header link
 * against libtrlan_b200.so unchanged.  Unlike the reference header this one
 * includes <stdio.h> itself (trl_info holds FILE pointers).
 *
 * Device residency: when `evec` passed to trlan() is CUDA device memory (or a
 * built-in device operator from trlx.h is used), the Lanczos basis stays in
 * GPU memory for the whole solve and `op` receives device pointers.  With a
 * host `evec` and a user host `op`, the solver stages each matrix-vector
 * product through pinned host buffers; everything else still runs on the GPU.
 */
#ifndef TRLAN_B200_TRLAN_H
#define TRLAN_B200_TRLAN_H

#include <stdio.h> /* FILE */
#include <time.h>  /* clock_t */

#ifdef __cplusplus
extern "C" {
#endif

#ifdef TRL_FORTRAN_COMPATIBLE
/* Fortran-callable operator: every argument by reference, no mvparam. */
typedef void (*trl_matvec)(int *pnrow, int *pncol, double *x, int *pldx,
                           double *y, int *pldy);
typedef void (*trl_uo)(int *pnrow, double *x, double *y);
#else
/*
 * y(:,j) = A * x(:,j) for j < ncol.  Column j of x starts at x + ldx*j, of y
 * at y + ldy*j.  The solver always calls it with ncol == 1.  `mvparam` is
 * info->mvparam, passed through untouched (reference INC/trlan.h:67-69).
 */
typedef void (*trl_matvec)(const int nrow, const int ncol, const double *x,
                           const int ldx, double *y, const int ldy,
                           void *mvparam);
/*
 * Optional extra orthogonalisation of v (length nrow) applied after each
 * Gram-Schmidt pass; when normDiff is not NULL it receives ||v_new - v_old||.
 */
typedef void (*trl_uo)(const int nrow, double *v, double *normDiff);
#endif

/*
 * Problem specification, progress counters and timers of one solve.
 * Field-for-field the same layout as the reference's struct (reference
 * INC/trlan.h:77-245); see the comments there for the historical meaning of
 * the restart-scheme bookkeeping fields.
 */
typedef struct strct_trl_info {
    int stat;        /* 0 on success, negative error code otherwise          */

    int lohi;        /* <0 smallest, >0 largest, 0 whichever converge first;
                        -2/-3/-4: closest to / above / below info->ref        */
    int ned;         /* number of eigenpairs wanted                          */
    int nec;         /* number of eigenpairs converged (locked on entry)     */
    double tol;      /* residual tolerance relative to ||A|| estimate        */

    void *mpicomp;   /* communicator handle (unused by the serial engine)    */
    int maxlan;      /* maximum basis size                                   */
    int klan;        /* current basis size limit (set by restart schemes)    */
    int maxmv;       /* maximum number of matrix-vector products             */

    int restart;     /* thick-restart scheme 1..8 (<=0 -> fixed scheme)      */
    int locked;      /* number of locked Ritz pairs                          */
    int guess;       /* <=0: ones vector (+random perturbation if <0);
                        1: user vector in column nec of evec;
                        >1: resume from checkpoint files                     */

    int matvec;      /* matrix-vector products performed                     */
    int nloop;       /* restarts performed                                   */
    int north;       /* full Gram-Schmidt passes performed                   */
    int nrand;       /* random vectors injected after breakdown              */
    int flop;        /* flop counters (excluding matvec)                     */
    int flop_h;
    int flop_r;
    double rflp;
    double rflp_h;
    double rflp_r;

    clock_t clk_rate; /* timer ticks per second                              */
    clock_t clk_max;
    clock_t clk_tot;
    clock_t clk_op;
    clock_t clk_orth;
    clock_t clk_res;
    double tick_t;   /* seconds: total, operator, orthogonalisation, restart */
    double tick_o;
    double tick_h;
    double tick_r;
    int clk_in;
    int wrds_in;
    int clk_out;
    int wrds_out;

    double anrm;     /* ||A|| estimate: largest |Ritz value| seen            */

    int my_pe;
    int npes;
    int nloc;        /* local problem size                                   */
    int ntot;        /* global problem size                                  */

    int verbose;
    double crat;     /* convergence rate of the current target              */
    double trgt;     /* Ritz value expected to converge next                 */
    double tres;     /* its residual norm                                    */
    int tmv;         /* matvec count when trgt/tres were recorded            */
    double avgm;

    double cfac;
    double ptres;
    double predicted_crate;
    double mgap;
    double mgamma, gamma0;
    double old_target;
    int target_id;
    int old_locked;
    int k1, k2, k;
    double rfact;

    double ref;      /* reference point for lohi = -2/-3/-4                  */

    int log_io;
    FILE *log_fp;
    char log_file[128];

    int cpflag, cpio; /* checkpoint roughly cpflag times during the solve    */
    FILE *cpt_fp;
    char cpfile[128], oldcpf[128];

    void *mvparam;   /* passed verbatim to the operator                      */
} trl_info;

/* Real symmetric solve (reference INC/trlan.h:308). */
void trlan(trl_matvec op, trl_uo user_ortho, trl_info *info, int nrow,
           int mev, double *eval, double *evec, int lde, int lwrk,
           double *wrk);

/* Residual / Rayleigh-quotient check of computed pairs (INC/trlan.h:346). */
void trl_check_ritz(trl_matvec op, trl_info *info, int nrow, int ncol,
                    double *rvec, int ldrvec, double *alpha, int *check,
                    double *beta, double *eval, double *wrk, int lwrk);

/* Initialise info; must precede every other call (INC/trlan.h:395). */
void trl_init_info(trl_info *info, int nrow, int mxlan, int lohi, int ned,
                   double tol, int restart, int maxmv, void *mpicomp);

/* Minimum basis-size factor for restart schemes 7/8 (INC/trlan.h:411). */
void trl_set_restart(trl_info *info, double rfact);

/* Verbosity and log-file prefix (INC/trlan.h:434). */
void trl_set_debug(trl_info *info, int msglvl, char *filename);

/* Checkpoint roughly cpflag times to files prefixed by file (:452). */
void trl_set_checkpoint(trl_info *info, int cpflag, char *file);

/* Converged count on entry and initial-guess option (INC/trlan.h:484). */
void trl_set_iguess(trl_info *info, int nec, int iguess, int ncps,
                    char *cpf);

/* Human-readable summary of a finished solve (INC/trlan.h:503). */
void trl_print_info(trl_info *info, int mvflop);

/* One-line-per-item summary to iou, stdout when NULL (INC/trlan.h:517). */
void trl_terse_info(trl_info *info, FILE *iou);

/* Rayleigh-Ritz projection of an approximate invariant subspace
   (INC/trlan.h:558). */
void trl_ritz_projection(trl_matvec op, trl_info *info, int mev,
                         double *evec, int lde, double *eres, double *wrk,
                         int lwrk, double *base);

/* Rayleigh quotients and residual norms of given vectors (:592). */
void trl_rayleigh_quotients(trl_matvec op, trl_info *info, int ncol,
                            double *evec, int lde, double *eres,
                            double *base);

#ifdef __cplusplus
}
#endif

#endif /* TRLAN_B200_TRLAN_H */

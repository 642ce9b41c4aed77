/*
 * ztrlan.h -- complex Hermitian interface of the B200 Lanczos engine.
 *
 * Drop-in replacement for nuTRLan's INC/ztrlan.h.  The reference header
 * relies on trl_dcomplex coming from its internal trl_map.h; this header
 * defines the identical {double r, i;} layout itself (guarded, so including
 * both is harmless).  Alpha/beta of the Hermitian tridiagonal are real, so
 * eigenvalues and residual norms are plain doubles.
 */
#ifndef TRLAN_B200_ZTRLAN_H
#define TRLAN_B200_ZTRLAN_H

#include "trlan.h"

#ifdef __cplusplus
extern "C" {
#endif

#ifndef TRL_DCOMPLEX_DEFINED
#define TRL_DCOMPLEX_DEFINED
typedef struct {
    double r, i;
} trl_dcomplex;
#endif

#ifdef TRL_FORTRAN_COMPATIBLE
typedef void (*ztrl_matvec)(int *pnrow, int *pncol, trl_dcomplex *x,
                            int *pldx, trl_dcomplex *y, int *pldy);
#else
/* y(:,j) = A * x(:,j); same conventions as trl_matvec. */
typedef void (*ztrl_matvec)(const int nrow, const int ncol,
                            const trl_dcomplex *x, const int ldx,
                            trl_dcomplex *y, const int ldy, void *mvparam);
#endif

/*
 * Complex Hermitian solve (reference INC/ztrlan.h:140).  `misc`/`dwrk` are
 * accepted for source compatibility; the engine keeps its workspaces on the
 * device and uses misc[0:nec].r for the residual norms on exit when nmis
 * allows it, like the reference.
 */
void ztrlan(ztrl_matvec op, trl_info *info, int nrow, int mev, double *eval,
            trl_dcomplex *evec, int lde, trl_dcomplex *misc, int nmis,
            double *dwrk, int ldwrk);

/* Residual check of complex Ritz pairs (reference INC/ztrlan.h:174). */
void ztrl_check_ritz(ztrl_matvec op, trl_info *info, int nrow, int ncol,
                     trl_dcomplex *rvec, int ldrvec, double *alpha,
                     int *check, double *beta, double *eval,
                     trl_dcomplex *wrk, int lwrk);

#ifdef __cplusplus
}
#endif

#endif /* TRLAN_B200_ZTRLAN_H */

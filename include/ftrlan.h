/*
 * ftrlan.h -- Fortran-callable entry points of the library: the reference's
 * Fortran interface (SRC/ftrlan.c, INC/ftrlan.h) in the form a Fortran
 * compiler actually calls -- trailing underscore, every argument by
 * reference, CHARACTER arguments blank-padded with their lengths appended
 * after the other arguments (size_t, as gfortran passes them), and the
 * operator in the reference's Fortran-compatible form (TRL_FORTRAN_COMPATIBLE,
 * INC/trlan.h:9-71): op(nrow, ncol, xin, ldx, yout, ldy), all by reference.
 * The trl_info argument is the same 800-byte structure (an opaque array on
 * the Fortran side).  The reference's own shim passes scalars by value and
 * names an undefined variable; this one follows the Fortran convention.
 */
#ifndef TRLAN_B200_FTRLAN_H
#define TRLAN_B200_FTRLAN_H

#include <stddef.h>

#include "trlan.h"
#include "ztrlan.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void (*trl_fmatvec)(int *nrow, int *ncol, double *xin, int *ldx,
                            double *yout, int *ldy);
typedef void (*ztrl_fmatvec)(int *nrow, int *ncol, trl_dcomplex *xin,
                             int *ldx, trl_dcomplex *yout, int *ldy);

/* trlan / ztrlan (SRC/ftrlan.c:9, :18). */
void trlan_(trl_fmatvec op, trl_info *info, int *nrow, int *mev, double *eval,
            double *evec, int *lde, int *lwrk, double *wrk);
void ztrlan_(ztrl_fmatvec op, trl_info *info, int *nrow, int *mev,
             double *eval, trl_dcomplex *evec, int *lde, trl_dcomplex *misc,
             int *nmis, double *dwrk, int *ldwrk);
/* Setters (SRC/ftrlan.c:27-55). */
void trl_init_info_(trl_info *info, int *nrow, int *mxlan, int *lohi,
                    int *ned, double *tol, int *restart, int *maxmv);
void trl_set_restart_(trl_info *info, double *rfact);
void trl_set_debug_(trl_info *info, int *msglvl, char *filename,
                    size_t filename_len);
void trl_set_iguess_(trl_info *info, int *nec, int *iguess, int *nopts,
                     char *cpf, size_t cpf_len);
void trl_set_checkpoint_(trl_info *info, int *cpflag, char *file,
                         size_t file_len);
void trl_print_info_(trl_info *info, int *mvflop);

#ifdef __cplusplus
}
#endif

#endif /* TRLAN_B200_FTRLAN_H */

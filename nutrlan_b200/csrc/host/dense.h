// Host entry points of the small dense FP64 routines of the thick-restart
// Lanczos engine (implementations shared with the device-side batched solver
// live in dense_core.h and restart_core.h).
//
// Everything here operates on the projected problem (size <= maxlan), never
// on length-n vectors, so it stays on the host in FP64.  The algorithms are
// textbook ones written for this engine:
//   * Householder tridiagonalisation that never touches the last coordinate
//     (the role of LAPACK dsytrd('U')+dorgtr in the reference's trl_tridiag,
//     reference SRC/trlcore.c:1978-2074),
//   * implicit QL with Wilkinson shifts (the published tql2/tqli method),
//     tracking either the full eigenvector matrix or only its last row
//     (the role of dstqrb_, reference SRC/dstqrb.c:22, and of dsyev/dstein),
//   * the gap-halving shell sorts whose tie order the restart logic relies on
//     (reference SRC/dsort2.c).
#pragma once

#include <complex>
#include <vector>

struct strct_trl_info;

namespace trlb {

// ---- paired shell sorts (gap n/2, halving), reference SRC/dsort2.c ------
void sort2(int n, double *key, double *other);                 // key ascending
void sort2_abs(int n, double *key, double *other);             // |key| ascending
void sort2_near(int n, double s, double *key, double *other);  // |key-s| ascending
void sort2_above(int n, double s, double *key, double *other); // values above s first
void sort2_below(int n, double s, double *key, double *other); // values below s first

// ---- tridiagonal / symmetric eigen-solvers --------------------------------
// A (n x n, column-major, lda) symmetric -> A = Q T Q^T with Q e_{n-1} = e_{n-1}.
// d[0..n) = diag(T), e[0..n-1) = superdiagonal.  If want_q, Q overwrites A.
void tridiag_upper(int n, double *A, int lda, double *d, double *e, bool want_q);

// Implicit QL on (d, e).  Z (zrows x n, column-major, ldz) receives the
// rotations: pass Z = Q to get eigenvectors of Q T Q^T.  Returns 0 or the
// (1-based) index of the eigenvalue that failed to converge.  Eigenvalues are
// NOT sorted.
int tql_implicit(int n, double *d, double *e, double *Z, int ldz, int zrows);

// Eigenvalues (ascending) and last components of the normalised eigenvectors
// of the symmetric tridiagonal matrix (d, e): the quantities dstqrb_ returns.
int tridiag_eig_last(int n, const double *d, const double *e, double *lambda,
                     double *zlast);

// Full symmetric eigen-decomposition: eigenvalues ascending into w, vectors
// into A (columns).  Returns 0 on success.
int sym_eig(int n, double *A, int lda, double *w);

// Hermitian eigen-decomposition (cyclic Jacobi; n small): eigenvalues
// ascending into w, unitary eigenvectors into Z (columns).  Returns 0, or 1
// if the sweeps did not converge.
int herm_eig(int n, const std::complex<double> *A, int lda, double *w, std::complex<double> *Z, int ldz);

// ---- pieces of the reference's Lanczos driver ----------------------------
// trl_tridiag: arrow matrix (alpha on diag, beta[0..nd-1) in the last
// row/column) -> tridiagonal (alfrot, betrot) with rotation rot (nd x nd).
int arrow_to_tridiag(int nd, const double *alpha, const double *beta,
                     double *rot, double *alfrot, double *betrot);

// trl_get_eval: Ritz values + residual estimates |beta_last * z_last|.
int get_eval(int nd, int locked, const double *alpha, const double *beta,
             double *lambda, double *res);

// trl_get_tvec: eigenvectors of the tridiagonal (alpha, beta) for the given
// Ritz values lambda[0..nlam), then rot (nrot x nrot) applied to rows
// irot..irot+nrot of each vector.  yy is nd x nlam.
int get_tvec(int nd, const double *alpha, const double *beta, int irot,
             int nrot, const double *rot, int nlam, const double *lambda,
             double *yy);

// trl_get_tvec_a: eigenvectors of the arrow+tridiagonal projection
// (first `kept` rows form the arrow) by a full symmetric solve; alpha is
// overwritten with the eigenvalues matched to lambda[0..nlam).
int get_tvec_a(int nd, int kept, double *alpha, const double *beta,
               int nlam, const double *lambda, double *yy);

// trl_set_locking: move pairs with negligible residual to the front.
void set_locking(int jnd, int nlam, double *lambda, double *res, double *yy,
                 double anrm, int *locked);

// trl_convergence_test and trl_sort_eig.
void convergence_test(int nd, double *lambda, double *res,
                      strct_trl_info *info, double *wrk);
void sort_eig(int nd, int lohi, int nec, double ref, double *lambda,
              double *res);

// trl_shuffle_eig: restart-scheme dispatch; decides kept (and klan).
void shuffle_eig(int nd, int mnd, double *lambda, double *res,
                 strct_trl_info *info, int *kept, int locked);

}  // namespace trlb

// Host entry points of the small dense routines: thin wrappers that give the
// shared __host__ __device__ implementations (dense_core.h, restart_core.h)
// a per-thread workspace.
#include "dense.h"

#include <vector>

#include "dense_core.h"
#include "restart_core.h"

namespace trlb {

namespace {

double *workspace(int nd) {
    static thread_local std::vector<double> ws;
    const size_t need = core::dense_ws_doubles(nd < 1 ? 1 : nd);
    if (ws.size() < need) ws.resize(need);
    return ws.data();
}

}  // namespace

void sort2(int n, double *key, double *other) { core::sort2(n, key, other); }
void sort2_abs(int n, double *key, double *other) { core::sort2_abs(n, key, other); }
void sort2_near(int n, double s, double *key, double *other) { core::sort2_near(n, s, key, other); }
void sort2_above(int n, double s, double *key, double *other) { core::sort2_above(n, s, key, other); }
void sort2_below(int n, double s, double *key, double *other) { core::sort2_below(n, s, key, other); }

void tridiag_upper(int n, double *A, int lda, double *d, double *e, bool want_q) {
    core::tridiag_upper(n, A, lda, d, e, want_q, workspace(n));
}
int tql_implicit(int n, double *d, double *e, double *Z, int ldz, int zrows) {
    return core::tql_implicit(n, d, e, Z, ldz, zrows);
}
int tridiag_eig_last(int n, const double *d, const double *e, double *lambda, double *zlast) {
    return core::tridiag_eig_last(n, d, e, lambda, zlast, workspace(n));
}
int sym_eig(int n, double *A, int lda, double *w) { return core::sym_eig(n, A, lda, w, workspace(n)); }
int arrow_to_tridiag(int nd, const double *alpha, const double *beta, double *rot, double *alfrot,
                     double *betrot) {
    return core::arrow_to_tridiag(nd, alpha, beta, rot, alfrot, betrot, workspace(nd));
}
int get_eval(int nd, int locked, const double *alpha, const double *beta, double *lambda, double *res) {
    return core::get_eval(nd, locked, alpha, beta, lambda, res, workspace(nd));
}
int get_tvec(int nd, const double *alpha, const double *beta, int irot, int nrot, const double *rot, int nlam,
             const double *lambda, double *yy) {
    return core::get_tvec(nd, alpha, beta, irot, nrot, rot, nlam, lambda, yy, workspace(nd));
}
int get_tvec_a(int nd, int kept, double *alpha, const double *beta, int nlam, const double *lambda, double *yy) {
    return core::get_tvec_a(nd, kept, alpha, beta, nlam, lambda, yy, workspace(nd));
}
void set_locking(int jnd, int nlam, double *lambda, double *res, double *yy, double anrm, int *locked) {
    core::set_locking(jnd, nlam, lambda, res, yy, anrm, locked);
}
void convergence_test(int nd, double *lambda, double *res, trl_info *info, double *wrk) {
    core::convergence_test(nd, lambda, res, info, wrk);
}
void sort_eig(int nd, int lohi, int nec, double ref, double *lambda, double *res) {
    core::sort_eig(nd, lohi, nec, ref, lambda, res);
}
void shuffle_eig(int nd, int mnd, double *lambda, double *res, trl_info *info, int *kept, int locked) {
    core::shuffle_eig(nd, mnd, lambda, res, info, kept, locked);
}

}  // namespace trlb

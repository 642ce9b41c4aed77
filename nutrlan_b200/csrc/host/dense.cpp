// Host entry points of the small dense routines: thin wrappers that give the
// shared __host__ __device__ implementations (dense_core.h, restart_core.h)
// a per-thread workspace.
#include "dense.h"

#include <complex>
#include <cmath>
#include <vector>

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

// Cyclic Jacobi for a small Hermitian matrix.  Each rotation first turns
// a_pq real with the phase e = a_pq / |a_pq| on column q, then applies the
// real rotation that annihilates it (t = sgn(tau) / (|tau| + sqrt(1 + tau^2)),
// tau = (a_qq - a_pp) / (2 |a_pq|)); U = diag(1, conj(e)) * [[c, s], [-s, c]]
// in the (p, q) plane, A <- U^H A U, Z <- Z U.  Sweeps stop when the
// off-diagonal Frobenius norm is below 1e-15 of the matrix norm.
int herm_eig(int n, const std::complex<double> *A, int lda, double *w, std::complex<double> *Z, int ldz) {
    using cd = std::complex<double>;
    if (n <= 0) return 0;
    std::vector<cd> B((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) B[i + (size_t)j * n] = A[i + (size_t)j * lda];
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) Z[i + (size_t)j * ldz] = cd(i == j ? 1.0 : 0.0, 0.0);
        B[j + (size_t)j * n] = cd(B[j + (size_t)j * n].real(), 0.0);
    }
    double tot = 0.0;
    for (const cd &v : B) tot += std::norm(v);
    int sweep = 0;
    for (; sweep < 64; ++sweep) {
        double off = 0.0;
        for (int q = 0; q < n; ++q)
            for (int p = 0; p < q; ++p) off += std::norm(B[p + (size_t)q * n]);
        if (off <= 1e-30 * tot || off == 0.0) break;
        for (int q = 1; q < n; ++q)
            for (int p = 0; p < q; ++p) {
                const cd apq = B[p + (size_t)q * n];
                const double g = std::abs(apq);
                if (g == 0.0) continue;
                const cd e = apq / g;
                const double app = B[p + (size_t)p * n].real(), aqq = B[q + (size_t)q * n].real();
                const double tau = (aqq - app) / (2.0 * g);
                const double t = (tau >= 0.0 ? 1.0 : -1.0) / (std::fabs(tau) + std::sqrt(1.0 + tau * tau));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = t * c;
                const cd se = s * std::conj(e), sec = s * e;
                for (int i = 0; i < n; ++i) {  // columns: B <- B U
                    const cd bp = B[i + (size_t)p * n], bq = B[i + (size_t)q * n];
                    B[i + (size_t)p * n] = c * bp - se * bq;
                    B[i + (size_t)q * n] = s * bp + c * std::conj(e) * bq;
                }
                for (int j = 0; j < n; ++j) {  // rows: B <- U^H B
                    const cd bp = B[p + (size_t)j * n], bq = B[q + (size_t)j * n];
                    B[p + (size_t)j * n] = c * bp - sec * bq;
                    B[q + (size_t)j * n] = s * bp + c * e * bq;
                }
                B[p + (size_t)q * n] = B[q + (size_t)p * n] = cd(0.0, 0.0);
                B[p + (size_t)p * n] = cd(B[p + (size_t)p * n].real(), 0.0);
                B[q + (size_t)q * n] = cd(B[q + (size_t)q * n].real(), 0.0);
                for (int i = 0; i < n; ++i) {
                    const cd zp = Z[i + (size_t)p * ldz], zq = Z[i + (size_t)q * ldz];
                    Z[i + (size_t)p * ldz] = c * zp - se * zq;
                    Z[i + (size_t)q * ldz] = s * zp + c * std::conj(e) * zq;
                }
            }
    }
    // Ascending eigenvalues with their vectors (stable selection sort).
    for (int i = 0; i < n; ++i) w[i] = B[i + (size_t)i * n].real();
    for (int i = 0; i < n; ++i) {
        int k = i;
        for (int j = i + 1; j < n; ++j)
            if (w[j] < w[k]) k = j;
        if (k != i) {
            std::swap(w[i], w[k]);
            for (int r = 0; r < n; ++r) std::swap(Z[r + (size_t)i * ldz], Z[r + (size_t)k * ldz]);
        }
    }
    return sweep >= 64 ? 1 : 0;
}
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

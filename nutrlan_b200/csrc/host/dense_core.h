// Small dense FP64 routines of the thick-restart Lanczos driver, written once
// for the host engine and the device-side batched solver (every function is
// __host__ __device__ when compiled by nvcc and uses caller-provided
// workspace instead of allocating).
//
// Map to the reference (roles, not code):
//   * tridiag_upper: Householder tridiagonalisation that never touches the
//     last coordinate (dsytrd('U') + dorgtr in trl_tridiag,
//     SRC/trlcore.c:1978-2074);
//   * tql_implicit / tridiag_eig_last: implicit QL with Wilkinson shifts
//     (the published tql2/tqli method) tracking the full eigenvector matrix or
//     only its last row (dstqrb_, SRC/dstqrb.c:22);
//   * get_eval, get_tvec, get_tvec_a, set_locking, convergence_test,
//     sort_eig: trl_get_eval, trl_get_tvec (dstein), trl_get_tvec_a (dsyev),
//     trl_set_locking, trl_convergence_test, trl_sort_eig
//     (SRC/trlcore.c:2077-2758);
//   * the gap-halving shell sorts of SRC/dsort2.c (tie order matters).
#pragma once

#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdlib>

#include "../../../include/trlan.h"

#if defined(__CUDACC__)
#define TRLB_HD __host__ __device__
#else
#define TRLB_HD
#endif

namespace trlb {
namespace core {

template <class X>
TRLB_HD inline X hmax(X a, X b) {
    return a > b ? a : b;
}
template <class X>
TRLB_HD inline X hmin(X a, X b) {
    return a < b ? a : b;
}
template <class X>
TRLB_HD inline void hswap(X &a, X &b) {
    X t = a;
    a = b;
    b = t;
}
TRLB_HD inline void hcopy(double *dst, const double *src, size_t n) {
    for (size_t i = 0; i < n; ++i) dst[i] = src[i];
}
TRLB_HD inline void hzero(double *p, size_t n) {
    for (size_t i = 0; i < n; ++i) p[i] = 0.0;
}

// Doubles of workspace any routine below needs for a problem of size nd.
TRLB_HD inline size_t dense_ws_doubles(int nd) { return 2 * (size_t)nd * nd + 8 * (size_t)nd + 16; }


// ---------------------------------------------------------------------------
// Paired shell sorts.  The gap sequence (n/2, n/4, ..., 1) and the strict
// ">" comparison are kept from the reference (SRC/dsort2.c:11-323) because
// the restart logic depends on where equal keys end up.
// ---------------------------------------------------------------------------
template <class Greater>
TRLB_HD inline void shell_pair(int n, double *key, double *other, Greater greater) {
    for (int gap = n / 2; gap > 0; gap /= 2) {
        for (int i = gap; i < n; ++i) {
            for (int j = i - gap; j >= 0 && greater(key[j], key[j + gap]); j -= gap) {
                hswap(key[j], key[j + gap]);
                hswap(other[j], other[j + gap]);
            }
        }
    }
}

TRLB_HD inline void sort2(int n, double *key, double *other) {
    shell_pair(n, key, other, [](double a, double b) { return a > b; });
}

TRLB_HD inline void sort2_abs(int n, double *key, double *other) {
    shell_pair(n, key, other, [](double a, double b) { return fabs(a) > fabs(b); });
}

TRLB_HD inline void sort2_near(int n, double s, double *key, double *other) {
    shell_pair(n, key, other,
               [s](double a, double b) { return fabs(a - s) > fabs(b - s); });
}

// Order: values whose magnitude lies above s by increasing distance, then
// the rest (reference dsort2su_, SRC/dsort2.c:179).
TRLB_HD inline void sort2_above(int n, double s, double *key, double *other) {
    if (n <= 0) return;
    double big = 0.0;
    for (int i = 0; i < n; ++i) big = hmax(big, fabs(key[i]));
    shell_pair(n, key, other, [s, big](double a, double b) {
        double va = fabs(a), vb = fabs(b);
        double da = va - s, db = vb - s;
        if (da < 0.0) da = big + va;
        if (db < 0.0) db = big + vb;
        return da > db;
    });
}

// Order: values whose magnitude lies below s by increasing distance, then
// the rest (reference dsort2sd, SRC/dsort2.c:252).
TRLB_HD inline void sort2_below(int n, double s, double *key, double *other) {
    if (n <= 0) return;
    double big = 0.0;
    for (int i = 0; i < n; ++i) big = hmax(big, fabs(key[i]));
    big += 1.0;
    shell_pair(n, key, other, [s, big](double a, double b) {
        double va = fabs(a), vb = fabs(b);
        double da = s - va, db = s - vb;
        if (da < 0.0) da = s + (big - va);
        if (db < 0.0) db = s + (big - vb);
        return da > db;
    });
}

// ---------------------------------------------------------------------------
// Householder tridiagonalisation, bottom-up.  Column k (k = n-1 .. 2) is
// reduced by a reflector acting on indices 0..k-1 only, so index n-1 is never
// mixed: Q e_{n-1} = e_{n-1}.  That is what lets the Lanczos driver read
// residual estimates off the last row of the rotated problem.
// ---------------------------------------------------------------------------
TRLB_HD inline void tridiag_upper(int n, double *A, int lda, double *d, double *e, bool want_q,
                                  double *ws) {
    auto a = [&](int i, int j) -> double & { return A[(size_t)j * lda + i]; };
    if (n <= 0) return;
    // ws: reflectors (n*n), taus (n), p (n), w (n)
    double *vs = ws, *taus = ws + (size_t)n * n, *p = taus + n, *w = p + n;
    hzero(vs, (size_t)n * n);
    hzero(taus, n);
    for (int k = n - 1; k >= 2; --k) {
        // x = A(0:k-1, k); annihilate x(0:k-2) keeping x(k-1).
        double alpha = a(k - 1, k);
        double sigma = 0.0;
        for (int i = 0; i < k - 1; ++i) sigma += a(i, k) * a(i, k);
        double *v = &vs[(size_t)k * n];
        if (sigma == 0.0) {
            taus[k] = 0.0;
            e[k - 1] = alpha;
            continue;
        }
        double mu = sqrt(alpha * alpha + sigma);
        double beta = alpha <= 0.0 ? mu : -mu;
        double tau = (beta - alpha) / beta;
        double scal = 1.0 / (alpha - beta);
        for (int i = 0; i < k - 1; ++i) v[i] = a(i, k) * scal;
        v[k - 1] = 1.0;
        taus[k] = tau;
        e[k - 1] = beta;
        // Two-sided update of the leading k x k block: A <- H A H.
        for (int i = 0; i < k; ++i) {
            double s = 0.0;
            for (int j = 0; j < k; ++j) s += a(i, j) * v[j];
            p[i] = tau * s;
        }
        double pv = 0.0;
        for (int i = 0; i < k; ++i) pv += p[i] * v[i];
        for (int i = 0; i < k; ++i) w[i] = p[i] - 0.5 * tau * pv * v[i];
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < k; ++i) a(i, j) -= v[i] * w[j] + w[i] * v[j];
        // Column/row k now hold (0,..,0,beta).
        for (int i = 0; i < k - 1; ++i) {
            a(i, k) = 0.0;
            a(k, i) = 0.0;
        }
        a(k - 1, k) = beta;
        a(k, k - 1) = beta;
    }
    if (n >= 2) e[0] = a(0, 1);
    for (int i = 0; i < n; ++i) d[i] = a(i, i);
    if (!want_q) return;
    // Q = H_{n-1} ... H_2; build it by applying H_2 first to the identity.
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) a(i, j) = (i == j) ? 1.0 : 0.0;
    for (int k = 2; k <= n - 1; ++k) {
        double tau = taus[k];
        if (tau == 0.0) continue;
        const double *v = &vs[(size_t)k * n];
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += v[i] * a(i, j);
            s *= tau;
            for (int i = 0; i < k; ++i) a(i, j) -= s * v[i];
        }
    }
}

// ---------------------------------------------------------------------------
// Implicit QL with Wilkinson shift on a symmetric tridiagonal matrix.
// e[i] couples rows i and i+1 (e[n-1] is scratch).  Every plane rotation of
// columns (i, i+1) is also applied to the zrows x n matrix Z.
// ---------------------------------------------------------------------------
TRLB_HD inline int tql_implicit(int n, double *d, double *e, double *Z, int ldz, int zrows) {
    if (n <= 1) return 0;
    e[n - 1] = 0.0;
    const int max_sweeps = 60;
    for (int l = 0; l < n; ++l) {
        int sweeps = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) <= DBL_EPSILON * dd) break;
            }
            if (m == l) break;
            if (++sweeps > max_sweeps) return l + 1;
            // Wilkinson shift from the leading 2x2 block.
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = m - 1; i >= l; --i) {
                double f = s * e[i];
                double b = c * e[i];
                r = hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
                if (Z) {
                    double *zi = Z + (size_t)i * ldz;
                    double *zi1 = Z + (size_t)(i + 1) * ldz;
                    for (int k = 0; k < zrows; ++k) {
                        double t = zi1[k];
                        zi1[k] = s * zi[k] + c * t;
                        zi[k] = c * zi[k] - s * t;
                    }
                }
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

TRLB_HD inline int tridiag_eig_last(int n, const double *d, const double *e, double *lambda,
                     double *zlast, double *ws) {
    if (n <= 0) return 0;
    double *dd = ws, *ee = ws + n;  // ws: 2n
    for (int i = 0; i < n; ++i) {
        dd[i] = d[i];
        ee[i] = 0.0;
    }
    for (int i = 0; i + 1 < n; ++i) ee[i] = e[i];
    for (int i = 0; i < n; ++i) zlast[i] = (i == n - 1) ? 1.0 : 0.0;
    // Z is the single row n-1 of the eigenvector matrix: zrows = 1, ldz = 1.
    int err = tql_implicit(n, dd, ee, zlast, 1, 1);
    if (err) return err;
    for (int i = 0; i < n; ++i) lambda[i] = dd[i];
    sort2(n, lambda, zlast);
    return 0;
}

TRLB_HD inline int sym_eig(int n, double *A, int lda, double *w, double *ws) {
    if (n <= 0) return 0;
    double *e = ws;  // ws: n + tridiag_upper's n*n + 3n
    hzero(e, n);
    tridiag_upper(n, A, lda, w, e, true, ws + n);
    int err = tql_implicit(n, w, e, A, lda, n);
    if (err) return err;
    // Selection sort of (w, columns of A) into ascending order.
    for (int i = 0; i < n - 1; ++i) {
        int k = i;
        for (int j = i + 1; j < n; ++j)
            if (w[j] < w[k]) k = j;
        if (k != i) {
            hswap(w[i], w[k]);
            double *ci = A + (size_t)i * lda, *ck = A + (size_t)k * lda;
            for (int r = 0; r < n; ++r) hswap(ci[r], ck[r]);
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Lanczos-driver pieces (reference SRC/trlcore.c:1978-2758).
// ---------------------------------------------------------------------------
TRLB_HD inline int arrow_to_tridiag(int nd, const double *alpha, const double *beta,
                     double *rot, double *alfrot, double *betrot, double *ws) {
    if (nd == 0) return 0;
    if (nd == 1) {
        rot[0] = 1.0;
        alfrot[0] = alpha[0];
        betrot[0] = beta[0];
        return 0;
    }
    hzero(rot, (size_t)nd * nd);
    for (int i = 0; i < nd; ++i) rot[(size_t)i * nd + i] = alpha[i];
    for (int i = 0; i < nd - 1; ++i) {
        rot[(size_t)(nd - 1) * nd + i] = beta[i];
        rot[(size_t)i * nd + (nd - 1)] = beta[i];
    }
    tridiag_upper(nd, rot, nd, alfrot, betrot, true, ws);
    betrot[nd - 1] = beta[nd - 1];
    return 0;
}

TRLB_HD inline int get_eval(int nd, int locked, const double *alpha, const double *beta,
             double *lambda, double *res, double *ws) {
    hcopy(lambda, alpha, nd);
    int m = nd - locked;
    int err = tridiag_eig_last(m, alpha + locked, beta + locked, lambda + locked,
                               res + locked, ws);
    if (err) return -122;
    for (int i = 0; i < locked; ++i) res[i] = 0.0;
    for (int i = locked; i < nd; ++i) res[i] = beta[nd - 1] * fabs(res[i]);
    return 0;
}

// Map each wanted value lam[i] to a distinct computed eigenvalue w[j]: the
// nearest not-yet-used one.  Returns -1 if some value has no computed
// eigenvalue within tol (tol < 0 disables the test).
TRLB_HD inline int match_values(int n, const double *w, int nlam, const double *lam,
                        double tol, int *idx, char *used) {
    for (int j = 0; j < n; ++j) used[j] = 0;
    for (int i = 0; i < nlam; ++i) {
        int best = -1;
        double bd = 0.0;
        for (int j = 0; j < n; ++j) {
            if (used[j]) continue;
            double dd = fabs(w[j] - lam[i]);
            if (best < 0 || dd < bd) {
                best = j;
                bd = dd;
            }
        }
        if (best < 0 || (tol >= 0.0 && bd > tol)) return -1;
        used[best] = 1;
        idx[i] = best;
    }
    return 0;
}

TRLB_HD inline double match_tol(int n, const double *w) {
    double span = hmax(w[n - 1] - w[0], hmax(fabs(w[n - 1]), fabs(w[0])));
    // Looser than the reference's nd*eps*span because the values being
    // matched come from a different (QL) solve of the same matrix.
    return hmax(1e3 * DBL_EPSILON * span * n, DBL_MIN);
}

TRLB_HD inline int get_tvec(int nd, const double *alpha, const double *beta, int irot,
             int nrot, const double *rot, int nlam, const double *lambda,
             double *yy, double *ws) {
    if (nlam <= 0) return 0;
    // ws: d (nd), e (nd), Z (nd*nd), tmp (nd), idx (nlam ints), used (nd chars)
    double *d = ws, *e = ws + nd, *Z = e + nd, *tmp = Z + (size_t)nd * nd;
    int *idx = reinterpret_cast<int *>(tmp + nd);
    char *used = reinterpret_cast<char *>(idx + nlam);
    for (int i = 0; i < nd; ++i) {
        d[i] = alpha[i];
        e[i] = 0.0;
    }
    hzero(Z, (size_t)nd * nd);
    for (int i = 0; i + 1 < nd; ++i) e[i] = beta[i];
    for (int i = 0; i < nd; ++i) Z[(size_t)i * nd + i] = 1.0;
    if (tql_implicit(nd, d, e, Z, nd, nd)) return -132;
    // The wanted values came from the same tridiagonal matrix, so the
    // nearest-unused assignment is exact up to rounding; no tolerance test.
    match_values(nd, d, nlam, lambda, -1.0, idx, used);
    for (int i = 0; i < nlam; ++i)
        hcopy(yy + (size_t)i * nd, Z + (size_t)idx[i] * nd, nd);
    if (nrot > 1) {
        for (int c = 0; c < nlam; ++c) {
            double *col = yy + (size_t)c * nd + irot;
            for (int i = 0; i < nrot; ++i) {
                double s = 0.0;
                for (int k = 0; k < nrot; ++k) s += rot[(size_t)k * nrot + i] * col[k];
                tmp[i] = s;
            }
            hcopy(col, tmp, nrot);
        }
    }
    return 0;
}

TRLB_HD inline int get_tvec_a(int nd, int kept, double *alpha, const double *beta, int nlam,
               const double *lambda, double *yy, double *ws) {
    if (nlam <= 0) return 0;
    // Projection matrix: diagonal alpha, arrow column `kept` holding
    // beta[0..kept), then the tridiagonal couplings beta[kept..nd-1).
    // ws: H (nd*nd), w (nd), wsel (nd), sym_eig (nd*nd + 4 nd), idx, used
    double *H = ws, *w = H + (size_t)nd * nd, *wsel = w + nd, *wse = wsel + nd;
    int *idx = reinterpret_cast<int *>(wse + (size_t)nd * nd + 4 * nd);
    char *used = reinterpret_cast<char *>(idx + nd);
    hzero(H, (size_t)nd * nd);
    for (int i = 0; i < nd; ++i) H[(size_t)i * nd + i] = alpha[i];
    for (int i = 0; i < kept; ++i) {
        H[(size_t)kept * nd + i] = beta[i];
        H[(size_t)i * nd + kept] = beta[i];
    }
    for (int i = kept; i < nd - 1; ++i) {
        H[(size_t)(i + 1) * nd + i] = beta[i];
        H[(size_t)i * nd + i + 1] = beta[i];
    }
    if (sym_eig(nd, H, nd, w, wse)) return -142;
    for (int i = 0; i < nd; ++i) alpha[i] = w[i];
    if (nlam >= nd) {
        hcopy(yy, H, (size_t)nd * nd);
        return 0;
    }
    double tol = hmax(DBL_EPSILON * nd *
                              hmax(w[nd - 1] - w[0], hmax(fabs(w[nd - 1]), fabs(w[0]))),
                          DBL_MIN);
    if (match_values(nd, w, nlam, lambda, hmax(tol, match_tol(nd, w)), idx, used) != 0)
        return -143;
    for (int i = 0; i < nlam; ++i) {
        wsel[i] = w[idx[i]];
        hcopy(yy + (size_t)i * nd, H + (size_t)idx[i] * nd, nd);
    }
    for (int i = 0; i < nlam; ++i) alpha[i] = wsel[i];
    return 0;
}

TRLB_HD inline void set_locking(int jnd, int nlam, double *lambda, double *res, double *yy,
                 double anrm, int *locked) {
    // A pair is lockable when its residual is below eps*|lambda|
    // (eps^2*anrm for lambda == 0); reference SRC/trlcore.c:2676-2758.
    const double eps = DBL_EPSILON;
    auto tiny = [&](int k) {
        double lam = fabs(lambda[k]);
        double thr = lam >= eps ? eps * lam : eps * eps * anrm;
        return fabs(res[k]) <= thr;
    };
    int i = 0, j = nlam - 1;
    bool ti = tiny(i), tj = tiny(j);
    while (i < j) {
        if (ti) {
            res[i] = 0.0;
            ++i;
            ti = (i <= j) ? tiny(i) : false;
        } else {
            if (tj) {
                hswap(lambda[i], lambda[j]);
                res[j] = res[i];
                res[i] = 0.0;
                double *ci = yy + (size_t)i * jnd, *cj = yy + (size_t)j * jnd;
                for (int r = 0; r < jnd; ++r) hswap(ci[r], cj[r]);
                ++i;
                ti = (i <= j) ? tiny(i) : false;
            }
            --j;
            tj = (j > i) ? tiny(j) : false;
        }
    }
    *locked = ti ? i + 1 : i;
}

TRLB_HD inline void convergence_test(int nd, double *lambda, double *res, trl_info *info,
                      double *wrk) {
    // wrk[0..nd) = |res|, wrk[nd..2nd) = lambda, sorted by the lohi order.
    if (info->lohi < -1) sort2_near(nd, info->ref, lambda, res);
    double *wl = wrk + nd, *wr = wrk;
    hcopy(wl, lambda, nd);
    for (int i = 0; i < nd; ++i) wr[i] = fabs(res[i]);
    if (info->lohi == -2)
        sort2_near(nd, info->ref, wl, wr);
    else if (info->lohi == -3)
        sort2_above(nd, info->ref, wl, wr);
    else if (info->lohi == -4)
        sort2_below(nd, info->ref, wl, wr);
    else
        sort2(nd, wl, wr);

    // Convergence rate of the previous target (per matvec).
    if (info->tmv > 0 && info->matvec > info->tmv) {
        int j = 0;
        double bnd = fabs(lambda[0] - info->trgt);
        for (int i = 0; i < nd; ++i) {
            double dd = fabs(lambda[i] - info->trgt);
            if (dd < bnd) {
                bnd = dd;
                j = i;
            }
        }
        if (info->tres > res[j]) {
            bnd = res[j] / info->tres;
            info->crat = bnd > 0.0 ? exp(log(bnd) / (double)(info->matvec - info->tmv)) : 1.0;
            info->cfac = bnd;
        } else {
            info->crat = 1.0;
            info->cfac = bnd;
        }
    }

    info->anrm = hmax(info->anrm, hmax(fabs(wl[1]), fabs(wl[nd - 1])));
    double bnd = DBL_MIN + info->tol * info->anrm;
    int ncl = 0, ncr = nd;
    if (info->lohi <= 0) {
        ncl = nd - 1;
        for (int i = 0; i < nd; ++i) {
            bool conv = wr[i] < bnd;
            bool stop = !conv || (info->lohi == -3 && wl[i] < info->ref) ||
                        (info->lohi == -4 && wl[i] > info->ref);
            if (stop) {
                ncl = i - 1;
                break;
            }
        }
    }
    if (info->lohi >= 0) {
        ncr = 0;
        for (int i = nd - 1; i >= 0; --i) {
            if (!(wr[i] < bnd)) {
                ncr = i + 1;
                break;
            }
        }
    }
    info->tmv = info->matvec;
    info->ptres = info->trgt;
    if (info->lohi < 0) {
        info->nec = ncl + 1;
        info->trgt = wl[hmin(nd - 1, ncl + 1)];
        info->tres = wr[hmin(nd - 1, ncl + 1)];
    } else if (info->lohi > 0) {
        info->nec = nd - ncr;
        info->trgt = wl[hmax(0, ncr - 1)];
        info->tres = wr[hmax(0, ncr - 1)];
    } else {
        if (ncr <= ncl) {
            ncl = nd / 2;
            ncr = ncl + 1;
            info->trgt = wl[(nd + 1) / 2 - 1];
            info->tres = wr[(nd + 1) / 2 - 1];
        } else if (wr[ncl + 1] <= wr[ncr - 1]) {
            info->trgt = wl[ncl + 1];
            info->tres = wr[ncl + 1];
        } else {
            info->trgt = wl[ncr - 1];
            info->tres = wr[ncr - 1];
        }
        info->nec = ncl + nd - ncr + 1;
        for (int i = ncl + 1; i < ncr; ++i)
            if (wr[i] < bnd) info->nec++;
    }
}

TRLB_HD inline void sort_eig(int nd, int lohi, int nec, double ref, double *lambda, double *res) {
    if (lohi == 0) {
        sort2_abs(nd, res, lambda);
        sort2(nec, lambda, res);
    } else if (lohi == -2) {
        sort2_near(nd, ref, lambda, res);
        sort2(nec, lambda, res);
    } else if (lohi == -3) {
        sort2_above(nd, ref, lambda, res);
        sort2(nec, lambda, res);
    } else if (lohi == -4) {
        sort2_below(nd, ref, lambda, res);
        sort2(nec, lambda, res);
    } else {
        sort2(nd, lambda, res);
        if (lohi > 0) {
            for (int i = 0, j = nd - nec; i < nec; ++i, ++j) {
                res[i] = res[j];
                lambda[i] = lambda[j];
            }
        }
    }
}


}  // namespace core
}  // namespace trlb

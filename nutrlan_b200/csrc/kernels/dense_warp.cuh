// Warp-parallel forms of the small dense routines the batched solver runs at
// every restart (host/dense_core.h): implicit QL with eigenvector
// accumulation, Householder tridiagonalisation with Q, the symmetric
// eigen-solve built on them, and trl_get_tvec / trl_get_tvec_a /
// trl_tridiag.  All 32 lanes of one warp call them with their lane index.
// Every element is computed with the same operations in the same order as
// the serial code, so the results are bitwise those of dense_core.h; only
// independent rows or columns are spread over the lanes:
//   * QL: each lane keeps private copies of d and e and runs the (cheap)
//     scalar bulge chase redundantly; the plane rotations are applied to the
//     lane's own rows of Z (rows k = lane, lane + 32, ...);
//   * Householder: p = tau A v by rows, the rank-2 update by columns, Q by
//     columns; the reflector scalars are computed redundantly.
// Shared arrays written by one lane and read by others are separated by
// __syncwarp().
#pragma once

#include <cfloat>

#include "../host/dense_core.h"

namespace trlb {
namespace warp {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxN = 66;  // largest projected problem (maxlan + 2)

__device__ inline int tql_implicit(int n, double *d, double *e, double *Z, int ldz, int zrows, int lane) {
    if (n <= 1) return 0;
    double dl[kMaxN], el[kMaxN];
    for (int i = 0; i < n; ++i) {
        dl[i] = d[i];
        el[i] = e[i];
    }
    el[n - 1] = 0.0;
    const int max_sweeps = 60;
    int err = 0;
    for (int l = 0; l < n && !err; ++l) {
        int sweeps = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                double dd = fabs(dl[m]) + fabs(dl[m + 1]);
                if (fabs(el[m]) <= DBL_EPSILON * dd) break;
            }
            if (m == l) break;
            if (++sweeps > max_sweeps) {
                err = l + 1;
                break;
            }
            double g = (dl[l + 1] - dl[l]) / (2.0 * el[l]);
            double r = hypot(g, 1.0);
            g = dl[m] - dl[l] + el[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            bool deflated = false;
            for (int i = m - 1; i >= l; --i) {
                double f = s * el[i];
                double b = c * el[i];
                r = hypot(f, g);
                el[i + 1] = r;
                if (r == 0.0) {
                    dl[i + 1] -= p;
                    el[m] = 0.0;
                    deflated = true;
                    break;
                }
                s = f / r;
                c = g / r;
                g = dl[i + 1] - p;
                r = (dl[i] - g) * s + 2.0 * c * b;
                p = s * r;
                dl[i + 1] = g + p;
                g = c * r - b;
                if (Z) {
                    double *zi = Z + (size_t)i * ldz;
                    double *zi1 = Z + (size_t)(i + 1) * ldz;
                    for (int k = lane; k < zrows; k += 32) {
                        double t = zi1[k];
                        zi1[k] = s * zi[k] + c * t;
                        zi[k] = c * zi[k] - s * t;
                    }
                }
            }
            if (deflated) continue;
            dl[l] -= p;
            el[l] = g;
            el[m] = 0.0;
        }
    }
    __syncwarp();
    if (lane == 0)
        for (int i = 0; i < n; ++i) {
            d[i] = dl[i];
            e[i] = el[i];
        }
    __syncwarp();
    return err;
}

__device__ inline void tridiag_upper(int n, double *A, int lda, double *d, double *e, bool want_q, double *ws,
                                     int lane) {
    auto a = [&](int i, int j) -> double & { return A[(size_t)j * lda + i]; };
    if (n <= 0) return;
    double *vs = ws, *taus = ws + (size_t)n * n, *p = taus + n, *w = p + n;
    for (size_t q = lane; q < (size_t)n * n; q += 32) vs[q] = 0.0;
    for (int q = lane; q < n; q += 32) taus[q] = 0.0;
    __syncwarp();
    for (int k = n - 1; k >= 2; --k) {
        const double alpha = a(k - 1, k);
        double sigma = 0.0;
        for (int i = 0; i < k - 1; ++i) sigma += a(i, k) * a(i, k);
        double *v = &vs[(size_t)k * n];
        if (sigma == 0.0) {
            __syncwarp();
            if (lane == 0) {
                taus[k] = 0.0;
                e[k - 1] = alpha;
            }
            __syncwarp();
            continue;
        }
        const double mu = sqrt(alpha * alpha + sigma);
        const double beta = alpha <= 0.0 ? mu : -mu;
        const double tau = (beta - alpha) / beta;
        const double scal = 1.0 / (alpha - beta);
        for (int i = lane; i < k - 1; i += 32) v[i] = a(i, k) * scal;
        if (lane == 0) {
            v[k - 1] = 1.0;
            taus[k] = tau;
            e[k - 1] = beta;
        }
        __syncwarp();
        for (int i = lane; i < k; i += 32) {
            double s = 0.0;
            for (int j = 0; j < k; ++j) s += a(i, j) * v[j];
            p[i] = tau * s;
        }
        __syncwarp();
        double pv = 0.0;
        for (int i = 0; i < k; ++i) pv += p[i] * v[i];
        for (int i = lane; i < k; i += 32) w[i] = p[i] - 0.5 * tau * pv * v[i];
        __syncwarp();
        for (int j = lane; j < k; j += 32)
            for (int i = 0; i < k; ++i) a(i, j) -= v[i] * w[j] + w[i] * v[j];
        __syncwarp();
        for (int i = lane; i < k - 1; i += 32) {
            a(i, k) = 0.0;
            a(k, i) = 0.0;
        }
        if (lane == 0) {
            a(k - 1, k) = beta;
            a(k, k - 1) = beta;
        }
        __syncwarp();
    }
    if (lane == 0) {
        if (n >= 2) e[0] = a(0, 1);
        for (int i = 0; i < n; ++i) d[i] = a(i, i);
    }
    __syncwarp();
    if (!want_q) return;
    for (int j = lane; j < n; j += 32)
        for (int i = 0; i < n; ++i) a(i, j) = (i == j) ? 1.0 : 0.0;
    __syncwarp();
    for (int k = 2; k <= n - 1; ++k) {
        const double tau = taus[k];
        if (tau == 0.0) continue;
        const double *v = &vs[(size_t)k * n];
        for (int j = lane; j < n; j += 32) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += v[i] * a(i, j);
            s *= tau;
            for (int i = 0; i < k; ++i) a(i, j) -= s * v[i];
        }
    }
    __syncwarp();
}

__device__ inline int sym_eig(int n, double *A, int lda, double *w, double *ws, int lane) {
    if (n <= 0) return 0;
    double *e = ws;
    for (int i = lane; i < n; i += 32) e[i] = 0.0;
    __syncwarp();
    tridiag_upper(n, A, lda, w, e, true, ws + n, lane);
    const int err = tql_implicit(n, w, e, A, lda, n, lane);
    if (err) return err;
    for (int i = 0; i < n - 1; ++i) {
        int k = i;
        for (int j = i + 1; j < n; ++j)
            if (w[j] < w[k]) k = j;
        __syncwarp();
        if (k != i) {
            double *ci = A + (size_t)i * lda, *ck = A + (size_t)k * lda;
            for (int r = lane; r < n; r += 32) core::hswap(ci[r], ck[r]);
            if (lane == 0) core::hswap(w[i], w[k]);
        }
        __syncwarp();
    }
    return 0;
}

__device__ inline int arrow_to_tridiag(int nd, const double *alpha, const double *beta, double *rot, double *alfrot,
                                       double *betrot, double *ws, int lane) {
    if (nd == 0) return 0;
    if (nd == 1) {
        if (lane == 0) {
            rot[0] = 1.0;
            alfrot[0] = alpha[0];
            betrot[0] = beta[0];
        }
        __syncwarp();
        return 0;
    }
    for (size_t q = lane; q < (size_t)nd * nd; q += 32) rot[q] = 0.0;
    __syncwarp();
    for (int i = lane; i < nd; i += 32) rot[(size_t)i * nd + i] = alpha[i];
    for (int i = lane; i < nd - 1; i += 32) {
        rot[(size_t)(nd - 1) * nd + i] = beta[i];
        rot[(size_t)i * nd + (nd - 1)] = beta[i];
    }
    __syncwarp();
    tridiag_upper(nd, rot, nd, alfrot, betrot, true, ws, lane);
    if (lane == 0) betrot[nd - 1] = beta[nd - 1];
    __syncwarp();
    return 0;
}

__device__ inline int get_tvec(int nd, const double *alpha, const double *beta, int irot, int nrot,
                               const double *rot, int nlam, const double *lambda, double *yy, double *ws, int lane) {
    if (nlam <= 0) return 0;
    double *d = ws, *e = ws + nd, *Z = e + nd, *tmp = Z + (size_t)nd * nd;
    int *idx = reinterpret_cast<int *>(tmp + nd);
    char *used = reinterpret_cast<char *>(idx + nlam);
    for (int i = lane; i < nd; i += 32) {
        d[i] = alpha[i];
        e[i] = (i + 1 < nd) ? beta[i] : 0.0;
    }
    for (size_t q = lane; q < (size_t)nd * nd; q += 32) Z[q] = 0.0;
    __syncwarp();
    for (int i = lane; i < nd; i += 32) Z[(size_t)i * nd + i] = 1.0;
    __syncwarp();
    if (tql_implicit(nd, d, e, Z, nd, nd, lane)) return -132;
    if (lane == 0) core::match_values(nd, d, nlam, lambda, -1.0, idx, used);
    __syncwarp();
    for (int i = 0; i < nlam; ++i)
        for (int r = lane; r < nd; r += 32) yy[(size_t)i * nd + r] = Z[(size_t)idx[i] * nd + r];
    __syncwarp();
    if (nrot > 1) {
        for (int c = 0; c < nlam; ++c) {
            double *col = yy + (size_t)c * nd + irot;
            for (int i = lane; i < nrot; i += 32) {
                double s = 0.0;
                for (int k = 0; k < nrot; ++k) s += rot[(size_t)k * nrot + i] * col[k];
                tmp[i] = s;
            }
            __syncwarp();
            for (int i = lane; i < nrot; i += 32) col[i] = tmp[i];
            __syncwarp();
        }
    }
    return 0;
}

__device__ inline int get_tvec_a(int nd, int kept, double *alpha, const double *beta, int nlam,
                                 const double *lambda, double *yy, double *ws, int lane) {
    if (nlam <= 0) return 0;
    double *H = ws, *w = H + (size_t)nd * nd, *wsel = w + nd, *wse = wsel + nd;
    int *idx = reinterpret_cast<int *>(wse + (size_t)nd * nd + 4 * nd);
    char *used = reinterpret_cast<char *>(idx + nd);
    for (size_t q = lane; q < (size_t)nd * nd; q += 32) H[q] = 0.0;
    __syncwarp();
    for (int i = lane; i < nd; i += 32) H[(size_t)i * nd + i] = alpha[i];
    for (int i = lane; i < kept; i += 32) {
        H[(size_t)kept * nd + i] = beta[i];
        H[(size_t)i * nd + kept] = beta[i];
    }
    for (int i = kept + lane; i < nd - 1; i += 32) {
        H[(size_t)(i + 1) * nd + i] = beta[i];
        H[(size_t)i * nd + i + 1] = beta[i];
    }
    __syncwarp();
    if (sym_eig(nd, H, nd, w, wse, lane)) return -142;
    for (int i = lane; i < nd; i += 32) alpha[i] = w[i];
    __syncwarp();
    if (nlam >= nd) {
        for (size_t q = lane; q < (size_t)nd * nd; q += 32) yy[q] = H[q];
        __syncwarp();
        return 0;
    }
    const double tol = core::hmax(DBL_EPSILON * nd *
                                      core::hmax(w[nd - 1] - w[0], core::hmax(fabs(w[nd - 1]), fabs(w[0]))),
                                  DBL_MIN);
    int rc = 0;
    if (lane == 0)
        rc = core::match_values(nd, w, nlam, lambda, core::hmax(tol, core::match_tol(nd, w)), idx, used);
    rc = __shfl_sync(kFull, rc, 0);
    __syncwarp();
    if (rc != 0) return -143;
    for (int i = 0; i < nlam; ++i) {
        for (int r = lane; r < nd; r += 32) yy[(size_t)i * nd + r] = H[(size_t)idx[i] * nd + r];
    }
    if (lane == 0)
        for (int i = 0; i < nlam; ++i) wsel[i] = w[idx[i]];
    __syncwarp();
    for (int i = lane; i < nlam; i += 32) alpha[i] = wsel[i];
    __syncwarp();
    return 0;
}

}  // namespace warp
}  // namespace trlb

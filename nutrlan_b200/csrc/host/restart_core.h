// Thick-restart policy: how many Ritz pairs to keep at a restart and (for
// schemes 7/8) the next basis size, shared by the host engine and the
// device-side batched solver (__host__ __device__ under nvcc).  The decision
// rules are those of the reference's SRC/restart.c (trl_shuffle_eig and the
// scheme helpers at :29-1408); they are restated here because
// info->restart must select the same behaviour, and hence the same matvec
// counts, as the reference.
#pragma once

#include "dense_core.h"

namespace trlb {
namespace core {

namespace restart_detail {

TRLB_HD inline int round_half_up(double x) { return (int)(x + 0.5); }

// Search window [klm, krm] for the brute-force schemes (restart.c:29-81).
// For lohi == 0 it also chooses a side and writes it to *lohi_out.
TRLB_HD inline void search_range(int nd, const double *res, trl_info *info, int ncl, int ncr,
                  int *lohi_out, int tind, int *klm, int *krm) {
    int kl = hmax(ncl, 0);
    int kr = hmin(ncr, nd - 1);
    double bnd = info->tol * info->anrm;
    *lohi_out = info->lohi;
    if (info->lohi > 0) {
        kr = hmin(hmax(info->maxlan - info->ned, (info->maxlan + info->nec) / 2) - 1,
                      hmin(kr, tind - 1));
        while (kr + kr > ncl + ncr && res[kr] < bnd) --kr;
    } else if (info->lohi < 0) {
        kl = hmax(hmin(info->ned, (info->maxlan + info->nec) / 2) - 1,
                      hmax(tind + 1, kl));
        while (kl + kl < ncl + ncr && res[kl] < bnd) ++kl;
    } else {
        if (tind - kl < kr - tind) {
            *lohi_out = -1;
            kl = tind + 1;
        } else {
            *lohi_out = 1;
            kr = tind - 1;
        }
        int j = info->locked + kl + nd - kr + 1;
        if (j > 0) {
            j /= 2;
            kl = hmax(0, kl - j);
            kr = hmin(kr + j, nd - 1);
        }
    }
    *klm = kl;
    *krm = kr;
}

// Smallest gap ratio that still converges all wanted pairs within maxmv.
TRLB_HD inline double min_gap_ratio(const trl_info *info, int nd, int tind, const double *res) {
    (void)nd;
    double gamma = info->maxmv * (info->nec + 1.0) / info->ned - info->matvec;
    if (gamma < info->klan)
        gamma = hmax((info->maxmv - info->matvec) / ((double)(info->ned - info->nec)), 2.0);
    return hmin(log(res[tind] / (info->tol * info->anrm)) / gamma, 0.5);
}

TRLB_HD inline double gap_ratio(int i, int j, int tind, const double *lambda) {
    return (lambda[i] - lambda[tind]) / (lambda[j] - lambda[tind]);
}

// Shared by the dynamic schemes 5 and 7: fraction of the search window that
// must separate the kept ends, from the observed vs predicted convergence.
TRLB_HD inline double dynamic_gap_fraction(trl_info *info) {
    const double kPi = 3.141592654;
    const double up = 1.0, dw = 0.7;
    info->avgm = (info->avgm * ((double)info->nloop - 1) + (double)(info->klan - info->k + 1)) /
                 ((double)info->nloop);
    double z1 = info->ptres / (info->tol * info->anrm);
    double z2 = 1.0 / info->cfac;
    if (z2 < 1.0) return 0.7;
    if (z1 < 1.0) return 1.0;
    double observed = log(z1 + sqrt(z1 - 1.0) * sqrt(z1 + 1.0)) / (2.0 * info->avgm);
    double achieved = log(z2 + sqrt(z2 - 1.0) * sqrt(z2 + 1.0)) /
                      (info->klan - info->k + 1);
    double t = pow(achieved / observed, 2.0);
    t = atan(t) * (2.0 / kPi);
    return dw + (up - dw) * t;
}

// Scheme 7: minimise (reorthogonalisation cost) / (expected residual
// reduction) over the kept ends (i, j) and the next basis size k.
TRLB_HD inline void scheme_gap_cost(int n, int tind, trl_info *info, const double *lambda,
                     const double *res, int *kl, int *kr) {
    int nd = info->ned, mn = info->maxlan, k1, k2;
    search_range(n, res, info, *kl, *kr, &info->lohi, tind, &k1, &k2);
    double frac = dynamic_gap_fraction(info);
    int t = (int)(abs(k2 - k1) * frac);
    double best = 0.0, best_gamma = 0.0, best_gamma0 = 0.0;
    int bk1 = k1, bk2 = k2, bm = info->klan, bl = 0;
    for (int i = k1; i <= k2 - t; ++i) {
        for (int j = i + t; j <= k2; ++j) {
            double gamma0 =
                sqrt((lambda[i + 1] - lambda[tind]) / (lambda[j - 1] - lambda[i + 1]));
            int l1 = (i + 1) + (n - j);
            int l2 = l1 + info->locked;
            int lo = hmax(hmin(l2 + 1, mn), nd);
            for (int k = lo; k <= mn; ++k) {
                double gamma = (k - l2) * gamma0;
                double val = ((k - l2) * (k + l2 - 1) + k * l1) / gamma;
                if (best == 0.0 || val < best) {
                    bk1 = i;
                    bk2 = j;
                    bm = k;
                    best = val;
                    best_gamma = gamma;
                    best_gamma0 = gamma0;
                    bl = l2;
                }
            }
        }
    }
    *kl = bk1;
    *kr = bk2;
    info->klan = bm;
    info->k1 = bk1;
    info->k2 = bk2;
    info->k = bl;
    info->predicted_crate = exp(-best_gamma);
    info->mgamma = best_gamma;
    info->gamma0 = best_gamma0;
    info->old_target = lambda[tind];
    info->target_id = tind;
    info->old_locked = info->locked;
}

// Scheme 8: as scheme 7 but the next basis size is fixed by rfact.
TRLB_HD inline void scheme_gap_cost_static(int n, int tind, trl_info *info, const double *lambda,
                            const double *res, int *kl, int *kr) {
    const double kPi = 3.141592654;
    int nd = info->ned, mn = info->maxlan, k1, k2, t;
    search_range(n, res, info, *kl, *kr, &info->lohi, tind, &k1, &k2);
    if (info->crat > 0.0) {
        double rate = -log(info->crat);
        double need = -(rate * info->maxlan) / log(info->tol * info->anrm);
        if (need >= 0.5 || info->klan < info->maxlan) {
            t = (int)(abs(k2 - k1) * 0.8);
        } else {
            double f = rate / min_gap_ratio(info, nd, tind, res);
            f = atan(pow(f, 0.25)) * (4.0 / kPi);
            t = (int)(abs(k2 - k1) * f);
        }
    } else {
        t = (int)(abs(k2 - k1) * 0.8);
    }
    int mn1 = round_half_up(2.0 * info->klan / 5.0);
    double best = 0.0;
    int bk1 = k1, bk2 = k2, bm = info->klan;
    for (int i = k1; i <= k2 - t; ++i) {
        for (int j = i + t; j <= k2; ++j) {
            double gamma0 =
                sqrt((lambda[i + 1] - lambda[tind]) / (lambda[j - 1] - lambda[i + 1]));
            int l1 = (i + 1) + (n - j);
            int l2 = l1 + info->locked;
            int m2 = mn1;
            if (mn1 < info->rfact * l2) m2 = (int)(info->rfact * l2);
            m2 = hmax(hmin(m2, mn), nd);
            double gamma = (m2 - l2 + 1) * gamma0;
            double val = (m2 * m2 - l2 * l2 + 2 * m2 * l1) / gamma;
            if (best == 0.0 || val < best) {
                bk1 = i;
                bk2 = j;
                bm = m2;
                best = val;
            }
        }
    }
    *kl = bk1;
    *kr = bk2;
    info->klan = bm;
}

// Number of extra pairs kept beyond the converged ones (schemes 1/2).
TRLB_HD inline int extra_pairs(int mnd, const trl_info *info) {
    int extra = round_half_up((mnd - info->nec) * (0.4 + 0.1 * info->ned / (double)mnd));
    if (extra > info->ned + info->ned && extra > 5) {
        double g = ((double)mnd) / ((double)info->ned);
        extra = round_half_up((extra + (log(g) * info->ned) * g) / (1.0 + g));
    }
    return extra;
}

// For lohi == 0: shift the window toward the end that converges faster.
TRLB_HD inline void balance_ends(const double *res, int kl0, int kr0, int *kl, int *kr) {
    while (*kl > kl0 && *kr < kr0) {
        if (10.0 * res[*kl] < res[*kr]) {
            if (res[*kl + 1] < res[*kr + 1]) {
                ++*kl;
                ++*kr;
            } else {
                break;
            }
        } else if (10.0 * res[*kr] < res[*kl]) {
            if (res[*kr - 1] < res[*kl - 1]) {
                --*kr;
                --*kl;
            } else {
                break;
            }
        } else {
            break;
        }
    }
}

// Scheme 1 (and 0): fixed number of extra pairs plus a minimum gap ratio.
TRLB_HD inline void scheme_fixed(int nd, int mnd, int tind, const double *lambda, const double *res,
                  trl_info *info, int *kl, int *kr) {
    int kli = *kl, kri = *kr, kl0 = kli, kr0 = kri;
    int extra = extra_pairs(mnd, info);
    int minsep = hmax(3, hmax(nd / 5, nd - 4 * info->ned));
    double gmin = min_gap_ratio(info, nd, tind, res);
    if (info->lohi > 0) {
        kri = hmin(tind - 1, kri) - extra;
        kli = -1;
    } else if (info->lohi < 0) {
        kli = hmax(tind + 1, kli) + extra;
        kri = nd;
    } else {
        ++extra;
        kli += extra / 2;
        kri -= extra / 2;
        balance_ends(res, kl0, kr0, &kli, &kri);
    }
    while (kli + minsep < kri &&
           gap_ratio(hmax(0, kli), hmin(kri, nd - 1), tind, lambda) < gmin) {
        if (info->lohi < 0)
            ++kli;
        else if (info->lohi > 0)
            --kri;
        else if (res[kli] < res[kri])
            ++kli;
        else
            ++kri;
    }
    // Keep near-duplicate Ritz values together.
    if (info->lohi > 0) {
        int i = kri - 1;
        while (i > kli + minsep && lambda[kri] - res[kri] < lambda[i] &&
               lambda[kri] + res[kri] < lambda[i] + res[i])
            --i;
        kri = i + 1;
    } else {
        int i = kli + 1;
        while (i < kri - minsep && lambda[kli] + res[kli] > lambda[i] &&
               lambda[kli] - res[kli] > lambda[i] - res[i])
            ++i;
        kli = i - 1;
    }
    *kl = kli;
    *kr = kri;
}

// Scheme 6: progressively vary the thickness.
TRLB_HD inline void scheme_scan(int nd, const double *res, trl_info *info, int kept, int *kl, int *kr) {
    int kli = *kl, kri = *kr;
    if (info->lohi < 0) {
        kri = nd;
        kli = kept + hmin(hmax(info->nec, 1), (nd - kept) / 2) - 1;
        if (kli <= 0) {
            if (nd > 6)
                kli = nd / 2 - 1;
            else if (nd > 2)
                kli = 1;
        } else if (kli + 3 > nd) {
            kli = info->nec + hmin(info->ned, hmin(10, (nd - info->ned) / 2)) - 1;
        }
    } else if (info->lohi > 0) {
        kli = -1;
        kri = kept + hmin(hmax(info->nec, 1), (nd - kept) / 2) - 1;
        if (kri <= 0) {
            if (nd > 6)
                kri = nd / 2 - 1;
            else if (nd > 2)
                kri = 1;
        } else if (kri + 4 > nd) {
            kri = info->nec + hmin(info->ned, hmin(10, (nd - info->ned) / 2));
        }
        kri = nd - kri - 1;
    } else {
        int kl0 = kli, kr0 = kri;
        int extra = kept + hmin(info->nec, (nd - kept) / 2) + 1;
        if (extra <= 0) {
            if (nd > 6)
                extra = nd / 2;
            else if (nd > 2)
                extra = 2;
        } else if (extra + 3 > nd) {
            extra = info->nec + hmin(info->ned, hmin(10, (nd - info->ned) / 2));
        }
        kli = hmax(kli, extra / 2 - 1);
        kri = hmin(kri, nd - extra / 2 - 1);
        balance_ends(res, kl0, kr0, &kli, &kri);
    }
    *kl = kli;
    *kr = kri;
}

// Scheme 2: keep the pairs whose residuals are close to the target's.
TRLB_HD inline void scheme_small_res(int nd, int mnd, int tind, const double *lambda, const double *res,
                      trl_info *info, int *kl, int *kr) {
    int minsep = hmax(3, hmax(nd / 5, nd - 4 * info->ned));
    int extra = extra_pairs(mnd, info);
    int kli = *kl, kri = *kr, kl0 = kli, kr0 = kri;
    double resmax = res[0];
    for (int i = 1; i < nd; ++i) resmax = hmax(resmax, res[i]);
    if (nd <= 0) resmax = 0.0;
    double acpt = resmax / res[tind];
    if (info->lohi > 0) {
        if (acpt < 0.999 && acpt >= 0.0) {
            int ii = tind - 1;
            acpt = hmin(hmax(sqrt(acpt) * res[tind], res[ii] + res[ii]), resmax);
            kri = ii - 1;
            while (res[kri] < acpt && kri > kli + 3) --kri;
        } else {
            kri = kr0 - extra;
        }
        kri = hmax(2, kri);
        kli = hmin(kli, kri - 2);
    } else if (info->lohi < 0) {
        if (acpt < 0.999 && acpt >= 0.0) {
            int ii = tind + 1;
            acpt = hmin(hmax(sqrt(acpt) * res[tind], res[ii] + res[ii]), resmax);
            kli = ii + 1;
            while (res[kli] < acpt && kli < kri - 3) ++kli;
        } else {
            kli = kl0 + extra;
        }
        kli = hmin(nd - 4, kli);
        kri = hmax(kri, kli + 2);
    } else {
        int i = kli + 1, j = kri - 1;
        for (int c = 1; c <= extra; ++c) {
            if (res[i] < res[j]) {
                kli = i++;
            } else if (res[i] > res[j]) {
                kri = j--;
            } else if (i < nd - j) {
                kli = i++;
            } else {
                kri = j--;
            }
        }
    }
    kl0 = kli;
    kr0 = kri;
    double gmin = min_gap_ratio(info, nd, tind, res);
    bool stuck = false;
    while (kli + minsep < kri &&
           gap_ratio(hmax(0, kli), hmin(nd - 1, kri), tind, lambda) < gmin && !stuck) {
        if (info->lohi < 0)
            ++kli;
        else if (info->lohi > 0)
            --kri;
        else if (res[kli] < res[kri])
            ++kli;
        else if (kri < nd - 1)
            ++kri;
        else
            stuck = true;
    }
    if (info->lohi > 0) {
        int i = kr0 - 1;
        while (i > kli + minsep && lambda[kri] - res[kri] < lambda[i] &&
               lambda[kri] + res[kri] < lambda[i] + res[i])
            --i;
        kri = hmin(kri, i + 1);
    } else {
        int i = kl0 + 1;
        while (i < kri - minsep && lambda[kli] + res[kli] > lambda[i] &&
               lambda[kli] - res[kli] > lambda[i] - res[i])
            ++i;
        kli = hmax(kli, i - 1);
    }
    *kl = kli;
    *kr = kri;
}

// Scheme 3: maximise the gap ratio of the target for a fixed window width.
TRLB_HD inline void scheme_max_gap(int nd, int tind, int kept, const double *lambda, const double *res,
                    trl_info *info, int *kl, int *kr) {
    auto gratio = [&](int i, int j) {
        return lambda[j] == info->trgt ? DBL_MAX
                                       : (lambda[i] - info->trgt) / (lambda[j] - info->trgt);
    };
    int lohi, klm, krm;
    search_range(nd, res, info, *kl, *kr, &lohi, tind, &klm, &krm);
    int kli = klm, kri = krm;
    int igap = hmax(hmin(nd - info->ned, round_half_up((krm - klm) * 0.4)), 2);
    if (igap > 2 && info->matvec > info->maxlan) {
        // The reference weighs operator time against the rest using its own
        // timers; the same fields are filled by this engine.
        if (info->clk_op + info->tick_o >
            10.0 * (info->clk_orth + info->tick_h + info->clk_res + info->tick_r)) {
            igap = hmax(2, nd - kept - 1);
        } else {
            double bnd = min_gap_ratio(info, nd, tind, res);
            if (info->crat < bnd) igap = hmax(2, nd - kept - 1);
        }
    }
    if (kli + igap > kri) {
        *kl = kli;
        *kr = kri;
        return;
    }
    if (lohi > 0) {
        double bnd = gratio(kri, kli);
        for (int i = klm; i <= krm - igap; ++i) {
            int j = i + igap;
            double tmp = gratio(j, i);
            if (tmp > bnd) {
                kli = i;
                kri = j;
                bnd = tmp;
            }
        }
    } else {
        double bnd = gratio(kli, kri);
        for (int i = klm; i <= krm - igap; ++i) {
            int j = i + igap;
            double tmp = gratio(i, j);
            if (tmp > bnd) {
                kli = i;
                kri = j;
                bnd = tmp;
            }
        }
    }
    *kl = kli;
    *kr = kri;
}

// Schemes 4 and 5: brute-force search of a merit function over (i, j).
template <class Merit>
TRLB_HD inline void brute_force(int lohi, int klm, int krm, int igap, Merit merit, double init, int *kl,
                 int *kr) {
    int kli = klm, kri = krm;
    double ss = init;
    for (int i = klm; i <= krm - igap; ++i) {
        for (int j = i + igap; j <= krm; ++j) {
            double tmp = lohi > 0 ? merit(j, i) : merit(i, j);
            if (tmp > ss) {
                ss = tmp;
                kli = i;
                kri = j;
            }
        }
    }
    *kl = kli;
    *kr = kri;
}

TRLB_HD inline void scheme_max_progress(int nd, int tind, int kept, const double *lambda, const double *res,
                         trl_info *info, int *kl, int *kr) {
    auto merit = [&](int i, int j) {
        return (lambda[i] - info->trgt) * abs(j - i) / (lambda[j] - info->trgt);
    };
    int lohi, klm, krm;
    search_range(nd, res, info, *kl, *kr, &lohi, tind, &klm, &krm);
    int igap = hmax(hmin(nd - info->ned, round_half_up((krm - klm) * 0.4)), 2);
    if (igap > 2 && igap + kept > nd && info->crat > 0.0) {
        double ss = min_gap_ratio(info, nd, tind, res);
        if (ss > info->crat) igap = hmax(2, nd - kept - 1);
    }
    double init = lohi > 0 ? merit(krm, klm) : merit(klm, krm);
    brute_force(lohi, klm, krm, igap, merit, init, kl, kr);
}

TRLB_HD inline void scheme_max_reduction(int nd, int tind, int kept, const double *lambda,
                          const double *res, trl_info *info, int *kl, int *kr) {
    auto merit = [&](int i, int j) {
        return sqrt((lambda[i] - info->trgt) / (lambda[j] - lambda[i])) * abs(j - i);
    };
    int lohi, klm, krm;
    search_range(nd, res, info, *kl, *kr, &lohi, tind, &klm, &krm);
    double frac = dynamic_gap_fraction(info);
    int igap = (int)(abs(krm - klm) * frac);
    if (igap > 2 && igap + kept > nd && info->crat > 0.0) {
        double ss = min_gap_ratio(info, nd, tind, res);
        if (ss > info->crat) igap = hmax(2, nd - kept - 1);
    }
    double init = lohi > 0 ? merit(krm, klm) : merit(klm, krm);
    brute_force(lohi, klm, krm, igap, merit, init, kl, kr);
}

}  // namespace restart_detail

TRLB_HD inline void shuffle_eig(int nd, int mnd, double *lambda, double *res, trl_info *info, int *kept,
                 int locked) {
    using namespace restart_detail;
    (void)locked;
    if (nd <= 5) {
        // Tiny basis: keep the pairs with the smallest residuals.
        sort2(nd, res, lambda);
        *kept = nd > 3 ? 2 : (nd > 0 ? 1 : 0);
        if (*kept > 1) sort2(*kept, lambda, res);
        return;
    }
    // Converged prefix/suffix (ncl: last converged from the left, ncr: first
    // converged from the right).
    double bnd = hmin(info->tol, DBL_EPSILON * info->anrm);
    int ncr = 0, ncl = nd - 1;
    for (int i = nd - 1; i >= 0; --i) {
        if (!(res[i] <= bnd)) {
            ncr = i + 1;
            break;
        }
    }
    for (int i = 0; i < nd; ++i) {
        if (!(res[i] <= bnd)) {
            ncl = i - 1;
            break;
        }
    }
    int kl = ncl, kr = ncr, tind;
    if (ncr > ncl) {
        // Binary search for the Ritz value closest to the target.
        tind = (kl + kr) / 2;
        while (lambda[tind] != info->trgt && kr > kl) {
            if (lambda[tind] < info->trgt) {
                kl = tind + 1;
                tind = (kl + kr) / 2;
            } else if (lambda[tind] > info->trgt) {
                kr = tind - 1;
                tind = (kl + kr) / 2;
            } else {
                kl = kr = tind;
            }
        }
        if (lambda[tind] == info->trgt) {
            kl = tind - 1;
            while (kl >= 0 && lambda[kl] == info->trgt) --kl;
            kr = tind + 1;
            while (kr < nd && lambda[kr] == info->trgt) ++kr;
        } else {
            kl = tind - 1;
            kr = tind + 1;
        }
        if (info->lohi > 0) {
            kr = kl;
            kl = hmin(ncl, hmax(0, nd - info->ned) - 1);
        } else if (info->lohi < 0) {
            kl = kr;
            kr = hmax(ncr, hmin(nd - info->nec, info->ned + 1) - 1);
        } else if (ncr - tind > tind - ncl) {
            kl = kr;
            kr = hmax(ncr, hmin(nd - info->nec, info->ned + 1) - 1);
        } else {
            kr = kl;
            kl = hmin(ncl, hmax(0, nd - info->ned) - 1);
        }
    } else {
        *kept = nd;
        return;
    }

    switch (info->restart) {
        case 0:
            if (info->restart <= -info->ned) {
                if (info->lohi >= 0) {
                    kl = -1;
                    kr = hmax(2, nd + info->restart);
                } else {
                    kl = hmin(-info->restart, nd - 3) - 1;
                    kr = nd;
                }
            } else {
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            }
            break;
        case 1:
            scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 2:
            scheme_small_res(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 3:
            if (info->nloop > 0)
                scheme_max_gap(nd, tind, *kept, lambda, res, info, &kl, &kr);
            else
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 4:
            if (info->nloop > 0)
                scheme_max_progress(nd, tind, *kept, lambda, res, info, &kl, &kr);
            else
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 5:
            if (info->nloop > 0)
                scheme_max_reduction(nd, tind, *kept, lambda, res, info, &kl, &kr);
            else
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 6:
            scheme_scan(nd, res, info, *kept, &kl, &kr);
            break;
        case 8:
            if (info->nloop > 0)
                scheme_gap_cost_static(nd, tind, info, lambda, res, &kl, &kr);
            else
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
        case 7:
        default:
            if (info->nloop > 0)
                scheme_gap_cost(nd, tind, info, lambda, res, &kl, &kr);
            else
                scheme_fixed(nd, mnd, tind, lambda, res, info, &kl, &kr);
            break;
    }

    // Enforce a minimum separation between the two kept ends.
    int minsep = hmax(3, hmax(nd / 6, nd - 6 * info->ned));
    if (kr <= kl + minsep || kl + nd - kr + minsep > mnd) {
        if (ncl < kl && kl < kr && kr < ncr) {
            --kl;
            ++kr;
        } else if (info->lohi > 0) {
            kr = hmax(minsep, hmin(nd / 3, ncr)) - 1;
            kl = -1;
        } else if (info->lohi < 0) {
            kl = hmin(nd - minsep, hmax((nd + nd) / 3, ncl + 2)) - 1;
            kr = nd;
        } else {
            kl = (nd - minsep) / 2 - 2;
            kr = (nd - minsep + 1) / 2;
        }
    }
    // Pack [0..kl] and [kr..nd) to the front.
    --kr;
    for (int i = 1; i < nd - kr; ++i) {
        lambda[kl + i] = lambda[kr + i];
        res[kl + i] = res[kr + i];
    }
    *kept = kl + hmax(1, nd - kr);
    if (info->lohi < -1) sort2(*kept, lambda, res);
}


}  // namespace core
}  // namespace trlb

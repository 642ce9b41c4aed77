// Batched thick-restart Lanczos: many independent real symmetric problems
// of uneven sizes solved by one persistent kernel launch.
//
// Every CTA repeatedly takes the next problem from an atomic work queue
// (problems sorted largest first) and runs a complete thick-restart Lanczos
// solve on it: the control flow of the reference's trlanczos
// (SRC/trlcore.c:723-1532; same usecgs decision, classical Gram-Schmidt pass
// loop, convergence tests and restart bookkeeping as the host engine), with
// the projected-problem work done by thread 0 using the very same
// __host__ __device__ routines as the host engine (dense_core.h,
// restart_core.h).  Vector work is block-wide: the operator (5-point
// stencil with a diagonal, or CSR), alpha and norm reductions, Gram-Schmidt
// projection/update against the problem's basis, and the restart
// recombination done in place tile by tile (the CTA owns all rows).
//
// The basis of each problem lives in HBM ((maxlan+1) columns); results are
// deterministic per problem regardless of which CTA solved it.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <numeric>
#include <vector>

#include "../../../include/trlx.h"
#include "../host/dense_core.h"
#include "../host/restart_core.h"
#include "batched.h"
#include "dense_warp.cuh"
#include "common.cuh"

namespace trlb {
namespace batched {

constexpr int kMaxL = 64;  // largest supported maxlan

struct Shared {
    trl_info info;
    double alpha[kMaxL + 2], beta[kMaxL + 2], alfrot[kMaxL + 2], betrot[kMaxL + 2];
    double lambda[kMaxL + 2], res[kMaxL + 2], h[kMaxL + 2], g[kMaxL + 2], wrk2[2 * (kMaxL + 2)];
    double red[32][17];
    double scal[8];
    int ctl[8];
};

// A group of threads of the CTA that solves one problem: its rank, size,
// named-barrier id and shared state.  The CTA is split into 1, 2 or 4
// groups per phase.
struct Grp {
    int tid, nt, bar;
    Shared *S;
    __device__ inline void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory"); }
};
// Dynamic shared memory after Shared: rot (L^2), yy (L^2), dense workspace.
__host__ __device__ inline size_t dyn_doubles(int maxlan) {
    return 2 * (size_t)maxlan * maxlan + core::dense_ws_doubles(maxlan) + 8;
}

size_t group_bytes(int maxlan);
__device__ inline size_t group_bytes_dev(int maxlan) {
    return ((sizeof(Shared) + 15) / 16 * 16 + dyn_doubles(maxlan) * sizeof(double) + 127) / 128 * 128;
}

enum { kAlpha = 0, kR2Pre = 1, kH2 = 2, kR2 = 3, kTmp = 4 };
enum { cGo = 0, cJnd = 1, cKept = 2, cLocked = 3, cFlag = 4, cIter = 5 };

// ---- block-wide helpers ---------------------------------------------------
// Sum K per-thread values over the block (fixed order); result in out[0..K).
template <int K>
__device__ inline void block_reduce(double (&v)[K], double *out, const Grp &G) {
    Shared &S = *G.S;
    const int lane = G.tid & 31, warp = G.tid >> 5, nw = G.nt >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) S.red[warp][k] = v[k];
    }
    G.sync();
    if (G.tid < K) {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += S.red[w][G.tid];
        out[G.tid] = s;
    }
    G.sync();
}

__device__ inline double block_sum1(double v, const Grp &G) {
    double a[1] = {v};
    block_reduce<1>(a, &G.S->scal[kTmp], G);
    return G.S->scal[kTmp];
}

// y = A x; returns alpha = x.y (all threads).
__device__ inline double apply_op(const Params &P, const Problem &pr, const double *x, double *y, const Grp &G) {
    double a = 0.0;
    const int n = pr.n;
    if (P.format == kFormatStencil5) {
        // Two rows per thread per round with all their loads issued first
        // (neighbour indices clamped into the grid, the boundary terms
        // dropped afterwards), so twice the loads are in flight; each row's
        // arithmetic and the order of the alpha sum are unchanged.
        constexpr int U = 2;
        const int L = pr.L;
        const double *d = P.diag + pr.diag_off;
        for (int i0 = G.tid; i0 < n; i0 += U * G.nt) {
            double xc[U], xl[U], xr[U], xd[U], xu[U], dd[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = min(i0 + u * G.nt, n - 1);
                xc[u] = x[i];
                dd[u] = d[i];
                xl[u] = x[max(i - 1, 0)];
                xr[u] = x[min(i + 1, n - 1)];
                xd[u] = x[max(i - L, 0)];
                xu[u] = x[min(i + L, n - 1)];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int i = i0 + u * G.nt;
                if (i < n) {
                    const int ix = i % L, iy = i / L;
                    double s = (4.0 + dd[u]) * xc[u];
                    if (ix > 0) s -= xl[u];
                    if (ix < L - 1) s -= xr[u];
                    if (iy > 0) s -= xd[u];
                    if (iy < L - 1) s -= xu[u];
                    y[i] = s;
                    a += xc[u] * s;
                }
            }
        }
    } else {
        const long long *rp = P.row_ptr + pr.rp_off;
        const int *ci = P.col + pr.ent_off;
        const double *va = P.val + pr.ent_off;
        for (int i = G.tid; i < n; i += G.nt) {
            double s = 0.0;
            for (long long k = rp[i]; k < rp[i + 1]; ++k) s += va[k] * x[ci[k]];
            y[i] = s;
            a += x[i] * s;
        }
    }
    return block_sum1(a, G);
}

// h[c] = V[:,c].r (c < m) with r = y - alpha x - beta xp when rec (r is
// written back into y by a first pass); returns |r|^2 and |h|^2 to every
// thread of the group.  The columns are cut
// into chunks of CW; the chunks of a round run side by side, each on its
// own subgroup of warps sweeping every row, so each row of y (and x, xp) is
// fetched from memory once per round and found in L1 by the other
// subgroups, and one reduction covers the whole round.  Rows are taken in
// pairs with 16-byte loads (basis columns are 256-byte aligned, ld a
// multiple of 32); an odd last row is handled by the first thread of each
// subgroup.  Padding rows (n .. ld) are never read.
__device__ inline double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }

struct Norms {
    double r2, h2;  // |r|^2 and |h|^2 of a projection
};

template <int CW>
__device__ inline Norms project(const double *V, int ld, int n, int m, double *y, bool rec, const double *x,
                                const double *xp, double alpha, double beta, const Grp &G) {
    Shared &S = *G.S;
    const int lane = G.tid & 31, warp = G.tid >> 5, nw = G.nt >> 5;
    const int np = n >> 1;
    const int nchunks = (m + CW - 1) / CW;
    double r2 = 0.0, r2tot = 0.0;
    if (rec) {
        // r = y - alpha x - beta xp written back into y first, so that the
        // column passes hold no recurrence operands (registers) and the
        // update reads one vector.
        // Two row pairs per thread per round, loads first.
        for (int p0 = G.tid; p0 < np; p0 += 2 * G.nt) {
            const int p1 = p0 + G.nt;
            const int i0 = 2 * p0, i1 = 2 * min(p1, np - 1);
            const double2 y0 = ld2(y + i0), x0 = ld2(x + i0), q0 = ld2(xp + i0);
            const double2 y1 = ld2(y + i1), x1 = ld2(x + i1), q1 = ld2(xp + i1);
            *reinterpret_cast<double2 *>(y + i0) =
                make_double2(y0.x - (alpha * x0.x + beta * q0.x), y0.y - (alpha * x0.y + beta * q0.y));
            if (p1 < np)
                *reinterpret_cast<double2 *>(y + i1) =
                    make_double2(y1.x - (alpha * x1.x + beta * q1.x), y1.y - (alpha * x1.y + beta * q1.y));
        }
        if ((n & 1) && G.tid == 0) y[n - 1] -= alpha * x[n - 1] + beta * xp[n - 1];
        G.sync();
    }
    for (int ch0 = 0; ch0 < max(nchunks, 1); ch0 += nw) {
        const int nc = max(1, min(nw, nchunks - ch0));  // chunks side by side (one when m == 0)
        const int wps = nw / nc;                         // warps per subgroup
        const int sub = warp / wps;
        const bool act = sub < nc;
        const int c0 = (ch0 + sub) * CW;
        const int mm = act ? max(0, min(CW, m - c0)) : 0;
        const int stride = wps * 32, t = G.tid - sub * stride;
        const bool count = act && ch0 == 0 && sub == 0;  // one subgroup sums |r|^2
        double acc[CW];
#pragma unroll
        for (int k = 0; k < CW; ++k) acc[k] = 0.0;
        if (act) {
            const double *Vc = V + (size_t)c0 * ld;
            for (int p = t; p < np; p += stride) {
                const int i = 2 * p;
                const double2 yv = ld2(y + i);
                const double r0 = yv.x, r1 = yv.y;
                if (count) {
                    r2 += r0 * r0;
                    r2 += r1 * r1;
                }
#pragma unroll
                for (int k = 0; k < CW; ++k)
                    if (k < mm) {
                        const double2 v = ld2(Vc + (size_t)k * ld + i);
                        acc[k] = fma(v.x, r0, acc[k]);
                        acc[k] = fma(v.y, r1, acc[k]);
                    }
            }
            if ((n & 1) && t == 0) {
                const int i = n - 1;
                const double ri = y[i];
                if (count) r2 += ri * ri;
#pragma unroll
                for (int k = 0; k < CW; ++k)
                    if (k < mm) acc[k] = fma(Vc[(size_t)k * ld + i], ri, acc[k]);
            }
        }
        // Warp partials, then each column summed over its subgroup's warps
        // in warp order (a fixed order: results do not depend on timing);
        // |r|^2 rides along in slot CW of the first round.
#pragma unroll
        for (int k = 0; k < CW; ++k) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
        }
        double r2w = r2;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r2w += __shfl_down_sync(0xffffffffu, r2w, o);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < CW; ++k) S.red[warp][k] = acc[k];
            S.red[warp][CW] = r2w;
        }
        G.sync();
        if (G.tid < nc * CW) {
            const int sc = G.tid / CW, k = G.tid - sc * CW;
            const int c = (ch0 + sc) * CW + k;
            if (c < m) {
                double v = 0.0;
                for (int w = sc * wps; w < (sc + 1) * wps; ++w) v += S.red[w][k];
                S.h[c] = v;
            }
        }
        if (ch0 == 0) {  // every thread forms the same total, in warp order
            r2tot = 0.0;
            for (int w = 0; w < nw; ++w) r2tot += S.red[w][CW];
        }
        G.sync();
    }
    double h2 = 0.0;
    for (int c = 0; c < m; ++c) h2 += S.h[c] * S.h[c];
    return Norms{r2tot, h2};
}

// r = (y - alpha x - beta xp) - V h (in place in y); returns |r|^2 to every
// thread (the reduction's barriers also publish the new y).
// Row pairs as in project; the column loop issues eight 16-byte loads before
// their FMAs (each element's FMA chain keeps the column order).
__device__ inline double update(const double *V, int ld, int n, int m, double *y, bool rec, const double *x,
                              const double *xp, double alpha, double beta, const double *h, const Grp &G) {
    constexpr int UC = 8;
    double r2 = 0.0;
    const int np = n >> 1;
    for (int p = G.tid; p < np; p += G.nt) {
        const int i = 2 * p;
        const double2 yv = ld2(y + i);
        double r0 = yv.x, r1 = yv.y;
        if (rec) {
            const double2 xv = ld2(x + i), pv = ld2(xp + i);
            r0 -= alpha * xv.x + beta * pv.x;
            r1 -= alpha * xv.y + beta * pv.y;
        }
        int c = 0;
        for (; c + UC <= m; c += UC) {
            double2 v[UC];
#pragma unroll
            for (int k = 0; k < UC; ++k) v[k] = ld2(V + (size_t)(c + k) * ld + i);
#pragma unroll
            for (int k = 0; k < UC; ++k) {
                r0 = fma(-v[k].x, h[c + k], r0);
                r1 = fma(-v[k].y, h[c + k], r1);
            }
        }
        if (c < m) {  // the last partial chunk, its loads issued together
            double2 v[UC];
#pragma unroll
            for (int k = 0; k < UC; ++k) v[k] = c + k < m ? ld2(V + (size_t)(c + k) * ld + i) : make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < UC; ++k)
                if (c + k < m) {
                    r0 = fma(-v[k].x, h[c + k], r0);
                    r1 = fma(-v[k].y, h[c + k], r1);
                }
        }
        *reinterpret_cast<double2 *>(y + i) = make_double2(r0, r1);
        r2 += r0 * r0;
        r2 += r1 * r1;
    }
    if ((n & 1) && G.tid == 0) {
        const int i = n - 1;
        double ri = y[i];
        if (rec) ri -= alpha * x[i] + beta * xp[i];
        for (int c = 0; c < m; ++c) ri = fma(-V[(size_t)c * ld + i], h[c], ri);
        y[i] = ri;
        r2 += ri * ri;
    }
    return block_sum1(r2, G);
}

__device__ inline void scale(double *y, int n, double sc, const Grp &G) {
    // Four elements per thread per round, loads first.
    constexpr int U = 4;
    for (int i0 = G.tid; i0 < n; i0 += U * G.nt) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = y[min(i0 + u * G.nt, n - 1)];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (i0 + u * G.nt < n) y[i0 + u * G.nt] = v[u] * sc;
    }
    G.sync();
}

// Smoothed random vector (the breakdown restart; same stencil as the engine).
__device__ inline void random_vector(double *y, int n, uint64_t seed, const Grp &G) {
    for (int i = G.tid; i < n; i += G.nt) {
        auto u = [&](long k) { return uniform01(seed, (uint64_t)k); };
        double v;
        if (n < 3)
            v = u(i);
        else if (i == 0)
            v = 2.0 * u(0) + u(2) + u(n - 1);
        else if (i == n - 1)
            v = 2.0 * u(n - 1) + (2.0 * u(1) + u(2) + u(0)) + u(n - 2);
        else
            v = 2.0 * u(i) + u(i + 1) + u(i - 1);
        y[i] = v;
    }
    G.sync();
}

// Classical Gram-Schmidt of column m against columns 0..m-1, continuing
// after a first pass whose scalars are in S.scal (trl_cgs,
// SRC/trlcore.c:2913-3117).  Returns the status; *rnrm the final norm.
template <int CW>
// pass_done: the first pass was made by the caller, whose |h|^2 and |r|^2
// are h2_done and r2_done.
__device__ inline int cgs(const Params &P, int pid, double *V, int ld, int n, int m, bool pass_done, double h2_done,
                          double r2_done, double *rnrm, const Grp &G) {
    Shared &S = *G.S;
    double *r = V + (size_t)m * ld;
    const int maxorth = 3;
    int irnd = 0, cnt = 0;
    double normrr2 = 0.0, normdiff2 = 0.0;
    if (m > 0) {
        bool first = true;
        while (cnt <= maxorth) {
            if (!(first && pass_done)) {
                normdiff2 = project<CW>(V, ld, n, m, r, false, nullptr, nullptr, 0.0, 0.0, G).h2;
                normrr2 = update(V, ld, n, m, r, false, nullptr, nullptr, 0.0, 0.0, S.h, G);
            } else {
                normdiff2 = h2_done;
                normrr2 = r2_done;
            }
            first = false;
            if (G.tid == 0) S.info.north++;
            cnt++;
            *rnrm = sqrt(normrr2);
            if (DBL_EPSILON * normrr2 > normdiff2) break;
            if ((cnt > 1 && (m * DBL_EPSILON * DBL_EPSILON * (normrr2 + normdiff2) < normdiff2)) ||
                !(normrr2 > DBL_MIN)) {
                if (irnd > 0) break;
                cnt = 0;
                irnd++;
                if (G.tid == 0) S.info.nrand++;
                G.sync();
                random_vector(r, n, P.seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(pid + 1)) ^
                                        (7919ull * (uint64_t)S.info.nrand), G);
            }
        }
        if (normrr2 < normdiff2) return -203;
    }
    if (*rnrm > DBL_MIN)
        scale(r, n, 1.0 / *rnrm, G);
    else
        return -204;
    if (irnd > 0) *rnrm = 0.0;
    return 0;
}

// trl_orth (SRC/trlcore.c:1766-1975) for the new column m: alpha(m-1) is in
// S.alpha, the recurrence uses beta_prev; sets S.beta[m-1].
template <int CW>
__device__ inline int orth(const Params &P, int pid, double *V, int ld, int n, int m, bool recur, double beta_prev,
                           double a, int kept, const Grp &G) {
    Shared &S = *G.S;
    const int jnd = m, jm1 = jnd - 1;
    double *r = V + (size_t)m * ld;
    const double *x = V + (size_t)(m - 1) * ld;
    const double *xp = m >= 2 ? V + (size_t)(m - 2) * ld : nullptr;
    const Norms pn = project<CW>(V, ld, n, m, r, recur, x, xp, a, beta_prev, G);
    const double normrr2 = pn.r2;
    if (!(normrr2 >= 0.0) || !(normrr2 <= DBL_MAX)) return -102;
    double tmp = a * a;
    // beta of the previous steps are in S.beta (thread-uniform reads).
    if (jm1 > kept) {
        tmp += S.beta[jm1 - 1] * S.beta[jm1 - 1];
    } else if (kept > 0) {
        for (int i = 0; i < jm1; ++i) tmp += S.beta[i] * S.beta[i];
    }
    bool usecgs;
    if (jm1 == kept) {
        usecgs = true;
    } else if (jnd >= S.info.ntot) {
        usecgs = false;
    } else if (DBL_EPSILON * normrr2 >= tmp) {
        double anorm = 0.0;
        for (int i = 0; i < jnd; ++i) anorm = fmax(anorm, fabs(S.alpha[i]) + fabs(i == jnd - 1 ? sqrt(normrr2) : S.beta[i]));
        usecgs = sqrt(normrr2) < DBL_EPSILON * anorm * S.info.ntot;
    } else {
        usecgs = true;
    }
    double beta_new;
    if (usecgs) {
        const double r2u = update(V, ld, n, m, r, false, nullptr, nullptr, 0.0, 0.0, S.h, G);
        double rnrm = sqrt(normrr2);
        const int st = cgs<CW>(P, pid, V, ld, n, m, true, pn.h2, r2u, &rnrm, G);
        if (st) return st;
        beta_new = rnrm;
    } else {
        // Local re-orthogonalisation against the last one or two vectors.
        if (G.tid == 0) {
            for (int c = 0; c < m; ++c) S.g[c] = (c >= m - min(2, m)) ? S.h[c] : 0.0;
        }
        G.sync();
        update(V, ld, n, m, r, false, nullptr, nullptr, 0.0, 0.0, S.g, G);
        if (G.tid == 0) S.alpha[jnd - 1] += S.h[m - 1];
        beta_new = sqrt(normrr2);
        G.sync();
        scale(r, n, 1.0 / beta_new, G);
    }
    if (G.tid == 0) {
        double b = beta_new;
        if (b <= DBL_EPSILON * fabs(S.alpha[jnd - 1]))
            b = 0.0;
        else if (jnd >= S.info.ntot)
            b = 0.0;
        S.beta[jnd - 1] = b;
    }
    G.sync();
    return 0;
}

// In place V[:, lck .. lck+kept) <- V[:, lck .. lck+jml) * yy (jml x kept),
// tile by tile (the CTA owns every row, so no other reader exists).
__device__ inline void ritz_in_place(double *V, int ld, int n, int lck, int jml, int kept, const double *yy,
                                     double *tile, long tile_cap /* doubles */, const Grp &G) {
    // As many rows per tile as the group's free shared memory holds (two
    // group barriers per tile), rounded down to a multiple of 32 when that
    // is at least 32; never more than the capacity.
    int kTile = (int)min((long)n, tile_cap / max(jml, 1));
    if (kTile >= 32) kTile = kTile / 32 * 32;
    kTile = max(kTile, 1);
    // Tile fill: row pairs with 16-byte loads when the tile height is even
    // (r0, rr even: aligned in the basis column and in the tile).  Products:
    // each thread forms two output columns from one read of the tile value;
    // every output sums over c in ascending order.
    const bool pairs = (kTile & 1) == 0;
    const int kp = kept / 2;
    for (int r0 = 0; r0 < n; r0 += kTile) {
        const int rows = min(kTile, n - r0);
        const int rp = pairs ? rows / 2 : 0;
        for (int e = G.tid; e < rp * jml; e += G.nt) {
            const int pr = e % rp, c = e / rp;
            const double2 v = ld2(V + (size_t)(lck + c) * ld + r0 + 2 * pr);
            *reinterpret_cast<double2 *>(tile + c * kTile + 2 * pr) = v;
        }
        const int rest = rows - 2 * rp;  // rows not covered by pairs
        for (int e = G.tid; e < rest * jml; e += G.nt) {
            const int rr = 2 * rp + e % rest, c = e / rest;
            tile[c * kTile + rr] = V[(size_t)(lck + c) * ld + r0 + rr];
        }
        G.sync();
        for (int e = G.tid; e < rows * kp; e += G.nt) {
            const int rr = e % rows, k = 2 * (e / rows);
            const double *y0 = yy + (size_t)k * jml, *y1 = y0 + jml;
            double s0 = 0.0, s1 = 0.0;
            for (int c = 0; c < jml; ++c) {
                const double t = tile[c * kTile + rr];
                s0 = fma(t, y0[c], s0);
                s1 = fma(t, y1[c], s1);
            }
            V[(size_t)(lck + k) * ld + r0 + rr] = s0;
            V[(size_t)(lck + k + 1) * ld + r0 + rr] = s1;
        }
        if (kept & 1) {
            const int k = kept - 1;
            for (int rr = G.tid; rr < rows; rr += G.nt) {
                double s = 0.0;
                for (int c = 0; c < jml; ++c) s = fma(tile[c * kTile + rr], yy[(size_t)k * jml + c], s);
                V[(size_t)(lck + k) * ld + r0 + rr] = s;
            }
        }
        G.sync();
    }
}

__device__ inline void init_info(trl_info *info, int n, int maxlan, int lohi, int ned, double tol, int restart,
                                 int maxmv) {
    unsigned char *b = reinterpret_cast<unsigned char *>(info);
    for (size_t i = 0; i < sizeof(trl_info); ++i) b[i] = 0;
    info->tol = tol;
    info->restart = restart > 0 ? restart : 0;
    info->maxmv = maxmv;
    info->maxlan = maxlan;
    info->lohi = lohi;
    info->ned = ned;
    info->nloc = info->ntot = n;
    info->tmv = -1;
    info->trgt = -DBL_MAX;
    info->tres = -1.0;
    info->crat = 1.0;
    info->npes = 1;
    info->klan = min(maxlan, n);
    if (info->restart >= 7) info->klan = min(maxlan, max(100, min(info->klan, 2 * ned)));
}

// One complete solve of problem pid by the calling CTA.
template <int CW>
__device__ void solve(const Params &P, int pid, const Grp &G, double *dyn, long tile_cap) {
    Shared &S = *G.S;
    const Problem pr = P.probs[pid];
    const int n = pr.n, ld = pr.ld, maxlan = P.maxlan, ned = P.ned, mev = ned + 1;
    double *V = P.basis + pr.basis_off;
    double *rot = dyn, *yy = dyn + (size_t)maxlan * maxlan, *dws = yy + (size_t)maxlan * maxlan;
    double *tile = dws;  // the restart tile reuses the dense workspace
    trl_info *info = &S.info;
    if (G.tid == 0) init_info(info, n, maxlan, P.lohi, ned, P.tol, P.restart, P.maxmv);
    G.sync();
    // Start vector: caller's, or seeded uniform[-1, 1].
    const uint64_t seed = P.seed + 0x9E3779B97F4A7C15ull * (uint64_t)(pid + 1);
    for (int i = G.tid; i < n; i += G.nt)
        V[i] = pr.start_off >= 0 ? P.start[pr.start_off + i] : 2.0 * uniform01(seed, (uint64_t)i) - 1.0;
    G.sync();
    double nrm = sqrt(block_sum1([&] {
        double s = 0.0;
        for (int i = G.tid; i < n; i += G.nt) s += V[i] * V[i];
        return s;
    }(), G));
    int stat = 0;
    if (!(nrm > DBL_MIN)) stat = -204;
    if (!stat) scale(V, n, 1.0 / nrm, G);
    int jnd = 0, kept = 0, locked = 0;
    int i1 = ned;
    int next_test = i1 + min(i1, min(6, ned / 2));
    int prek = 0;
    while (!stat && info->matvec < info->maxmv && info->nec < info->ned) {
        jnd++;
        if (jnd + 1 > maxlan + 1) {
            stat = -1111;
            break;
        }
        // First step after (re)start: arrowhead coupling.
        double a = apply_op(P, pr, V + (size_t)(jnd - 1) * ld, V + (size_t)jnd * ld, G);
        if (G.tid == 0) {
            info->matvec++;
            S.alpha[jnd - 1] = a;
            S.beta[jnd - 1] = a;
        }
        G.sync();
        update(V, ld, n, jnd, V + (size_t)jnd * ld, false, nullptr, nullptr, 0.0, 0.0, S.beta, G);
        stat = orth<CW>(P, pid, V, ld, n, jnd, false, 0.0, a, kept, G);
        if (stat) break;
        if (G.tid < 32) {
            const int lane = G.tid;
            for (int i = lane; i < locked; i += 32) {
                S.alfrot[i] = S.alpha[i];
                S.betrot[i] = 0.0;
            }
            __syncwarp();
            warp::arrow_to_tridiag(jnd - locked, &S.alpha[locked], &S.beta[locked], rot, &S.alfrot[locked],
                                   &S.betrot[locked], dws, lane);
            if (lane == 0) S.betrot[jnd - 1] = S.beta[jnd - 1];
        }
        G.sync();
        while (jnd < info->klan && info->nec < info->ned) {
            jnd++;
            a = apply_op(P, pr, V + (size_t)(jnd - 1) * ld, V + (size_t)jnd * ld, G);
            if (G.tid == 0) {  // published by the projection's first barrier
                info->matvec++;
                S.alpha[jnd - 1] = a;
            }
            stat = orth<CW>(P, pid, V, ld, n, jnd, true, S.beta[jnd - 2], a, kept, G);
            if (G.tid == 0) {
                S.alfrot[jnd - 1] = S.alpha[jnd - 1];
                S.betrot[jnd - 1] = S.beta[jnd - 1];
                if (!stat && info->matvec >= next_test) {
                    int e = core::get_eval(jnd, locked, S.alfrot, S.betrot, S.lambda, S.res, dws);
                    if (e) {
                        S.ctl[cFlag] = e;
                    } else {
                        core::convergence_test(jnd, S.lambda, S.res, info, S.wrk2);
                        if (info->nec < info->ned && info->nec > 0) {
                            next_test = (int)((double)(info->ned * info->matvec) / (double)info->nec);
                        } else if (info->nec == 0) {
                            next_test = next_test + next_test;
                            if (info->maxlan == info->ntot) next_test = (int)ceil(0.5 * (info->maxlan + info->matvec));
                        }
                        S.ctl[cFlag] = 0;
                    }
                } else {
                    S.ctl[cFlag] = 0;
                }
                S.ctl[cIter] = next_test;
            }
            G.sync();
            next_test = S.ctl[cIter];
            if (stat) break;
            if (S.ctl[cFlag]) {
                stat = S.ctl[cFlag];
                break;
            }
        }
        if (stat) break;
        // ---- restart or finish ------------------------------------------------
        // Lane 0 of warp 0 takes the decisions; the O(maxlan^3) eigenvector
        // work runs on the whole warp (dense_warp.cuh), then all apply.
        prek = kept;
        if (G.tid < 32) {
            const int lane = G.tid;
            int st = 0, go = 0, path = 0;
            const int jml = jnd - locked;
            int i2 = kept - locked + 1;
            int kk = kept;
            if (lane == 0) {
                if (info->nec < info->ned) {
                    st = core::get_eval(jnd, locked, S.alfrot, S.betrot, S.lambda, S.res, dws);
                    if (!st) core::convergence_test(jnd, S.lambda, S.res, info, S.wrk2);
                }
                if (!st && info->nec < info->ned && info->matvec < info->maxmv) {
                    go = 1;
                    core::shuffle_eig(jml, info->klan - locked, &S.lambda[locked], &S.res[locked], info, &kk,
                                      locked);
                    path = kk * 3 < jml ? 1 : 2;
                } else if (!st) {
                    // Final: sort and compute the wanted eigenvectors.
                    kk = min(info->nec, max(info->ned, mev - 1));
                    info->nec = kk;
                    if (kk == 0) kk = min(mev - 1, info->ned);
                    core::sort_eig(jnd, info->lohi, kk, info->ref, S.lambda, S.res);
                    for (int i = 0; i < kk; ++i) S.wrk2[i] = S.lambda[i];
                    path = kk * 3 < jnd ? 3 : 4;
                }
            }
            st = __shfl_sync(0xffffffffu, st, 0);
            go = __shfl_sync(0xffffffffu, go, 0);
            path = __shfl_sync(0xffffffffu, path, 0);
            kk = __shfl_sync(0xffffffffu, kk, 0);
            __syncwarp();
            int ts = 0;
            if (!st && go) {
                if (path == 1) {
                    ts = warp::get_tvec(jml, &S.alfrot[locked], &S.betrot[locked], 0, i2, rot, kk, &S.lambda[locked],
                                        yy, dws, lane);
                    if (ts == 0 && lane == 0)
                        for (int i = 0; i < locked + kk; ++i) S.alpha[i] = S.lambda[i];
                    __syncwarp();
                }
                if (path == 2 || ts != 0) {
                    if (lane == 0)
                        for (int i = 0; i < locked + kk; ++i) S.alfrot[i] = S.lambda[i];
                    __syncwarp();
                    ts = warp::get_tvec_a(jml, prek - locked, &S.alpha[locked], &S.beta[locked], kk,
                                          &S.alfrot[locked], yy, dws, lane);
                }
                if (lane == 0) {
                    if (ts) st = ts;
                    if (!st) {
                        for (int i = 0; i < kk; ++i) S.beta[locked + i] = yy[(size_t)(i + 1) * jml - 1] * S.betrot[jnd - 1];
                        if (jml > info->ned + (info->ned / 5 + 6))
                            core::set_locking(jml, kk, &S.alpha[locked], &S.beta[locked], yy, info->anrm, &i2);
                        else
                            i2 = 0;
                        S.ctl[cJnd] = jml;       // columns recombined
                        S.ctl[cKept] = kk;
                        S.ctl[cLocked] = i2;     // newly locked
                    }
                }
            } else if (!st) {
                double *ev = S.wrk2;
                if (path == 3) ts = warp::get_tvec(jnd, S.alfrot, S.betrot, locked, i2, rot, kk, ev, yy, dws, lane);
                if (path == 4 || ts != 0) ts = warp::get_tvec_a(jnd, prek, S.alpha, S.beta, kk, ev, yy, dws, lane);
                if (lane == 0) {
                    if (ts) st = ts;
                    for (int i = 0; i < kk; ++i) {
                        S.alpha[i] = ev[i];
                        S.beta[i] = S.betrot[jnd - 1] * yy[(size_t)(1 + i) * jnd - 1];
                    }
                    S.ctl[cJnd] = jnd;
                    S.ctl[cKept] = kk;
                }
            }
            if (lane == 0) {
                S.ctl[cGo] = go;
                S.ctl[cFlag] = st;
            }
        }
        G.sync();
        if (S.ctl[cFlag]) {
            stat = S.ctl[cFlag];
            break;
        }
        const int jml = S.ctl[cJnd];
        kept = S.ctl[cKept];
        if (S.ctl[cGo]) {
            // Restart: kept Ritz vectors in place, then the residual vector.
            ritz_in_place(V, ld, n, locked, jml, kept, yy, tile, tile_cap, G);
            const double *rr = V + (size_t)jnd * ld;
            double *dst = V + (size_t)(locked + kept) * ld;
            for (int i = G.tid; i < n; i += G.nt) dst[i] = rr[i];
            G.sync();
            kept += locked;
            locked += S.ctl[cLocked];
            jnd = kept;
            if (G.tid == 0) {
                info->locked = locked;
                if (info->nec > 0)
                    next_test = (int)(((double)(info->matvec * info->ned)) / ((double)info->nec));
                else
                    next_test = next_test + info->maxlan;
                S.ctl[cIter] = next_test;
                info->nloop++;
            }
            G.sync();
            next_test = S.ctl[cIter];
        } else {
            // Final eigenvectors straight into the output (not in place).
            double *out = P.evec + pr.evec_off;
            for (long e = G.tid; e < (long)n * kept; e += G.nt) {
                const int i = (int)(e % n), k = (int)(e / n);
                double s = 0.0;
                for (int c = 0; c < jml; ++c) s = fma(V[(size_t)c * ld + i], yy[(size_t)k * jml + c], s);
                out[(size_t)k * n + i] = s;
            }
            if (G.tid == 0) info->nloop++;
            G.sync();
            break;
        }
    }
    if (G.tid == 0) {
        const int ne = min(ned, max(info->nec, 0));
        for (int i = 0; i < ned; ++i) {
            P.eval[(size_t)pid * ned + i] = i < ne ? S.alpha[i] : 0.0;
            P.res[(size_t)pid * ned + i] = i < ne ? fabs(S.beta[i]) : -1.0;
        }
        int *o = P.info_out + (size_t)pid * 4;
        o[0] = stat;
        o[1] = info->nec;
        o[2] = info->matvec;
        o[3] = info->nloop;
    }
    G.sync();
}

// Phases run largest problems first; in phase f the CTA is split into
// groups of P.phase_threads[f] threads, each group taking problems from the
// phase's queue until it is empty, then the whole CTA moves on.
// CTA: threads per CTA; CW: basis columns per projection pass.  The
// 1024-thread form has 64 registers per thread (CW 8 or 4); the 512-thread
// form has up to 128 (CW 16).
template <int CTA, int CW>
__global__ void __launch_bounds__(CTA, 1) k_batched(Params P) {
    extern __shared__ __align__(16) unsigned char smem[];
    for (int f = 0; f < P.nphases; ++f) {
        const int nt = P.phase_threads[f];
        const int gidx = threadIdx.x / nt;
        const int ngroups = blockDim.x / nt;
        // Each group gets an equal share of the CTA's shared memory; what
        // its fixed state leaves free extends the restart tile (which starts
        // at the dense workspace).
        const size_t per_group = max(group_bytes_dev(P.maxlan), P.smem_total / (size_t)ngroups / 128 * 128);
        const size_t head = (sizeof(Shared) + 15) / 16 * 16;
        const long tile_cap =
            (long)((per_group - head) / sizeof(double)) - 2L * P.maxlan * P.maxlan;
        if (gidx < ngroups) {
            // Barrier ids by split level (1 for the whole CTA, 2-3 for
            // halves, 4-7 for quarters, 8-15 for eighths), so groups of
            // different phases never share one.
            Grp G{(int)threadIdx.x - gidx * nt, nt, ngroups + gidx,
                  reinterpret_cast<Shared *>(smem + gidx * per_group)};
            double *dyn = reinterpret_cast<double *>(smem + gidx * per_group + (sizeof(Shared) + 15) / 16 * 16);
            for (;;) {
                if (G.tid == 0) G.S->ctl[cGo] = P.phase_begin[f] + (int)atomicAdd(P.queue + f, 1u);
                G.sync();
                const int q = G.S->ctl[cGo];
                G.sync();
                if (q >= P.phase_end[f]) break;
                solve<CW>(P, P.order[q], G, dyn, tile_cap);
            }
        }
        // When the next phase splits each group further (or not at all),
        // its groups are made of this group's threads and shared memory
        // (equal shares nest), so a group goes on without waiting for the
        // rest of the CTA; a coarser next phase needs the whole CTA.
        const bool nested = f + 1 < P.nphases && nt % P.phase_threads[f + 1] == 0;
        if (!nested) __syncthreads();
    }
}

size_t group_bytes(int maxlan) {
    return ((sizeof(Shared) + 15) / 16 * 16 + dyn_doubles(maxlan) * sizeof(double) + 127) / 128 * 128;
}
// Shared memory for the largest split used by the launch.
size_t smem_bytes(int maxlan, int min_threads, int cta) { return group_bytes(maxlan) * (cta / min_threads); }

// What a launch asks for: the split's need, raised to kLaunchSmem so the
// restart tiles of 1024- and 512-thread groups hold a few hundred rows; the
// rest of the SM's 256 KB stays L1 cache, which the Gram-Schmidt passes'
// re-reads of r and the previous vectors rely on.
constexpr size_t kLaunchSmem = 96 * 1024;
static size_t launch_smem(int maxlan, int min_threads, int cta) {
    static const size_t want = [] {
        const char *e = std::getenv("TRLX_BATCH_SMEM_KB");  // tuning only
        const long kb = e ? std::atol(e) : 0;
        return kb > 0 ? (size_t)kb * 1024 : kLaunchSmem;
    }();
    return std::max(smem_bytes(maxlan, min_threads, cta), want);
}

// Columns per projection pass of the 1024-thread form: 8, or 4 under
// TRLX_BATCH_CW=4 (tuning only; fewer live registers under the 64-register
// cap).  The 512-thread form uses 16.
static int cw1024() {
    static const int cw = [] {
        const char *e = std::getenv("TRLX_BATCH_CW");
        return (e && std::atoi(e) == 4) ? 4 : 8;
    }();
    return cw;
}

template <int CTA, int CW>
static int launch_cta(const Params &P, int blocks, cudaStream_t st) {
    int min_threads = CTA;
    for (int f = 0; f < P.nphases; ++f) min_threads = std::min(min_threads, P.phase_threads[f]);
    const size_t sm = launch_smem(P.maxlan, min_threads, CTA);
    if (cudaFuncSetAttribute(k_batched<CTA, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
        cudaSuccess)
        return -1001;
    Params Q = P;
    Q.smem_total = sm;
    k_batched<CTA, CW><<<blocks, CTA, sm, st>>>(Q);
    return cudaGetLastError() == cudaSuccess ? 0 : -1001;
}

int launch(const Params &P, int blocks, cudaStream_t st) {
    if (P.cta == 512) return launch_cta<512, 16>(P, blocks, st);
    return cw1024() == 4 ? launch_cta<1024, 4>(P, blocks, st) : launch_cta<1024, 8>(P, blocks, st);
}

template <int CTA, int CW>
static int blocks_per_sm(int min_threads, int maxlan) {
    int nb = 0;
    const size_t sm = launch_smem(maxlan, min_threads, CTA);
    cudaFuncSetAttribute(k_batched<CTA, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_batched<CTA, CW>, CTA, sm) != cudaSuccess) return 1;
    return std::max(nb, 1);
}

int max_blocks_per_sm(int min_threads, int maxlan, int cta) {
    if (cta == 512) return blocks_per_sm<512, 16>(min_threads, maxlan);
    return cw1024() == 4 ? blocks_per_sm<1024, 4>(min_threads, maxlan) : blocks_per_sm<1024, 8>(min_threads, maxlan);
}

}  // namespace batched
}  // namespace trlb

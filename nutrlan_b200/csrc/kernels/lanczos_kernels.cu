// Lanczos vector kernels for sm_100a: classical Gram-Schmidt projection and
// update (tall-skinny V^H r and r - V h), normalisation, and the restart
// recombination V*Y.  These replace the reference's BLAS-2/3 calls in
// trl_cgs (SRC/trlcore.c:2993-3011, trl_g_dot_ in SRC/trl_comm_none.c:238)
// and trl_ritz_vectors (SRC/trlcore.c:2761-2910), and their complex twins
// (SRC/ztrlcore.c:1977-2203, 1570-1751).
//
// All streaming kernels read 16-byte vectors per lane, keep every partial sum
// in FP64, and reduce across the grid in a fixed order (per-block partials,
// summed in block order by the last block to finish), so results are
// bitwise reproducible run to run.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include "lanczos_kernels.h"

namespace trlb {

namespace {

int g_num_sms = 0;

int num_sms() {
    if (g_num_sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (g_num_sms <= 0) g_num_sms = 148;
    }
    return g_num_sms;
}

constexpr int kThreads = 256;
// Columns per warp in the projection: 8 warps x 16 = 128 real columns per
// sweep (8 for complex types, which carry twice the accumulator registers).
template <class T>
constexpr int proj_cpw() {
    return std::is_same<typename Store<T>::C, double>::value ? 16 : 8;
}

enum TicketSlot { kTicketDot = 0, kTicketProject = 1, kTicketUpdate = 2 };

// ---------------------------------------------------------------------------
template <class C>
__global__ void __launch_bounds__(kThreads) k_dot(const C *__restrict__ x, const C *__restrict__ y,
                                                  long n_pad, double *part, unsigned *ticket,
                                                  double *out) {
    __shared__ double red[32];
    double acc = 0.0;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
        C xv = x[i], yv = y[i];
        C t = czero(xv);
        fma_conj(t, xv, yv);
        acc += real_part(t);
    }
    double s = block_sum(acc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part, gridDim.x, red);
        if (threadIdx.x == 0) {
            *out = tot;
            *ticket = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Projection h = V^H r.  Block b owns rows [b*chunk, (b+1)*chunk).  Columns
// are cut into groups of CPW; a sweep gives each of the 8 warps one group
// when there are at least 8 groups, otherwise the warps of a group split the
// block's rows between them (so a short basis still keeps every warp
// streaming).  Every lane keeps one FP64 accumulator per column across its
// rows, each basis element is read once, and partial sums are combined in a
// fixed order (lanes by shuffle tree, warps of a group in warp order).
// Resident blocks per SM the projection is compiled for: as many as the
// accumulators (CPW per lane, complex counts double) and the per-lane loads
// (R elements per column) leave registers for, without spilling.
template <class T, int CPW>
constexpr int proj_min_blocks() {
    return !std::is_same<typename Store<T>::C, double>::value
               ? 2
               : (Store<T>::R == 4 ? (CPW >= 12 ? 2 : 3) : (CPW >= 16 ? 2 : (CPW >= 12 ? 3 : 4)));
}

// Shared by the projection kernels (register and staged forms).
// End of one sweep: each warp's CPW column sums are reduced over its lanes,
// then each column over the warps of its group in warp order, into the
// block's partials.
template <class C, int CPW>
__device__ __forceinline__ void project_sweep_end(C (&acc)[CPW], C (*red_c)[CPW], int c0, int G, int per, int wpg,
                                                  int m, C *part) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < CPW; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] = acc[k] + shfl_down(acc[k], o);
        if (lane == 0) red_c[warp][k] = acc[k];
    }
    __syncthreads();
    if (threadIdx.x < G * CPW) {
        const int gg = threadIdx.x / CPW, k = threadIdx.x - gg * CPW;
        const int c = c0 + gg * per + k;
        if (k < per && c < m) {
            C s = czero(C());
            for (int sl = 0; sl < wpg; ++sl) s = s + red_c[gg * wpg + sl][k];
            part[(long)blockIdx.x * m + c] = s;
        }
    }
    __syncthreads();
}

// With no columns (m == 0) the pass still returns ||r||^2 of the block's
// rows; the NT threads split the rows.
template <int R, int NT, class C>
__device__ __forceinline__ double project_norm_only(const C *r, Recur<C> rec, double alpha, double beta, long row0,
                                                    long row1) {
    double r2acc = 0.0;
    for (long i = row0 + (long)threadIdx.x * R; i < row1; i += (long)NT * R) {
        C rv[R];
        load_c<R>(r + i, rv);
        if (rec.on) {
            C xv[R], xpv[R];
            load_c<R>(rec.x + i, xv);
            load_c<R>(rec.xp + i, xpv);
#pragma unroll
            for (int q = 0; q < R; ++q) rv[q] = rv[q] - alpha * xv[q] - beta * xpv[q];
        }
#pragma unroll
        for (int q = 0; q < R; ++q) r2acc += abs2(rv[q]);
    }
    return r2acc;
}

// The block's ||r||^2 partial (warps in order), then, in the last block to
// finish, the grid totals: h (column sums in block order), ||h||^2 and
// ||r||^2.  NT is the block size.
template <class C, int NT>
__device__ __forceinline__ void project_finish(double r2acc, C *part, double *part_r2, unsigned *ticket, C *h,
                                               double *out2, int m) {
    constexpr int W = NT / 32;
    __shared__ double red_r2[W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r2acc += __shfl_down_sync(0xffffffffu, r2acc, o);
    if (lane == 0) red_r2[warp] = r2acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < W; ++w) s += red_r2[w];
        part_r2[blockIdx.x] = s;
    }
    if (last_block_arrived(ticket)) {
        __shared__ C red_cols[NT];
        __shared__ double red_r2x[32];
        const int nb = gridDim.x;
        const double h2 = reduce_columns(part, nb, m, h, red_cols);
        const double r2 = sum_partials(part_r2, nb, red_r2x);
        if (threadIdx.x == 0) {
            out2[0] = r2;
            out2[1] = h2;
            *ticket = 0;
        }
    }
}

// PS: the warp's column pointers live in shared memory and are re-read at
// every use instead of being held in 2 * CPW registers.  For 64-bit and
// complex storage the freed registers buy a third resident block; for FP32
// storage they hold the 16 columns' float4 loads, all issued before the
// first is consumed, at two blocks per SM (a third block would leave room
// for about half of them).
template <class T>
constexpr int proj_ps_blocks() {
    return std::is_same<T, float>::value ? 2 : 3;
}

template <class T, int CPW, bool PS = false>
__global__ void __launch_bounds__(kThreads, (PS ? proj_ps_blocks<T>() : proj_min_blocks<T, CPW>()))
    k_project(T *const *__restrict__ cols, int m, long n_pad, long chunk,
              const typename Store<T>::C *__restrict__ r, Recur<typename Store<T>::C> rec,
              typename Store<T>::C *part, double *part_r2, unsigned *ticket,
              typename Store<T>::C *h, double *out2) {
    using S = Store<T>;
    using C = typename S::C;
    constexpr int R = S::R;
    constexpr int W = kThreads / 32;
    __shared__ C red_c[W][CPW];
    __shared__ const T *sp[PS ? W : 1][PS ? CPW : 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long row0 = (long)blockIdx.x * chunk;
    const long row1 = min(n_pad, row0 + chunk);
    const double alpha = rec.on ? *rec.alpha : 0.0;
    const double beta = rec.on ? (rec.beta_r2 ? sqrt(*rec.beta_r2) : rec.beta) : 0.0;
    double r2acc = 0.0;
    // A sweep covers up to W * CPW columns.  Its mc columns are cut into G
    // groups (G the smallest power of two with G * CPW >= mc) of `per`
    // columns each, and each group's W / G warps split the rows, so every
    // warp streams whatever the basis size.
    for (int c0 = 0; c0 < m; c0 += W * CPW) {
        const int mc = min(W * CPW, m - c0);
        int G = 1;
        while (G < W && G * CPW < mc) G *= 2;
        const int per = (mc + G - 1) / G;
        const int wpg = W / G;
        const int grp = warp / wpg, slice = warp - grp * wpg;
        const int cb = c0 + grp * per;
        const int cn = max(0, min(per, m - cb));
        const bool active = cn > 0;
        const T *p[PS ? 1 : CPW];
        if constexpr (PS) {
            if (lane < CPW) sp[warp][lane] = lane < cn ? cols[cb + lane] : nullptr;
            __syncwarp();
        } else {
#pragma unroll
            for (int k = 0; k < CPW; ++k) p[k] = k < cn ? cols[cb + k] : nullptr;
        }
        C acc[CPW];
#pragma unroll
        for (int k = 0; k < CPW; ++k) acc[k] = czero(C());
        const bool count_r2 = (c0 == 0 && grp == 0);
        if (active) {
            for (long i = row0 + (long)(slice * 32 + lane) * R; i < row1; i += (long)wpg * 32 * R) {
                C rv[R];
                load_c<R>(r + i, rv);
                if (rec.on) {
                    C xv[R], xpv[R];
                    load_c<R>(rec.x + i, xv);
                    load_c<R>(rec.xp + i, xpv);
#pragma unroll
                    for (int q = 0; q < R; ++q) rv[q] = rv[q] - alpha * xv[q] - beta * xpv[q];
                }
                if (count_r2) {
#pragma unroll
                    for (int q = 0; q < R; ++q) r2acc += abs2(rv[q]);
                }
#pragma unroll
                for (int k = 0; k < CPW; ++k) {
                    const T *pk;
                    if constexpr (PS)
                        pk = *reinterpret_cast<const T *const volatile *>(&sp[warp][k]);
                    else
                        pk = p[k];
                    if (pk) {
                        C v[R];
                        S::load(pk + i, v);
#pragma unroll
                        for (int q = 0; q < R; ++q) fma_conj(acc[k], v[q], rv[q]);
                    }
                }
            }
        }
        project_sweep_end<C, CPW>(acc, red_c, c0, G, per, wpg, m, part);
    }
    if (m == 0) r2acc = project_norm_only<R, kThreads>(r, rec, alpha, beta, row0, row1);
    project_finish<C, kThreads>(r2acc, part, part_r2, ticket, h, out2, m);
}

// ---------------------------------------------------------------------------
// Projection with the basis staged through shared memory by cp.async
// (kProjectAsync).  The register forms above hold every basis load in
// flight in registers, next to an FP64 accumulator and a pointer per
// column, and the register file caps the bytes in flight per SM: FP32 and
// complex storage stop at 80-90% of the HBM peak.  Here each lane copies its
// own 16 bytes of each of its warp's CPW columns into a ring of NS stages in
// shared memory (NW = 16 warps x 8 columns x 3 stages = 192 KB, one block of
// 512 threads per SM), so NS - 1 stages (128 KB per SM) are in flight while
// the warp consumes the oldest.  A lane reads back only
// the bytes it copied itself, so the ring needs no barrier: the thread's own
// cp.async.wait_group orders them.  r, x and x' (shared by the block's warps
// and mostly served by L1/L2) are plain loads issued one iteration ahead.
// Column groups, row split and the order of every sum are those of
// k_project.
// 16 warps of 8 columns and three stages measured best among 8 x 16,
// 16 x 8, 16 x 6 (four stages) and 32 x 4 (spills for complex storage) on
// FP64, FP32, complex128 and complex64 columns at 16-128 columns.
constexpr int kAsyncWarps = 16, kAsyncCols = 8, kAsyncStages = 3;
template <int NW, int CPW, int NS>
constexpr size_t async_smem() {
    return (size_t)NW * NS * CPW * 32 * 16;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <class T, int NW, int CPW, int NS>
__global__ void __launch_bounds__(NW * 32, 1)
    k_project_async(T *const *__restrict__ cols, int m, long n_pad, long chunk,
                    const typename Store<T>::C *__restrict__ r, Recur<typename Store<T>::C> rec,
                    typename Store<T>::C *part, double *part_r2, unsigned *ticket,
                    typename Store<T>::C *h, double *out2) {
    using S = Store<T>;
    using C = typename S::C;
    constexpr int R = S::R;
    constexpr int W = NW, NT = NW * 32;
    static_assert(sizeof(T) * R == 16, "one 16-byte copy per lane and column");
    extern __shared__ __align__(16) unsigned char ring_raw[];
    __shared__ C red_c[W][CPW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // This lane's 16 bytes of column k in stage q.
    T *const ring = reinterpret_cast<T *>(ring_raw) + (size_t)warp * NS * CPW * 32 * R;
    auto slot = [&](int q, int k) { return ring + ((size_t)(q * CPW + k) * 32 + lane) * R; };
    const long row0 = (long)blockIdx.x * chunk;
    const long row1 = min(n_pad, row0 + chunk);
    const double alpha = rec.on ? *rec.alpha : 0.0;
    const double beta = rec.on ? (rec.beta_r2 ? sqrt(*rec.beta_r2) : rec.beta) : 0.0;
    double r2acc = 0.0;
    for (int c0 = 0; c0 < m; c0 += W * CPW) {
        const int mc = min(W * CPW, m - c0);
        int G = 1;
        while (G < W && G * CPW < mc) G *= 2;
        const int per = (mc + G - 1) / G;
        const int wpg = W / G;
        const int grp = warp / wpg, slice = warp - grp * wpg;
        const int cb = c0 + grp * per;
        const int cn = max(0, min(per, m - cb));
        const T *p[CPW];
#pragma unroll
        for (int k = 0; k < CPW; ++k) p[k] = k < cn ? cols[cb + k] : nullptr;
        C acc[CPW];
#pragma unroll
        for (int k = 0; k < CPW; ++k) acc[k] = czero(C());
        const bool count_r2 = (c0 == 0 && grp == 0);
        const long step = (long)wpg * 32 * R;
        const long first = row0 + (long)(slice * 32 + lane) * R;  // this lane's first row
        const long wfirst = row0 + (long)slice * 32 * R;           // the warp's first row
        const int nit = (cn > 0 && wfirst < row1) ? (int)((row1 - wfirst + step - 1) / step) : 0;
        auto issue = [&](int t) {
            const long i = first + (long)t * step;
            if (t < nit && i < row1) {
#pragma unroll
                for (int k = 0; k < CPW; ++k)
                    if (p[k]) cp_async16(slot(t % NS, k), p[k] + i);
            }
            cp_async_commit();
        };
        C rn[R], xn[R], xpn[R];
#pragma unroll
        for (int q = 0; q < R; ++q) rn[q] = xn[q] = xpn[q] = czero(C());
        auto load_vectors = [&](int t) {
            const long i = first + (long)t * step;
            if (t < nit && i < row1) {
                load_c<R>(r + i, rn);
                if (rec.on) {
                    load_c<R>(rec.x + i, xn);
                    load_c<R>(rec.xp + i, xpn);
                }
            }
        };
#pragma unroll
        for (int q = 0; q < NS - 1; ++q) issue(q);
        load_vectors(0);
        for (int t = 0; t < nit; ++t) {
            issue(t + NS - 1);  // into the slot consumed at t - 1
            C rv[R];
#pragma unroll
            for (int q = 0; q < R; ++q) rv[q] = rec.on ? rn[q] - alpha * xn[q] - beta * xpn[q] : rn[q];
            load_vectors(t + 1);
            cp_async_wait<NS - 1>();  // this thread's copies of stage t have landed
            if (first + (long)t * step < row1) {
                if (count_r2) {
#pragma unroll
                    for (int q = 0; q < R; ++q) r2acc += abs2(rv[q]);
                }
#pragma unroll
                for (int k = 0; k < CPW; ++k) {
                    if (p[k]) {
                        C v[R];
                        S::lds(slot(t % NS, k), v);
#pragma unroll
                        for (int q = 0; q < R; ++q) fma_conj(acc[k], v[q], rv[q]);
                    }
                }
            }
        }
        cp_async_wait<0>();
        project_sweep_end<C, CPW>(acc, red_c, c0, G, per, wpg, m, part);
    }
    if (m == 0) r2acc = project_norm_only<R, NT>(r, rec, alpha, beta, row0, row1);
    project_finish<C, NT>(r2acc, part, part_r2, ticket, h, out2, m);
}

// ---------------------------------------------------------------------------
// Update for short vectors (few rows per thread): a block works on tiles of
// 32 * R rows; its 8 warps take every 8th column of the tile, so each
// thread's chain of dependent loads is m / 8 long instead of m, and the
// slices' partial sums are combined in shared memory in slice order.
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_update_split(T *const *__restrict__ cols, int m, long n_pad, const typename Store<T>::C *r,
                   Recur<typename Store<T>::C> rec, const typename Store<T>::C *__restrict__ h,
                   typename Store<T>::C *r_out, double *part_r2, unsigned *ticket, double *out_r2) {
    using S = Store<T>;
    using C = typename S::C;
    constexpr int R = S::R;
    constexpr int NS = kThreads / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *hs = reinterpret_cast<C *>(smem_raw);
    const T **ps = reinterpret_cast<const T **>(smem_raw + sizeof(C) * m);
    __shared__ C red[NS][32 * R];
    for (int c = threadIdx.x; c < m; c += blockDim.x) {
        hs[c] = h[c];
        ps[c] = cols[c];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, sl = threadIdx.x >> 5;
    const double alpha = rec.on ? *rec.alpha : 0.0;
    const double beta = rec.on ? (rec.beta_r2 ? sqrt(*rec.beta_r2) : rec.beta) : 0.0;
    double r2acc = 0.0;
    for (long t0 = (long)blockIdx.x * 32 * R; t0 < n_pad; t0 += (long)gridDim.x * 32 * R) {
        const long i = t0 + (long)lane * R;
        C acc[R];
#pragma unroll
        for (int q = 0; q < R; ++q) acc[q] = czero(C());
        for (int c = sl; c < m; c += NS) {
            C v[R];
            S::load(ps[c] + i, v);
            const C hc = hs[c];
#pragma unroll
            for (int q = 0; q < R; ++q) fms(acc[q], v[q], hc);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) red[sl][lane * R + q] = acc[q];
        __syncthreads();
        if (sl == 0) {
            C base[R];
            load_c<R>(r + i, base);
            if (rec.on) {
                C xv[R], xpv[R];
                load_c<R>(rec.x + i, xv);
                load_c<R>(rec.xp + i, xpv);
#pragma unroll
                for (int q = 0; q < R; ++q) base[q] = base[q] - alpha * xv[q] - beta * xpv[q];
            }
#pragma unroll
            for (int q = 0; q < R; ++q) {
                for (int k = 0; k < NS; ++k) base[q] = base[q] + red[k][lane * R + q];
                r2acc += abs2(base[q]);
            }
            store_c<R>(r_out + i, base);
        }
        __syncthreads();
    }
    __shared__ double redb[32];
    double s = block_sum(r2acc, redb);
    if (threadIdx.x == 0) part_r2[blockIdx.x] = s;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part_r2, gridDim.x, redb);
        if (threadIdx.x == 0) {
            *out_r2 = tot;
            *ticket = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Update r_out = r - V h with h and the column pointers staged in shared
// memory; each thread owns R consecutive rows and walks the columns with four
// independent 16-byte loads in flight.
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_update(T *const *__restrict__ cols, int m, long n_pad, const typename Store<T>::C *r,
             Recur<typename Store<T>::C> rec, const typename Store<T>::C *__restrict__ h,
             typename Store<T>::C *r_out, double *part_r2, unsigned *ticket, double *out_r2) {
    using S = Store<T>;
    using C = typename S::C;
    constexpr int R = S::R;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *hs = reinterpret_cast<C *>(smem_raw);
    const T **ps = reinterpret_cast<const T **>(smem_raw + sizeof(C) * m);
    for (int c = threadIdx.x; c < m; c += blockDim.x) {
        hs[c] = h[c];
        ps[c] = cols[c];
    }
    __syncthreads();
    const double alpha = rec.on ? *rec.alpha : 0.0;
    const double beta = rec.on ? (rec.beta_r2 ? sqrt(*rec.beta_r2) : rec.beta) : 0.0;
    double r2acc = 0.0;
    const long stride = (long)gridDim.x * blockDim.x * R;
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) * R; i < n_pad; i += stride) {
        C acc[R];
        load_c<R>(r + i, acc);
        if (rec.on) {
            C xv[R], xpv[R];
            load_c<R>(rec.x + i, xv);
            load_c<R>(rec.xp + i, xpv);
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] = acc[q] - alpha * xv[q] - beta * xpv[q];
        }
        int c = 0;
        for (; c + 4 <= m; c += 4) {
            C v0[R], v1[R], v2[R], v3[R];
            S::load(ps[c] + i, v0);
            S::load(ps[c + 1] + i, v1);
            S::load(ps[c + 2] + i, v2);
            S::load(ps[c + 3] + i, v3);
            const C h0 = hs[c], h1 = hs[c + 1], h2 = hs[c + 2], h3 = hs[c + 3];
#pragma unroll
            for (int q = 0; q < R; ++q) {
                fms(acc[q], v0[q], h0);
                fms(acc[q], v1[q], h1);
                fms(acc[q], v2[q], h2);
                fms(acc[q], v3[q], h3);
            }
        }
        for (; c < m; ++c) {
            C v[R];
            S::load(ps[c] + i, v);
            const C hc = hs[c];
#pragma unroll
            for (int q = 0; q < R; ++q) fms(acc[q], v[q], hc);
        }
        store_c<R>(r_out + i, acc);
#pragma unroll
        for (int q = 0; q < R; ++q) r2acc += abs2(acc[q]);
    }
    __shared__ double red[32];
    double s = block_sum(r2acc, red);
    if (threadIdx.x == 0) part_r2[blockIdx.x] = s;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part_r2, gridDim.x, red);
        if (threadIdx.x == 0) {
            *out_r2 = tot;
            *ticket = 0;
        }
    }
}

// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kThreads)
    k_normalize(typename Store<T>::C *r, long n_pad, const double *r2, double fixed,
                typename Store<T>::C *q, T *vcol) {
    using S = Store<T>;
    using C = typename S::C;
    // Four elements per thread per round, their loads issued together
    // (coalesced: element u of a round is `stride` after element u - 1).
    constexpr int U = 4;
    const double sc = r2 ? 1.0 / sqrt(*r2) : fixed;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i0 = (long)blockIdx.x * blockDim.x + threadIdx.x; i0 < n_pad; i0 += U * stride) {
        C v[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (i0 + u * stride < n_pad) v[u] = r[i0 + u * stride];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long i = i0 + u * stride;
            if (i < n_pad) {
                const C w = v[u] * sc;
                q[i] = w;
                if (vcol) vcol[i] = S::from_c(w);
            }
        }
    }
}

constexpr int kBK = 16;  // K columns per shared-memory stage of the Ritz product

// ---------------------------------------------------------------------------
// Restart recombination out[:,k] = sum_c in[:,c] Y[c,k] with a real Y (FP64
// accumulate) on the FP64 tensor-core instruction (mma.sync.m8n8k4.f64;
// FP64 has no tcgen05 kind).  Complex bases use it through their real view
// (ritz_dispatch).  A block of 8 warps computes BM x BN outputs; each
// warp owns a 32 x 32 tile (4 x 4 mma tiles of 8 x 8, 32 accumulators per
// thread), so 8 fragment loads from shared memory feed 16 mma (4096 FMAs).
// K advances 16 columns per shared-memory stage (4 mma k-steps) with the
// next stage prefetched into registers.  Shared tiles are k-major with a row
// pitch of (rows + 4) doubles.  A warp's 64-bit fragment loads are served per
// half-warp (4 rows x 4 k); with a pitch of 4 mod 16 doubles the four k rows
// start 8 banks apart, so each half-warp is one conflict-free wavefront.
// Fragment layout of m8n8k4 .f64 (g = lane / 4, t = lane % 4):
// A (row-major 8x4): a = A[g][t]; B (col-major 4x8): b = B[t][g];
// C/D (8x8): c0, c1 = C[g][2t], C[g][2t+1].
template <int BN>
struct MmaShape {
    static constexpr int WC = BN / 32;      // warps along columns
    static constexpr int WR = 8 / WC;       // warps along rows
    static constexpr int BM = 32 * WR;      // rows per block (256 or 128)
};

__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <class T, class OutT, int BN>
__global__ void __launch_bounds__(kThreads)
    k_ritz_mma(T *const *__restrict__ in_cols, int jml, const double *__restrict__ Y, int ldy, int kept,
               OutT *const *out_cols, OutT *out, long ldo, long n_valid) {
    using S = Store<T>;
    using Sh = MmaShape<BN>;
    constexpr int BM = Sh::BM, APITCH = BM + 4, BPITCH = BN + 4;
    static_assert(APITCH % 16 == 4 && BPITCH % 16 == 4 && (APITCH * 8) % 16 == 0, "bank-spread pitches");
    // Rows per load: two for every storage type (a 16-byte FP64 load, an
    // 8-byte FP32 one), so that each thread's two rows land in shared memory
    // as one conflict-free 16-byte store (four FP32 rows per thread spread a
    // half-warp's stores over twice the banks' wavefronts).
    constexpr int R = 2;
    static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value, "real storage only");
    constexpr int CH = BM / R / 16;      // loads per thread per stage
    constexpr int BPT = BN * kBK / kThreads;
    __shared__ __align__(16) double As[kBK][APITCH];
    __shared__ double Bs[kBK][BPITCH];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int g = lane >> 2, tg = lane & 3;
    const int wr = warp % Sh::WR, wc = warp / Sh::WR;
    const long i0 = (long)blockIdx.x * BM;
    const int k0 = blockIdx.y * BN;
    // Stage loads: 16 threads per column (a_kk = t / 16); thread chunk j
    // covers rows ((t % 16) + 16 j) * R .. + R, so 16 consecutive threads read
    // 256 contiguous bytes and write 16 consecutive smem chunks.
    const int a_kk = t >> 4, a_ch = t & 15;
    double areg[CH * R];
    double breg[BPT];
    auto load_stage = [&](int c0) {
        const int c = c0 + a_kk;
        if (c < jml) {
            const T *col = in_cols[c] + i0;
#pragma unroll
            for (int j = 0; j < CH; ++j) {
                const T *p = col + (a_ch + 16 * j) * R;
                if constexpr (std::is_same<T, float>::value) {
                    const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
                    areg[j * R] = v.x;
                    areg[j * R + 1] = v.y;
                } else {
                    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
                    areg[j * R] = v.x;
                    areg[j * R + 1] = v.y;
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < CH * R; ++q) areg[q] = 0.0;
        }
#pragma unroll
        for (int e = 0; e < BPT; ++e) {
            const int idx = t + e * kThreads;
            const int kk = idx / BN, kc = idx % BN;
            const int cc = c0 + kk, k = k0 + kc;
            breg[e] = (cc < jml && k < kept) ? Y[(long)cc + (long)k * ldy] : 0.0;
        }
    };
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    load_stage(0);
    for (int c0 = 0; c0 < jml; c0 += kBK) {
#pragma unroll
        for (int j = 0; j < CH; ++j)
#pragma unroll
            for (int r = 0; r < R; r += 2)
                *reinterpret_cast<double2 *>(&As[a_kk][(a_ch + 16 * j) * R + r]) =
                    make_double2(areg[j * R + r], areg[j * R + r + 1]);
#pragma unroll
        for (int e = 0; e < BPT; ++e) {
            const int idx = t + e * kThreads;
            Bs[idx / BN][idx % BN] = breg[e];
        }
        __syncthreads();
        if (c0 + kBK < jml) load_stage(c0 + kBK);
#pragma unroll
        for (int ks = 0; ks < kBK; ks += 4) {
            double a[4], b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = As[ks + tg][32 * wr + 8 * q + g];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = Bs[ks + tg][32 * wc + 8 * q + g];
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) mma_f64(acc[x][y][0], acc[x][y][1], a[x], b[y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int k = k0 + 32 * wc + 8 * y + 2 * tg + i;
            if (k >= kept) continue;
            OutT *dst = out_cols ? out_cols[k] : out + (long)k * ldo;
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const long row = i0 + 32 * wr + 8 * x + g;
                if (row < n_valid) dst[row] = (OutT)acc[x][y][i];
            }
        }
}

// ---------------------------------------------------------------------------
template <class T>
__global__ void k_store(const typename Store<T>::C *src, long n_pad, T *dst) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride)
        dst[i] = Store<T>::from_c(src[i]);
}
template <class T>
__global__ void k_load(const T *src, long n, typename Store<T>::C *dst) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = Store<T>::to_c(src[i]);
}

// Smoothed random vector: s_i = 2u_i + u_{i+1} + u_{i-1} (cyclic), with the
// reference's boundary stencil (trl_smooth_rr, SRC/trlcore.c:1534-1575):
// s_0 uses u_2 and s_{n-1} uses the already smoothed s_1.
__device__ inline double smooth_at(uint64_t seed, long n, long i) {
    auto u = [&](long k) { return uniform01(seed, (uint64_t)k); };
    if (n < 3) return u(i);
    if (i == 0) return 2.0 * u(0) + u(2) + u(n - 1);
    if (i == n - 1) {
        double s1 = 2.0 * u(1) + u(2) + u(0);
        return 2.0 * u(n - 1) + s1 + u(n - 2);
    }
    return 2.0 * u(i) + u(i + 1) + u(i - 1);
}
__global__ void k_random_real(double *dst, long n, long n_pad, uint64_t seed) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride)
        dst[i] = i < n ? smooth_at(seed, n, i) : 0.0;
}
__global__ void k_random_cplx(zd *dst, long n, long n_pad, uint64_t seed) {
    const long stride = (long)gridDim.x * blockDim.x;
    const uint64_t seed_im = seed ^ 0x5DEECE66Dull;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride)
        dst[i] = i < n ? zd{smooth_at(seed, n, i), smooth_at(seed_im, n, i)} : zd{0.0, 0.0};
}

int elementwise_blocks(long n) {
    long b = (n + kThreads - 1) / kThreads;
    return (int)std::max<long>(1, std::min<long>(b, (long)num_sms() * 8));
}

}  // namespace

int stream_blocks(long n_pad, int rows_per_group) {
    long need = (n_pad + (long)kThreads * rows_per_group - 1) / ((long)kThreads * rows_per_group);
    const long cap = (long)num_sms() * 4;
    const long fill = (long)num_sms() * 2;
    if (need < fill) {
        // Short vectors: smaller blocks (down to one warp-row of
        // 32 * rows_per_group rows) so that every SM has work in flight.
        const long min_rows = 32L * rows_per_group;
        need = std::min(fill, (n_pad + min_rows - 1) / min_rows);
    }
    return (int)std::max<long>(1, std::min(need, cap));
}

template <class C>
void launch_dot(const C *x, const C *y, long n_pad, double *out, Scratch &s, cudaStream_t st) {
    int nb = std::min(stream_blocks(n_pad, 1), s.max_blocks);
    k_dot<C><<<nb, kThreads, 0, st>>>(x, y, n_pad, reinterpret_cast<double *>(s.partials),
                                      s.tickets + kTicketDot, out);
}

template <class T>
void launch_project(T *const *cols, int m, long n_pad, const typename Store<T>::C *r,
                    Recur<typename Store<T>::C> rec, typename Store<T>::C *h, double *out2,
                    Scratch &s, cudaStream_t st, int form_req) {
    using C = typename Store<T>::C;
    constexpr int R = Store<T>::R;
    // The staged form runs one block per SM (its ring fills shared memory).
    // The staged form needs 192 KB of dynamic shared memory per block; a
    // device that does not grant it runs the default register form.
    const auto staged_kern = k_project_async<T, kAsyncWarps, kAsyncCols, kAsyncStages>;
    constexpr size_t staged_smem = async_smem<kAsyncWarps, kAsyncCols, kAsyncStages>();
    bool staged = false;
    if (form_req == kProjectAsync) {
        staged = cudaFuncSetAttribute(staged_kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_smem) ==
                 cudaSuccess;
        if (!staged) {
            cudaGetLastError();
            form_req = kProjectDefault;
        }
    }
    int nb = std::min(staged ? num_sms() : stream_blocks(n_pad, R), s.max_blocks);
    long per = (n_pad + nb - 1) / nb;
    long chunk = (per + 32 * R - 1) / (32 * R) * (32 * R);
    nb = (int)((n_pad + chunk - 1) / chunk);
    C *part = reinterpret_cast<C *>(s.partials);
    double *part_r2 = reinterpret_cast<double *>(part + (long)nb * m);
    auto args = [&](auto kern) {
        kern<<<nb, kThreads, 0, st>>>(cols, m, n_pad, chunk, r, rec, part, part_r2, s.tickets + kTicketProject, h,
                                      out2);
    };
    if (staged) {
        staged_kern<<<nb, kAsyncWarps * 32, staged_smem, st>>>(cols, m, n_pad, chunk, r, rec, part, part_r2,
                                                              s.tickets + kTicketProject, h, out2);
        return;
    }
    if constexpr (std::is_same<C, double>::value) {
        // Forms (kProject*): 16 columns per warp keep one accumulator per
        // column for 128 columns per sweep (2 blocks/SM); 12 and 8 trade a
        // second sweep for 3-4 resident blocks; 16 with the pointer table in
        // shared memory frees registers for a third block.  The caller's
        // choice (the operator's autotuned form), else TRLX_PROJECT_CPW
        // (8, 12, 16), else 16.
        static const int form_env = [] {
            const char *e = std::getenv("TRLX_PROJECT_CPW");
            int v = e ? std::atoi(e) : 16;
            return v == 8 ? kProject8 : (v == 12 ? kProject12 : kProject16);
        }();
        const int form = (form_req >= kProject8 && form_req <= kProject16Shared) ? form_req : form_env;
        if (form == kProject8)
            args(k_project<T, 8>);
        else if (form == kProject12)
            args(k_project<T, 12>);
        else if (form == kProject16Shared)
            args(k_project<T, 16, true>);
        else
            args(k_project<T, 16>);
    } else {
        // Complex storage: 8 columns per warp, the pointer table in
        // registers (default) or in shared memory (kProject16Shared, three
        // blocks per SM).
        if (form_req == kProject16Shared)
            args(k_project<T, proj_cpw<T>(), true>);
        else
            args(k_project<T, proj_cpw<T>()>);
    }
}

template <class T>
void launch_update(T *const *cols, int m, long n_pad, const typename Store<T>::C *r,
                   Recur<typename Store<T>::C> rec, const typename Store<T>::C *h,
                   typename Store<T>::C *r_out, double *out_r2, Scratch &s, cudaStream_t st) {
    using C = typename Store<T>::C;
    constexpr int R = Store<T>::R;
    int nb = std::min(stream_blocks(n_pad, R), s.max_blocks);
    size_t smem = (sizeof(C) + sizeof(T *)) * (size_t)std::max(m, 1);
    // Short vectors (at most one row tile per thread at this grid) with
    // enough columns: split the columns across the warps of a block.
    const bool split = m >= 16 && n_pad <= (long)nb * kThreads * R;
    if (split) {
        const int nt = (int)std::min<long>((n_pad + 32L * R - 1) / (32L * R), s.max_blocks);
        if (smem > 40 * 1024)
            cudaFuncSetAttribute(k_update_split<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_update_split<T><<<nt, kThreads, smem, st>>>(cols, m, n_pad, r, rec, h, r_out,
                                                       reinterpret_cast<double *>(s.partials),
                                                       s.tickets + kTicketUpdate, out_r2);
        return;
    }
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_update<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_update<T><<<nb, kThreads, smem, st>>>(cols, m, n_pad, r, rec, h, r_out,
                                             reinterpret_cast<double *>(s.partials),
                                             s.tickets + kTicketUpdate, out_r2);
}

template <class T>
void launch_normalize(typename Store<T>::C *r, long n_pad, const double *r2, double fixed,
                      typename Store<T>::C *q, T *vcol, cudaStream_t st) {
    k_normalize<T><<<elementwise_blocks(n_pad), kThreads, 0, st>>>(r, n_pad, r2, fixed, q, vcol);
}

// The real scalar type of a storage or compute type (complex: its parts).
template <class X>
struct RealView {
    using type = X;
};
template <>
struct RealView<zd> {
    using type = double;
};
template <>
struct RealView<zf> {
    using type = float;
};

template <class T, class OutT>
void ritz_dispatch(T *const *in_cols, int jml, long n_pad, const double *Y, int ldy, int kept, OutT *const *out_cols,
                   OutT *out, long ldo, long n_valid, cudaStream_t st) {
    if (kept <= 0) return;
    if constexpr (!std::is_same<typename RealView<T>::type, T>::value) {
        // A complex column times a real Y is the real product of its
        // interleaved (re, im) view: 2 n_pad real rows, the same for the
        // output columns (2 ldo, 2 n_valid).
        using RT = typename RealView<T>::type;
        using RO = typename RealView<OutT>::type;
        ritz_dispatch<RT, RO>(reinterpret_cast<RT *const *>(in_cols), jml, 2 * n_pad, Y, ldy, kept,
                              reinterpret_cast<RO *const *>(out_cols), reinterpret_cast<RO *>(out), 2 * ldo,
                              2 * n_valid, st);
        return;
    } else {
        if (kept <= 32) {
            k_ritz_mma<T, OutT, 32><<<dim3((unsigned)(n_pad / MmaShape<32>::BM), 1), kThreads, 0, st>>>(
                in_cols, jml, Y, ldy, kept, out_cols, out, ldo, n_valid);
        } else {
            dim3 grid((unsigned)(n_pad / MmaShape<64>::BM), (unsigned)((kept + 63) / 64));
            k_ritz_mma<T, OutT, 64><<<grid, kThreads, 0, st>>>(in_cols, jml, Y, ldy, kept, out_cols, out, ldo,
                                                                n_valid);
        }
    }
}

template <class T>
void launch_ritz(T *const *in_cols, int jml, long n_pad, const double *Y, int ldy, int kept, T *const *out_cols,
                 cudaStream_t st) {
    ritz_dispatch<T, T>(in_cols, jml, n_pad, Y, ldy, kept, out_cols, nullptr, 0, n_pad, st);
}

template <class T>
void launch_ritz_out(T *const *in_cols, int jml, long n_pad, const double *Y, int ldy, int kept,
                     typename Store<T>::C *out, long ldo, long n, cudaStream_t st) {
    using C = typename Store<T>::C;
    ritz_dispatch<T, C>(in_cols, jml, n_pad, Y, ldy, kept, nullptr, out, ldo, n, st);
}

template <class T>
void launch_store(const typename Store<T>::C *src, long n_pad, T *dst, cudaStream_t st) {
    k_store<T><<<elementwise_blocks(n_pad), kThreads, 0, st>>>(src, n_pad, dst);
}
template <class T>
void launch_load(const T *src, long n, typename Store<T>::C *dst, cudaStream_t st) {
    k_load<T><<<elementwise_blocks(n), kThreads, 0, st>>>(src, n, dst);
}

template <>
void launch_random<double>(double *dst, long n, long n_pad, uint64_t seed, cudaStream_t st) {
    k_random_real<<<elementwise_blocks(n_pad), kThreads, 0, st>>>(dst, n, n_pad, seed);
}
template <>
void launch_random<zd>(zd *dst, long n, long n_pad, uint64_t seed, cudaStream_t st) {
    k_random_cplx<<<elementwise_blocks(n_pad), kThreads, 0, st>>>(dst, n, n_pad, seed);
}

// out = a * (ay - c * y) + b * yp  (one step of a scaled Chebyshev filter;
// out may alias yp).
__global__ void k_cheb(const double *__restrict__ ay, const double *__restrict__ y, const double *yp, long n_pad,
                       double a, double c, double b, double *out) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
        const double prev = yp ? yp[i] : 0.0;
        out[i] = a * (ay[i] - c * y[i]) + b * prev;
    }
}

__global__ void __launch_bounds__(kThreads) k_sumsq(const double *__restrict__ v, long n, double *out) {
    __shared__ double red[32];
    double s = 0.0;
    for (long i = threadIdx.x; i < n; i += kThreads) s = fma(v[i], v[i], s);
    s = block_sum(s, red);
    if (threadIdx.x == 0) *out = s;
}

void launch_sumsq(const double *v, long n, double *out, cudaStream_t st) {
    k_sumsq<<<1, kThreads, 0, st>>>(v, n, out);
}

void launch_cheb(const double *ay, const double *y, const double *yp, long n_pad, double a, double c, double b,
                 double *out, cudaStream_t st) {
    k_cheb<<<elementwise_blocks(n_pad), kThreads, 0, st>>>(ay, y, yp, n_pad, a, c, b, out);
}
// Complex vectors with real coefficients: the same recurrence on the
// interleaved real and imaginary parts.
void launch_cheb(const zd *ay, const zd *y, const zd *yp, long n_pad, double a, double c, double b, zd *out,
                 cudaStream_t st) {
    k_cheb<<<elementwise_blocks(2 * n_pad), kThreads, 0, st>>>(
        reinterpret_cast<const double *>(ay), reinterpret_cast<const double *>(y),
        reinterpret_cast<const double *>(yp), 2 * n_pad, a, c, b, reinterpret_cast<double *>(out));
}

#define TRLB_INST(T)                                                                              \
    template void launch_project<T>(T *const *, int, long, const Store<T>::C *, Recur<Store<T>::C>, \
                                    Store<T>::C *, double *, Scratch &, cudaStream_t, int);       \
    template void launch_update<T>(T *const *, int, long, const Store<T>::C *, Recur<Store<T>::C>,  \
                                   const Store<T>::C *, Store<T>::C *, double *, Scratch &,        \
                                   cudaStream_t);                                                 \
    template void launch_normalize<T>(Store<T>::C *, long, const double *, double, Store<T>::C *,  \
                                      T *, cudaStream_t);                                         \
    template void launch_ritz<T>(T *const *, int, long, const double *, int, int, T *const *,     \
                                 cudaStream_t);                                                   \
    template void launch_ritz_out<T>(T *const *, int, long, const double *, int, int,             \
                                     Store<T>::C *, long, long, cudaStream_t);                    \
    template void launch_store<T>(const Store<T>::C *, long, T *, cudaStream_t);                  \
    template void launch_load<T>(const T *, long, Store<T>::C *, cudaStream_t);

TRLB_INST(double)
TRLB_INST(float)
TRLB_INST(zd)
TRLB_INST(zf)
template void launch_dot<double>(const double *, const double *, long, double *, Scratch &,
                                 cudaStream_t);
template void launch_dot<zd>(const zd *, const zd *, long, double *, Scratch &, cudaStream_t);

}  // namespace trlb

// Kernel-level entry point for the Gram-Schmidt projection of the reference:
// trl_g_dot_ (SRC/trl_comm_none.c:238-329) computes wrk = [v1 v2]^T rr over
// two blocks of basis columns, ztrl_g_dot_ (SRC/ztrl_comm_none.c:16-130) the
// conjugate-transposed product.  The engine's own projection kernel assumes
// its padded, 16-byte aligned column pool; this one accepts any device
// pointers and leading dimensions (scalar, coalesced loads, bounds checked).
//
// Reduction scratch (one partial per block and column plus a ticket) comes
// from a per-thread cached device buffer.
#include <algorithm>
#include <cstdio>

#include "../../../include/trlx.h"
#include "common.cuh"
#include "gdot.h"

namespace trlb {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kCols = 8;  // columns per warp group

template <class C>
__device__ __forceinline__ C load_elem(const C *p) {
    return *p;
}
__device__ __forceinline__ zd load_elem(const zd *p) {
    const double *q = reinterpret_cast<const double *>(p);
    return zd{q[0], q[1]};
}

}  // namespace

// Block b owns rows [b*chunk, (b+1)*chunk); column groups of kCols are
// spread over the warps, and when there are fewer groups than warps the
// warps of a group split the rows.  Partial sums are combined in a fixed
// order; the last block to finish writes wrk.
template <class C>
__global__ void __launch_bounds__(kThreads)
    k_gdot(int n, long chunk, const C *v1, long ld1, int m1, const C *v2, long ld2, int m2,
           const C *__restrict__ rr, C *part, unsigned *ticket, C *wrk) {
    __shared__ C red[kWarps][kCols];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = m1 + m2;
    const long row0 = (long)blockIdx.x * chunk;
    const long row1 = min((long)n, row0 + chunk);
    const int ngroups = (m + kCols - 1) / kCols;
    for (int g0 = 0; g0 < ngroups; g0 += kWarps) {
        const int G = min(kWarps, ngroups - g0);
        const int wpg = kWarps / G;
        const int grp = warp / wpg, slice = warp - grp * wpg;
        const bool active = grp < G;
        const int cb = (g0 + grp) * kCols;
        const C *p[kCols];
#pragma unroll
        for (int k = 0; k < kCols; ++k) {
            const int c = cb + k;
            p[k] = (!active || c >= m) ? nullptr : (c < m1 ? v1 + (long)c * ld1 : v2 + (long)(c - m1) * ld2);
        }
        C acc[kCols];
#pragma unroll
        for (int k = 0; k < kCols; ++k) acc[k] = czero(C());
        if (active) {
            for (long i = row0 + slice * 32 + lane; i < row1; i += (long)wpg * 32) {
                const C r = load_elem(rr + i);
#pragma unroll
                for (int k = 0; k < kCols; ++k)
                    if (p[k]) fma_conj(acc[k], load_elem(p[k] + i), r);
            }
        }
#pragma unroll
        for (int k = 0; k < kCols; ++k) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[k] = acc[k] + shfl_down(acc[k], o);
            if (lane == 0) red[warp][k] = acc[k];
        }
        __syncthreads();
        if (threadIdx.x < G * kCols) {
            const int gg = threadIdx.x / kCols, k = threadIdx.x - gg * kCols;
            const int c = (g0 + gg) * kCols + k;
            if (c < m) {
                C s = czero(C());
                for (int sl = 0; sl < wpg; ++sl) s = s + red[gg * wpg + sl][k];
                part[(long)blockIdx.x * m + c] = s;
            }
        }
        __syncthreads();
    }
    if (last_block_arrived(ticket)) {
        __shared__ C red_cols[kThreads];
        reduce_columns(part, (int)gridDim.x, m, wrk, red_cols);
        if (threadIdx.x == 0) *ticket = 0;
    }
}

int gdot_grid(int n, int max_blocks, long *chunk) {
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    long want = std::max<long>(1, std::min<long>((long)sms * 4, ((long)n + 2047) / 2048));
    want = std::min<long>(want, max_blocks);
    long per = ((long)n + want - 1) / want;
    *chunk = std::max<long>(32, (per + 31) / 32 * 32);
    return (int)(((long)n + *chunk - 1) / *chunk);
}

template <class C>
int launch_gdot(int nrow, const C *v1, int ld1, int m1, const C *v2, int ld2, int m2, const C *rr, C *wrk,
                C *part, unsigned *ticket, int nblocks, long chunk, cudaStream_t st) {
    k_gdot<C><<<nblocks, kThreads, 0, st>>>(nrow, chunk, v1, ld1, m1, v2, ld2, m2, rr, part, ticket, wrk);
    return cudaGetLastError() == cudaSuccess ? 0 : -1001;
}

template int launch_gdot<double>(int, const double *, int, int, const double *, int, int, const double *, double *,
                                 double *, unsigned *, int, long, cudaStream_t);
template int launch_gdot<zd>(int, const zd *, int, int, const zd *, int, int, const zd *, zd *, zd *, unsigned *, int,
                             long, cudaStream_t);

namespace {

// Per-thread scratch for the allocating entry points.
struct GdotScratch {
    void *buf = nullptr;
    size_t bytes = 0;
    int device = -1;
    ~GdotScratch() { cudaFree(buf); }
};

template <class C>
int gdot_entry(int nrow, const C *v1, int ld1, int m1, const C *v2, int ld2, int m2, const C *rr, C *wrk,
               void *stream) {
    const int m = m1 + m2;
    if (m1 < 0 || m2 < 0 || nrow < 0) return -1;
    if (m <= 0) return 0;
    if (ld1 < nrow || ld2 < nrow) {
        std::fprintf(stderr, "trlx_g_dot: incorrect array sizes\n");
        return -201;
    }
    if (!rr || !wrk || (m1 > 0 && !v1) || (m2 > 0 && !v2)) return -1;
    // No local rows (a rank that owns none): the partial products are zero.
    if (nrow == 0)
        return cudaMemsetAsync(wrk, 0, sizeof(C) * m, static_cast<cudaStream_t>(stream)) == cudaSuccess ? 0 : -1001;
    static thread_local GdotScratch sc;
    int dev = 0;
    cudaGetDevice(&dev);
    if (sc.device != dev) {
        cudaFree(sc.buf);
        sc.buf = nullptr;
        sc.bytes = 0;
        sc.device = dev;
    }
    long chunk = 0;
    const int nb = gdot_grid(nrow, 148 * 4, &chunk);
    const size_t need = 256 + sizeof(C) * (size_t)nb * m;
    if (sc.bytes < need) {
        cudaFree(sc.buf);
        sc.buf = nullptr;
        sc.bytes = 0;
        if (cudaMalloc(&sc.buf, need) != cudaSuccess) {
            cudaGetLastError();
            return -5;
        }
        cudaMemset(sc.buf, 0, 256);
        sc.bytes = need;
    }
    unsigned *ticket = static_cast<unsigned *>(sc.buf);
    C *part = reinterpret_cast<C *>(static_cast<char *>(sc.buf) + 256);
    return launch_gdot<C>(nrow, v1, ld1, m1, v2, ld2, m2, rr, wrk, part, ticket, nb, chunk,
                          static_cast<cudaStream_t>(stream));
}

}  // namespace

}  // namespace trlb

extern "C" int trlx_g_dot(int nrow, const double *v1, int ld1, int m1, const double *v2, int ld2, int m2,
                          const double *rr, double *wrk, void *stream) {
    return trlb::gdot_entry<double>(nrow, v1, ld1, m1, v2, ld2, m2, rr, wrk, stream);
}

extern "C" int trlx_zg_dot(int nrow, const trl_dcomplex *v1, int ld1, int m1, const trl_dcomplex *v2, int ld2,
                           int m2, const trl_dcomplex *rr, trl_dcomplex *wrk, void *stream) {
    using trlb::zd;
    return trlb::gdot_entry<zd>(nrow, reinterpret_cast<const zd *>(v1), ld1, m1, reinterpret_cast<const zd *>(v2),
                                ld2, m2, reinterpret_cast<const zd *>(rr), reinterpret_cast<zd *>(wrk), stream);
}

// One cooperative kernel for a run of speculative Lanczos steps on short
// vectors (built-in CSR operator, FP64 / c128 basis).
//
// Each block owns a contiguous chunk of rows for the whole run.  A step is
// five phases separated by grid-wide barriers:
//   A  y = A q_{j-1} on the block's rows (8 lanes per row, y kept in shared
//      memory), partial alpha = Re(q_{j-1}^H y);
//   B  alpha = sum of the partials (fixed order), r = y - alpha q_{j-1} -
//      beta q_{j-2} (beta = sqrt of the previous step's |r|^2, or the host's
//      value for the first step), partial |r|^2 and partial h_c = V_c^H r for
//      every basis column c < j;
//   C  block b reduces columns c = b, b + G, ... (and |r|^2) in block order;
//   D  r <- r - V h on the block's rows, partial |r|^2;
//   E  |r|^2 summed, q_j = r / |r| written to column j.
// The per-step log (alpha, |r|^2 before and after the pass, |h|^2) is the
// one the host replays to accept or discard steps, exactly as for the
// discrete kernels; only the summation order of the reductions differs.
// Basis columns written by other blocks are read through L2 (ld.global.cg),
// never through the non-coherent read-only path.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdlib>

#include "coop.h"
#include "spmv.h"

namespace trlb {

namespace {

namespace cg = cooperative_groups;

constexpr int kThreads = 256;
constexpr int kGroup = 8;     // lanes per CSR row
constexpr int kPassRows = 64; // rows per pass of the update phase
constexpr int kSlices = kThreads / kPassRows;

__device__ __forceinline__ double mulx(double a, double x) { return a * x; }
__device__ __forceinline__ zd mulx(zd a, zd x) { return zd{a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x}; }
__device__ __forceinline__ double shfl_x(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ zd shfl_x(zd v, int o) {
    return zd{__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o)};
}
__device__ __forceinline__ double ldgv(const double *p) { return __ldg(p); }
__device__ __forceinline__ zd ldgv(const zd *p) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return zd{v.x, v.y};
}
__device__ __forceinline__ double as_c(double v, double) { return v; }
__device__ __forceinline__ zd as_c(double v, zd) { return zd{v, 0.0}; }

// Total of nb values of part (stride `stride`) by the whole block in a fixed
// order; returned to every thread.
template <class C>
__device__ __forceinline__ C block_total(const C *part, int nb, long stride, C *red, C *bcast) {
    C s = czero(C());
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s = s + ldcg(part + (long)b * stride);
    s = block_sum(s, red);
    if (threadIdx.x == 0) *bcast = s;
    __syncthreads();
    const C out = *bcast;
    __syncthreads();
    return out;
}

template <class C>
__global__ void __launch_bounds__(kThreads) k_spec_coop(CoopArgs<C> a) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *rs = reinterpret_cast<C *>(smem_raw);        // the block's rows of y, then r
    C *hs = rs + a.chunk;                           // h (maxcols)
    C *tmp = hs + a.maxcols;                        // [kSlices][kPassRows]
    __shared__ C red[32];
    __shared__ C bc;
    __shared__ double redd[32];
    __shared__ double bcd;
    const int G = gridDim.x, bid = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const long r0 = (long)bid * a.chunk;
    const long r1 = min(a.n_pad, r0 + a.chunk);
    const int rows = (int)max(0L, r1 - r0);
    // Scalar partials live after the column partials ((maxcols + 1) * G).
    double *partd = reinterpret_cast<double *>(a.part + (long)(a.maxcols + 1) * G);
    for (int s = 1; s <= a.S; ++s) {
        const int j = a.j0 + s;
        const C *qa = a.cols[j - 1];
        const C *qb = a.cols[j - 2];
        C *q = a.cols[j];
        double *lg = a.log + 4 * s;
        // ---- A: y = A qa on own rows, partial alpha --------------------------
        double aacc = 0.0;
        {
            const int g = tid & (kGroup - 1);
            for (int i0 = 0; i0 < rows; i0 += kThreads / kGroup) {
                const int i = i0 + tid / kGroup;
                const long row = r0 + i;
                C acc = czero(C());
                if (i < rows && row < a.nrow) {
                    const long b = a.rp[row], e = a.rp[row + 1];
                    for (long k = b + g; k < e; k += kGroup) acc = acc + mulx(ldgv(a.va + k), ldcg(qa + a.ci[k]));
                }
#pragma unroll
                for (int o = kGroup / 2; o > 0; o >>= 1) acc = acc + shfl_x(acc, o);
                if (g == 0 && i < rows) {
                    rs[i] = acc;
                    C t = czero(C());
                    fma_conj(t, ldcg(qa + row), acc);
                    aacc += real_part(t);
                }
            }
        }
        {
            const double sa = block_sum(aacc, redd);
            if (tid == 0) partd[bid] = sa;
        }
        grid.sync();
        // ---- B: recurrence, |r|^2 and h partials --------------------------
        const double alpha = block_total(partd, G, 1, redd, &bcd);
        const double beta = s == 1 ? a.beta0 : sqrt(ldcg(a.log + 4 * (s - 1) + 3));
        double r2acc = 0.0;
        for (int i = tid; i < rows; i += kThreads) {
            const long row = r0 + i;
            const C v = rs[i] - alpha * ldcg(qa + row) - beta * ldcg(qb + row);
            rs[i] = v;
            r2acc += abs2(v);
        }
        __syncthreads();
        // Four columns per warp and sweep: four independent loads in flight.
        for (int c0 = warp * 4; c0 < j; c0 += kThreads / 32 * 4) {
            const C *v[4];
            C acc[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] = c0 + u < j ? a.cols[c0 + u] + r0 : nullptr;
                acc[u] = czero(C());
            }
            for (int i = lane; i < rows; i += 32) {
                const C ri = rs[i];
                C x[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) x[u] = v[u] ? ldcg(v[u] + i) : czero(C());
#pragma unroll
                for (int u = 0; u < 4; ++u) fma_conj(acc[u], x[u], ri);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[u] = acc[u] + shfl_down(acc[u], o);
                if (lane == 0 && v[u]) a.part[(long)(c0 + u) * G + bid] = acc[u];
            }
        }
        {
            const double sr = block_sum(r2acc, redd);
            if (tid == 0) a.part[(long)j * G + bid] = as_c(sr, C());
        }
        grid.sync();
        // ---- C: column reductions (and |r|^2 before the pass) --------------
        for (int c = bid; c <= j; c += G) {
            const C t = block_total(a.part + (long)c * G, G, 1, red, &bc);
            if (tid == 0) {
                if (c < j)
                    a.h[c] = t;
                else
                    lg[1] = real_part(t);
            }
        }
        grid.sync();
        // ---- D: r <- r - V h on own rows ----------------------------------
        for (int c = tid; c < j; c += kThreads) hs[c] = ldcg(a.h + c);
        __syncthreads();
        double r2post = 0.0;
        {
            const int sl = tid / kPassRows, ri = tid % kPassRows;
            for (int p0 = 0; p0 < rows; p0 += kPassRows) {
                const int i = p0 + ri;
                C acc = czero(C());
                if (i < rows) {
                    int c = sl;
                    for (; c + 3 * kSlices < j; c += 4 * kSlices) {
                        const C x0 = ldcg(a.cols[c] + r0 + i), x1 = ldcg(a.cols[c + kSlices] + r0 + i);
                        const C x2 = ldcg(a.cols[c + 2 * kSlices] + r0 + i), x3 = ldcg(a.cols[c + 3 * kSlices] + r0 + i);
                        fms(acc, x0, hs[c]);
                        fms(acc, x1, hs[c + kSlices]);
                        fms(acc, x2, hs[c + 2 * kSlices]);
                        fms(acc, x3, hs[c + 3 * kSlices]);
                    }
                    for (; c < j; c += kSlices) fms(acc, ldcg(a.cols[c] + r0 + i), hs[c]);
                }
                tmp[sl * kPassRows + ri] = acc;
                __syncthreads();
                if (sl == 0 && i < rows) {
                    C v = rs[i];
                    for (int k = 0; k < kSlices; ++k) v = v + tmp[k * kPassRows + ri];
                    rs[i] = v;
                    r2post += abs2(v);
                }
                __syncthreads();
            }
        }
        {
            const double sp = block_sum(r2post, redd);
            if (tid == 0) partd[bid] = sp;
        }
        if (bid == 0) {
            double h2 = 0.0;
            for (int c = tid; c < j; c += kThreads) h2 += abs2(hs[c]);
            h2 = block_sum(h2, redd);
            if (tid == 0) {
                lg[0] = alpha;
                lg[2] = h2;
            }
        }
        grid.sync();
        // ---- E: normalise into column j -----------------------------------
        const double r2 = block_total(partd, G, 1, redd, &bcd);
        const double sc = 1.0 / sqrt(r2);
        for (int i = tid; i < rows; i += kThreads) q[r0 + i] = rs[i] * sc;
        if (bid == 0 && tid == 0) lg[3] = r2;
        grid.sync();
    }
}

int num_sms_coop() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

}  // namespace

template <class C>
int launch_spec_coop(const trlx_operator *A, C *const *cols, long n_pad, int maxcols, int j0, int S, double beta0,
                     double *log, C *part, long part_elems, C *h, cudaStream_t st) {
    if (!A || (A->kind != 0 && A->kind != 2) || S < 1) return -1;
    int dev = 0, coop = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop) return -1;
    // Blocks: enough rows per block to keep the chunk a multiple of 64 and
    // at most two blocks per SM (all must be resident).
    const int sms = num_sms_coop();
    // Smallest chunk (rows per block); TRLX_COOP_ROWS overrides (tuning).
    static const long min_rows = [] {
        const char *e = std::getenv("TRLX_COOP_ROWS");
        const long v = e ? std::atol(e) : kPassRows;
        return v >= kPassRows ? v : (long)kPassRows;
    }();
    long G = std::min<long>(2L * sms, (n_pad + min_rows - 1) / min_rows);
    long chunk = (n_pad + G - 1) / G;
    chunk = (chunk + kPassRows - 1) / kPassRows * kPassRows;
    G = (n_pad + chunk - 1) / chunk;
    const size_t smem = sizeof(C) * ((size_t)chunk + maxcols + kSlices * kPassRows);
    if (smem > 200 * 1024) return -1;
    static const void *attr_set[2] = {nullptr, nullptr};
    const void *fn = reinterpret_cast<const void *>(&k_spec_coop<C>);
    const int which = sizeof(C) == sizeof(double) ? 0 : 1;
    if (attr_set[which] != fn) {
        cudaFuncSetAttribute(k_spec_coop<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set[which] = fn;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spec_coop<C>, kThreads, smem) != cudaSuccess ||
        (long)per_sm * sms < G)
        return -1;
    if ((long)(maxcols + 2) * G > part_elems) return -1;
    CoopArgs<C> a;
    a.nrow = A->nrow;
    a.n_pad = n_pad;
    a.chunk = chunk;
    a.maxcols = maxcols;
    a.rp = A->row_ptr;
    a.ci = A->col;
    a.va = static_cast<const C *>(A->val);
    a.cols = cols;
    a.j0 = j0;
    a.S = S;
    a.beta0 = beta0;
    a.log = log;
    a.part = part;
    a.h = h;
    void *args[] = {&a};
    const cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3((unsigned)G), dim3(kThreads), args, smem, st);
    return e == cudaSuccess ? 0 : -1001;
}

template int launch_spec_coop<double>(const trlx_operator *, double *const *, long, int, int, int, double, double *,
                                      double *, long, double *, cudaStream_t);
template int launch_spec_coop<zd>(const trlx_operator *, zd *const *, long, int, int, int, double, double *, zd *,
                                  long, zd *, cudaStream_t);

}  // namespace trlb

// Sparse matrix-vector kernels for the built-in operators.
//
// CSR: one row per group of 8 lanes (rows of the configured stencils have
// 5-7 entries), so each group reads its row's values and column indices
// coalesced and reduces with 3 shuffles.  SELL-C-32: one row per lane, the
// slice stored column-major (entry k of the 32 rows contiguous), so every
// value/index load of a warp is one 128/256-byte segment.  Both fuse the
// Lanczos alpha = x^H y into the same pass.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "../../../include/trlx.h"
#include "spmv.h"
#include "../host/comm.h"
#include "../host/hostcopy.h"

namespace trlb {

namespace {

constexpr int kThreads = 256;
constexpr int kGroup = 8;
constexpr int kTicketSpmv = 3;

template <class V>
__device__ __forceinline__ V ld_val(const V *p) {
    return *p;
}
__device__ __forceinline__ double mulx(double a, double x) { return a * x; }
__device__ __forceinline__ zd mulx(zd a, zd x) { return zd{a.x * x.x - a.y * x.y, a.x * x.y + a.y * x.x}; }
__device__ __forceinline__ double shfl_xor(double v, int o) { return __shfl_xor_sync(0xffffffffu, v, o); }
__device__ __forceinline__ zd shfl_xor(zd v, int o) {
    return zd{__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o)};
}
__device__ __forceinline__ double ldg_c(const double *p) { return __ldg(p); }
__device__ __forceinline__ zd ldg_c(const zd *p) {
    double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    return zd{v.x, v.y};
}

template <class V>
__global__ void __launch_bounds__(kThreads)
    k_csr(int nrow, long n_pad, const long long *__restrict__ rp, const int *__restrict__ ci,
          const V *__restrict__ va, const V *__restrict__ x, V *__restrict__ y, double *part,
          unsigned *ticket, double *alpha_out) {
    const int g = threadIdx.x & (kGroup - 1);
    const long groups = (long)gridDim.x * (kThreads / kGroup);
    double aacc = 0.0;
    // Rows are visited in rounds so that all lanes of a warp stay converged
    // for the shuffles (bounds are uniform per round across the grid).
    const long rounds = (n_pad + groups - 1) / groups;
    for (long rd = 0; rd < rounds; ++rd) {
        const long row = rd * groups + (long)blockIdx.x * (kThreads / kGroup) + (threadIdx.x / kGroup);
        V acc = czero(V());
        if (row < nrow) {
            const long b = rp[row], e = rp[row + 1];
            for (long k = b + g; k < e; k += kGroup) acc = acc + mulx(ld_val(va + k), ldg_c(x + ci[k]));
        }
#pragma unroll
        for (int o = kGroup / 2; o > 0; o >>= 1) acc = acc + shfl_xor(acc, o);
        if (g == 0 && row < n_pad) {
            y[row] = acc;  // rows in [nrow, n_pad) get zero
            if (alpha_out) {
                V t = czero(V());
                fma_conj(t, ldg_c(x + row), acc);
                aacc += real_part(t);
            }
        }
    }
    if (!alpha_out) return;
    __shared__ double red[32];
    double s = block_sum(aacc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part, gridDim.x, red);
        if (threadIdx.x == 0) {
            *alpha_out = tot;
            *ticket = 0;
        }
    }
}

// CSR in row tiles of kThreads rows: the tile's entries are processed in
// chunks of kChunk; all threads compute val*x[col] products with coalesced
// loads (kChunk/kThreads independent loads in flight per thread) into shared
// memory, then each thread sums its own row's products in index order.
constexpr int kChunk = 2048;

template <class V>
__global__ void __launch_bounds__(kThreads)
    k_csr_stream(int nrow, long n_pad, const long long *__restrict__ rp, const int *__restrict__ ci,
                 const V *__restrict__ va, const V *__restrict__ x, V *__restrict__ y, double *part,
                 unsigned *ticket, double *alpha_out) {
    __shared__ V prod[kChunk];
    __shared__ long long rps[kThreads + 1];
    const int t = threadIdx.x;
    double aacc = 0.0;
    const long ntiles = n_pad / kThreads;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long r0 = tile * kThreads;
        for (int k = t; k <= kThreads; k += kThreads) rps[k] = rp[(r0 + k < nrow) ? (r0 + k) : (long)nrow];
        __syncthreads();
        const long long eb = rps[0], ee = rps[kThreads];
        const long long mb = rps[t], me = rps[t + 1];
        V acc = czero(V());
        for (long long c0 = eb; c0 < ee; c0 += kChunk) {
            const long long c1 = min(ee, c0 + (long long)kChunk);
            for (long long e = c0 + t; e < c1; e += kThreads) prod[e - c0] = mulx(ld_val(va + e), ldg_c(x + ci[e]));
            __syncthreads();
            const long long lo = max(mb, c0), hi = min(me, c1);
            for (long long e = lo; e < hi; ++e) acc = acc + prod[e - c0];
            __syncthreads();
        }
        const long row = r0 + t;
        y[row] = acc;  // rows in [nrow, n_pad) have no entries: zero
        if (alpha_out) {
            V tt = czero(V());
            fma_conj(tt, ldg_c(x + row), acc);
            aacc += real_part(tt);
        }
    }
    if (!alpha_out) return;
    __shared__ double red[32];
    double s = block_sum(aacc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part, gridDim.x, red);
        if (threadIdx.x == 0) {
            *alpha_out = tot;
            *ticket = 0;
        }
    }
}

// acc + a * x (real: one FMA; complex: four).
__device__ __forceinline__ double mac(double acc, double a, double x) { return fma(a, x, acc); }
__device__ __forceinline__ zd mac(zd acc, zd a, zd x) {
    return zd{fma(a.x, x.x, fma(-a.y, x.y, acc.x)), fma(a.x, x.y, fma(a.y, x.x, acc.y))};
}
// aacc + Re(conj(x) * y).
__device__ __forceinline__ double alpha_add(double aacc, double x, double y) { return fma(x, y, aacc); }
__device__ __forceinline__ double alpha_add(double aacc, zd x, zd y) { return fma(x.x, y.x, fma(x.y, y.y, aacc)); }

// Eight blocks per SM (32 registers): the product is latency-bound, and the
// full 64 warps beat the complex form's unconstrained 40 registers (6 blocks;
// a few bytes of spills outside the entry loop): 0.132 -> 0.104 ms per
// product on Peierls 2048^2, 0.314 -> 0.299 ms for the real form at 256^3.
template <class V>
__global__ void __launch_bounds__(kThreads, 8)
    k_sell(int nrow, long n_pad, int nslice, const long long *__restrict__ sp,
           const int *__restrict__ ci, const V *__restrict__ va, const int *__restrict__ perm,
           const V *__restrict__ x, V *__restrict__ y, double *part, unsigned *ticket,
           double *alpha_out) {
    const int lane = threadIdx.x & 31;
    const long warps = (long)gridDim.x * (kThreads / 32);
    double aacc = 0.0;
    for (long s = (long)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); s < nslice; s += warps) {
        const long b = sp[s];
        const int w = (int)((sp[s + 1] - b) >> 5);
        V acc = czero(V());
        const V *v = va + b + lane;
        const int *c = ci + b + lane;
#pragma unroll 4
        for (int k = 0; k < w; ++k) acc = mac(acc, ldg_c(v + (long)k * 32), ldg_c(x + __ldg(c + (long)k * 32)));
        const long srow = s * 32 + lane;
        if (srow < nrow) {
            const int row = perm ? perm[srow] : (int)srow;
            y[row] = acc;
            if (alpha_out) aacc = alpha_add(aacc, ldg_c(x + row), acc);
        }
    }
    // Zero the padding rows [nrow, n_pad).
    for (long i = nrow + (long)blockIdx.x * kThreads + threadIdx.x; i < n_pad; i += (long)gridDim.x * kThreads)
        y[i] = czero(V());
    if (!alpha_out) return;
    __shared__ double red[32];
    double s2 = block_sum(aacc, red);
    if (threadIdx.x == 0) part[blockIdx.x] = s2;
    if (last_block_arrived(ticket)) {
        const double tot = sum_partials(part, gridDim.x, red);
        if (threadIdx.x == 0) {
            *alpha_out = tot;
            *ticket = 0;
        }
    }
}

int spmv_blocks(long work_items, int per_block) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    long need = (work_items + per_block - 1) / per_block;
    return (int)std::max<long>(1, std::min<long>(need, (long)sms * 8));
}

}  // namespace

// The 256-row-tile CSR kernel needs whole tiles and pays off once every SM
// has at least two tiles; shorter vectors use the 8-lanes-per-row kernel,
// whose many small blocks hide latency better.
static bool use_row_tiles(long n_pad) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return n_pad % kThreads == 0 && n_pad / kThreads >= 2L * sms;
}

void spmv_fused_real(const trlx_operator *A, const double *x, double *y, long n_pad,
                     double *alpha_out, Scratch *s, cudaStream_t st) {
    double *part = s ? reinterpret_cast<double *>(s->partials) : nullptr;
    unsigned *tk = s ? s->tickets + kTicketSpmv : nullptr;
    if (A->kind == 0) {
        if (use_row_tiles(n_pad)) {
            int nb = spmv_blocks(n_pad, kThreads);
            if (s) nb = std::min(nb, s->max_blocks);
            k_csr_stream<double><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->row_ptr, A->col,
                                                          static_cast<const double *>(A->val), x, y, part, tk,
                                                          alpha_out);
            return;
        }
        int nb = spmv_blocks(n_pad, kThreads / kGroup);
        if (s) nb = std::min(nb, s->max_blocks);
        k_csr<double><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->row_ptr, A->col,
                                               static_cast<const double *>(A->val), x, y, part, tk,
                                               alpha_out);
    } else {
        int nb = spmv_blocks((long)A->nslice * 32, kThreads);
        if (s) nb = std::min(nb, s->max_blocks);
        k_sell<double><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->nslice, A->slice_ptr, A->col,
                                                static_cast<const double *>(A->val), A->perm, x, y, part, tk,
                                                alpha_out);
    }
}

void spmv_fused_cplx(const trlx_operator *A, const zd *x, zd *y, long n_pad, double *alpha_out,
                     Scratch *s, cudaStream_t st) {
    double *part = s ? reinterpret_cast<double *>(s->partials) : nullptr;
    unsigned *tk = s ? s->tickets + kTicketSpmv : nullptr;
    if (A->kind == 3) {
        int nb = spmv_blocks((long)A->nslice * 32, kThreads);
        if (s) nb = std::min(nb, s->max_blocks);
        k_sell<zd><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->nslice, A->slice_ptr, A->col,
                                            static_cast<const zd *>(A->val), A->perm, x, y, part, tk, alpha_out);
        return;
    }
    if (use_row_tiles(n_pad)) {
        int nb = spmv_blocks(n_pad, kThreads);
        if (s) nb = std::min(nb, s->max_blocks);
        k_csr_stream<zd><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->row_ptr, A->col,
                                                  static_cast<const zd *>(A->val), x, y, part, tk, alpha_out);
        return;
    }
    int nb = spmv_blocks(n_pad, kThreads / kGroup);
    if (s) nb = std::min(nb, s->max_blocks);
    k_csr<zd><<<nb, kThreads, 0, st>>>(A->nrow, n_pad, A->row_ptr, A->col,
                                       static_cast<const zd *>(A->val), x, y, part, tk, alpha_out);
}

void spmv_plain(const trlx_operator *A, const void *x, void *y, cudaStream_t st) {
    // n_pad == nrow: no padding rows written.
    if (A->halo) {
        const double *xe = nullptr;
        if (halo_exchange(A, static_cast<const double *>(x), st, &xe) != 0) return;
        spmv_fused_real(A, xe, static_cast<double *>(y), A->nrow, nullptr, nullptr, st);
        return;
    }
    if (op_complex(A))
        spmv_fused_cplx(A, static_cast<const zd *>(x), static_cast<zd *>(y), A->nrow, nullptr, nullptr, st);
    else
        spmv_fused_real(A, static_cast<const double *>(x), static_cast<double *>(y), A->nrow, nullptr,
                        nullptr, st);
}

double spmv_bytes(const trlx_operator *A) {
    const double vs = op_complex(A) ? 16.0 : 8.0;
    double b = (double)A->nnz * (vs + 4.0) + 2.0 * vs * A->nrow;
    if (op_sell(A))
        b += 8.0 * (A->nslice + 1) + (A->perm ? 4.0 * A->nrow : 0.0);
    else
        b += 8.0 * (A->nrow + 1.0);
    return b;
}

// ---- block-row distribution -------------------------------------------------
struct Halo {
    Comm *comm = nullptr;  // borrowed from the trlx_comm given at creation
    long long row0 = 0;    // global index of this rank's first row
    int nhalo = 0;
    long long nsend = 0;
    int *send_idx = nullptr;     // local rows other ranks need, grouped by receiver
    double *send_buf = nullptr;  // nsend values
    double *x_ext = nullptr;     // this rank's rows, then the halo
    long ext_len = 0;
    std::vector<long> soff, roff, counts;  // per peer offsets; size x size lengths
};

namespace {

__global__ void k_gather(const double *__restrict__ x, const int *__restrict__ idx, long long n,
                         double *__restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = x[idx[i]];
}

// Columns outside [lo, hi) (another rank's rows): counted, and with out set
// stored at atomically taken positions (the host sorts them); columns
// outside [0, ntot) raise *bad.
__global__ void k_halo_scan(const int *__restrict__ ci, long long nnz, long long lo, long long hi, long long ntot,
                            unsigned long long *count, int *out, unsigned long long cap, int *bad) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const long long c = ci[k];
        if (c < 0 || c >= ntot) {
            *bad = 1;
        } else if (c < lo || c >= hi) {
            const unsigned long long pos = atomicAdd(count, 1ull);
            if (out && pos < cap) out[pos] = (int)c;
        }
    }
}

// Local numbering: own rows to c - lo, halo columns to nloc + their position
// in the sorted halo list ext (binary search).
__global__ void k_halo_renumber(const int *__restrict__ ci, long long nnz, long long lo, long long hi, int nloc,
                                const int *__restrict__ ext, int next, int *__restrict__ out) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const long long c = ci[k];
        if (c >= lo && c < hi) {
            out[k] = (int)(c - lo);
        } else {
            int a = 0, b = next;
            while (a < b) {
                const int mid = (a + b) >> 1;
                if (ext[mid] < c)
                    a = mid + 1;
                else
                    b = mid;
            }
            out[k] = nloc + a;
        }
    }
}

}  // namespace

void launch_halo_scan(const int *ci, long long nnz, long long lo, long long hi, long long ntot,
                      unsigned long long *count, int *out, unsigned long long cap, int *bad) {
    const int nb = (int)std::max<long long>(1, std::min<long long>((nnz + 255) / 256, 148LL * 16));
    k_halo_scan<<<nb, 256>>>(ci, nnz, lo, hi, ntot, count, out, cap, bad);
}

void launch_halo_renumber(const int *ci, long long nnz, long long lo, long long hi, int nloc, const int *ext,
                          int next, int *out) {
    const int nb = (int)std::max<long long>(1, std::min<long long>((nnz + 255) / 256, 148LL * 16));
    k_halo_renumber<<<nb, 256>>>(ci, nnz, lo, hi, nloc, ext, next, out);
}

int halo_exchange(const trlx_operator *A, const double *x, cudaStream_t st, const double **x_ext) {
    Halo *h = A->halo;
    if (h->nsend > 0) {
        const int nb = (int)std::min<long long>((h->nsend + 255) / 256, 148LL * 8);
        k_gather<<<nb, 256, 0, st>>>(x, h->send_idx, h->nsend, h->send_buf);
    }
    if (cudaMemcpyAsync(h->x_ext, x, sizeof(double) * (size_t)A->nrow, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return -1001;
    if (int e = h->comm->exchange(h->send_buf, h->soff, h->x_ext + A->nrow, h->roff, h->counts, st)) return e;
    *x_ext = h->x_ext;
    return 0;
}

// ---- SELL-C-32 construction ------------------------------------------------
// Stored row r of slice s = r / 32 is original row perm[r] (r without a
// permutation).  Slice s holds width(s) = max row length of its 32 rows
// entries per row, column-major: entry k of stored row s*32+l at
// slice_ptr[s] + 32k + l.  Padding entries have value 0 and the column of
// their own row (row 0 for the rows past nrow), so they read a valid x.

namespace {

__global__ void k_slice_width(int nrow, int nslice, const long long *__restrict__ rp,
                              const int *__restrict__ perm, int *__restrict__ width) {
    const int lane = threadIdx.x & 31;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long s = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslice; s += warps) {
        const long r = s * 32 + lane;
        long long len = 0;
        if (r < nrow) {
            const long o = perm ? perm[r] : r;
            len = rp[o + 1] - rp[o];
        }
        for (int d = 16; d; d >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, d));
        if (lane == 0) width[s] = (int)len;
    }
}

template <class V>
__global__ void k_sell_fill(int nrow, int nslice, const long long *__restrict__ rp, const int *__restrict__ ci,
                            const V *__restrict__ va, const int *__restrict__ perm,
                            const long long *__restrict__ sp, int *__restrict__ sc, V *__restrict__ sv) {
    const int lane = threadIdx.x & 31;
    const long warps = ((long)gridDim.x * blockDim.x) >> 5;
    for (long s = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nslice; s += warps) {
        const long r = s * 32 + lane;
        const long o = r < nrow ? (perm ? perm[r] : r) : -1;
        const long long beg = o >= 0 ? rp[o] : 0;
        const long long len = o >= 0 ? rp[o + 1] - beg : 0;
        const long long base = sp[s];
        const long long w = (sp[s + 1] - base) >> 5;
        const int pad_col = o >= 0 ? (int)o : 0;
        for (long long k = 0; k < w; ++k) {
            const long long d = base + 32 * k + lane;
            if (k < len) {
                sc[d] = ci[beg + k];
                sv[d] = va[beg + k];
            } else {
                sc[d] = pad_col;
                sv[d] = czero(V());
            }
        }
    }
}

}  // namespace

int sell_build_grid(int nslice) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    const long need = ((long)nslice + 7) / 8;  // 8 warps (slices) per 256-thread block
    return (int)std::max<long>(1, std::min<long>(need, (long)sms * 8));
}

void launch_slice_width(int nrow, int nslice, const long long *rp, const int *perm, int *width, int grid) {
    k_slice_width<<<grid, 256>>>(nrow, nslice, rp, perm, width);
}

template <class V>
void launch_sell_fill(int nrow, int nslice, const long long *rp, const int *ci, const V *va, const int *perm,
                      const long long *sp, int *sc, V *sv, int grid) {
    k_sell_fill<V><<<grid, 256>>>(nrow, nslice, rp, ci, va, perm, sp, sc, sv);
}

}  // namespace trlb

// ---------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------
namespace {

// Device memory of the built-in operators comes from a per-device
// stream-ordered pool that keeps what is freed (release threshold
// unlimited): creating and destroying operators of similar size again and
// again then reuses the same memory instead of going through the driver's
// allocation path, where GB-sized cudaMalloc/cudaFree calls on a busy host
// now and then take hundreds of milliseconds.  trlx_release_workspace()
// returns the unused pool memory.  Devices without pool support use
// cudaMalloc/cudaFree.
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDevices] = {};
int g_pool_state[kMaxDevices] = {};  // 0 not tried, 1 pool, -1 no pool

cudaMemPool_t op_pool(int dev) {
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> g(g_pool_mu);
    if (g_pool_state[dev] == 0) {
        g_pool_state[dev] = -1;
        int supported = 0;
        cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev);
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (supported && cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
            uint64_t keep = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            g_pool[dev] = pool;
            g_pool_state[dev] = 1;
        } else {
            cudaGetLastError();
        }
    }
    return g_pool[dev];
}

int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

// Allocation on the current device, ordered on the legacy default stream
// (every use of operator memory comes after a synchronisation).
cudaError_t op_alloc(void **p, size_t bytes) {
    cudaMemPool_t pool = op_pool(current_device());
    cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, 0) : cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
    }
    return e;
}

// Free on the current device (the one the memory was allocated on).
void op_free(void *p) {
    if (!p) return;
    if (op_pool(current_device()))
        cudaFreeAsync(p, 0);
    else
        cudaFree(p);
}

template <class X>
int to_device(const X *src, size_t count, int where, X **dst) {
    if (count == 0) {
        *dst = nullptr;
        return 0;
    }
    if (op_alloc(reinterpret_cast<void **>(dst), count * sizeof(X)) != cudaSuccess) return -2;
    cudaError_t e = where == TRLX_DEVICE_ARRAYS
                        ? cudaMemcpy(*dst, src, count * sizeof(X), cudaMemcpyDeviceToDevice)
                        : trlb::host_copy(*dst, src, count * sizeof(X), cudaMemcpyHostToDevice, 0);
    return e == cudaSuccess ? 0 : -3;
}

template <class X>
std::vector<X> to_host(const X *src, size_t count, int where) {
    std::vector<X> h(count);
    if (count == 0) return h;
    if (where == TRLX_DEVICE_ARRAYS)
        cudaMemcpy(h.data(), src, count * sizeof(X), cudaMemcpyDeviceToHost);
    else
        std::memcpy(h.data(), src, count * sizeof(X));
    return h;
}

int check_csr(int nrow, const long long *rp, const int *ci, const void *val) {
    if (nrow <= 0 || !rp || !ci || !val) return -1;
    return 0;
}

}  // namespace

extern "C" int trlx_csr_create(int nrow, const long long *row_ptr, const int *col_idx,
                               const double *val, int where, trlx_operator **out) {
    if (!out || check_csr(nrow, row_ptr, col_idx, val)) return -1;
    auto *A = new trlx_operator();
    A->kind = 0;
    A->nrow = nrow;
    long long nnz = 0;
    if (where == TRLX_DEVICE_ARRAYS)
        cudaMemcpy(&nnz, row_ptr + nrow, sizeof(long long), cudaMemcpyDeviceToHost);
    else
        nnz = row_ptr[nrow];
    A->nnz = nnz;
    cudaGetDevice(&A->device);
    int rc = to_device(row_ptr, (size_t)nrow + 1, where, &A->row_ptr);
    if (!rc) rc = to_device(col_idx, (size_t)nnz, where, &A->col);
    double *dv = nullptr;
    if (!rc) rc = to_device(val, (size_t)nnz, where, &dv);
    A->val = dv;
    if (rc) {
        trlx_operator_destroy(A);
        return rc;
    }
    *out = A;
    return 0;
}

extern "C" int trlx_zcsr_create(int nrow, const long long *row_ptr, const int *col_idx,
                                const trl_dcomplex *val, int where, trlx_operator **out) {
    if (!out || check_csr(nrow, row_ptr, col_idx, val)) return -1;
    auto *A = new trlx_operator();
    A->kind = 2;
    A->nrow = nrow;
    long long nnz = 0;
    if (where == TRLX_DEVICE_ARRAYS)
        cudaMemcpy(&nnz, row_ptr + nrow, sizeof(long long), cudaMemcpyDeviceToHost);
    else
        nnz = row_ptr[nrow];
    A->nnz = nnz;
    cudaGetDevice(&A->device);
    int rc = to_device(row_ptr, (size_t)nrow + 1, where, &A->row_ptr);
    if (!rc) rc = to_device(col_idx, (size_t)nnz, where, &A->col);
    trlb::zd *dv = nullptr;
    if (!rc) rc = to_device(reinterpret_cast<const trlb::zd *>(val), (size_t)nnz, where, &dv);
    A->val = dv;
    if (rc) {
        trlx_operator_destroy(A);
        return rc;
    }
    *out = A;
    return 0;
}

namespace {

// SELL-C-32 from CSR input with values of type V (double: kind 1, zd: kind 3).
template <class V>
int sell_create(int nrow, const long long *row_ptr, const int *col_idx, const V *val, int sigma, int where,
                int kind, trlx_operator **out) {
    if (!out || check_csr(nrow, row_ptr, col_idx, val)) return -1;
    if (sigma < 1) sigma = 1;
    const bool dev = where == TRLX_DEVICE_ARRAYS;
    long long nnz = 0;
    if (dev)
        cudaMemcpy(&nnz, row_ptr + nrow, sizeof(long long), cudaMemcpyDeviceToHost);
    else
        nnz = row_ptr[nrow];
    // Within windows of sigma rows, order rows by decreasing length (stable):
    // host work on the row pointers only.
    std::vector<int> order;
    if (sigma > 1) {
        std::vector<long long> rp = to_host(row_ptr, (size_t)nrow + 1, where);
        order.resize(nrow);
        std::iota(order.begin(), order.end(), 0);
        for (long w0 = 0; w0 < nrow; w0 += sigma) {
            long w1 = std::min<long>(nrow, w0 + sigma);
            std::stable_sort(order.begin() + w0, order.begin() + w1, [&](int a, int b) {
                return (rp[a + 1] - rp[a]) > (rp[b + 1] - rp[b]);
            });
        }
        bool identity = true;
        for (int i = 0; i < nrow && identity; ++i) identity = (order[i] == i);
        if (identity) order.clear();
    }
    auto *A = new trlx_operator();
    A->kind = kind;
    A->nrow = nrow;
    A->nslice = (nrow + 31) / 32;
    A->sigma = sigma;
    cudaGetDevice(&A->device);
    // CSR arrays on the device (the caller's own when they already are).
    long long *d_rp = dev ? const_cast<long long *>(row_ptr) : nullptr;
    int *d_ci = dev ? const_cast<int *>(col_idx) : nullptr;
    V *d_va = dev ? const_cast<V *>(val) : nullptr;
    int *d_w = nullptr;
    int rc = 0;
    if (!dev) {
        rc = to_device(row_ptr, (size_t)nrow + 1, where, &d_rp);
        if (!rc) rc = to_device(col_idx, (size_t)nnz, where, &d_ci);
        if (!rc) rc = to_device(val, (size_t)nnz, where, &d_va);
    }
    if (!rc && !order.empty()) rc = to_device(order.data(), order.size(), TRLX_HOST_ARRAYS, &A->perm);
    // Slice widths on the device, their prefix sum on the host (nrow/32 values).
    const int nslice = A->nslice;
    const int grid = trlb::sell_build_grid(nslice);
    std::vector<long long> sp(nslice + 1, 0);
    if (!rc && op_alloc(reinterpret_cast<void **>(&d_w), sizeof(int) * nslice) != cudaSuccess) rc = -2;
    if (!rc) {
        trlb::launch_slice_width(nrow, nslice, d_rp, A->perm, d_w, grid);
        std::vector<int> w(nslice);
        if (cudaMemcpy(w.data(), d_w, sizeof(int) * nslice, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -3;
        for (int s = 0; s < nslice && !rc; ++s) sp[s + 1] = sp[s] + 32LL * w[s];
    }
    if (!rc) rc = to_device(sp.data(), sp.size(), TRLX_HOST_ARRAYS, &A->slice_ptr);
    const long long total = sp[nslice];
    A->nnz = total;
    V *dv = nullptr;
    if (!rc && (op_alloc(reinterpret_cast<void **>(&A->col), sizeof(int) * std::max<long long>(total, 1)) !=
                    cudaSuccess ||
                op_alloc(reinterpret_cast<void **>(&dv), sizeof(V) * std::max<long long>(total, 1)) !=
                    cudaSuccess))
        rc = -2;
    A->val = dv;
    if (!rc) {
        trlb::launch_sell_fill(nrow, nslice, d_rp, d_ci, d_va, A->perm, A->slice_ptr, A->col, dv, grid);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = -3;
    }
    op_free(d_w);
    if (!dev) {
        op_free(d_rp);
        op_free(d_ci);
        op_free(d_va);
    }
    if (rc) {
        cudaGetLastError();
        trlx_operator_destroy(A);
        return rc;
    }
    *out = A;
    return 0;
}

}  // namespace

extern "C" int trlx_sell_create(int nrow, const long long *row_ptr, const int *col_idx,
                                const double *val, int sigma, int where, trlx_operator **out) {
    return sell_create<double>(nrow, row_ptr, col_idx, val, sigma, where, 1, out);
}

extern "C" int trlx_zsell_create(int nrow, const long long *row_ptr, const int *col_idx,
                                 const trl_dcomplex *val, int sigma, int where, trlx_operator **out) {
    return sell_create<trlb::zd>(nrow, row_ptr, col_idx, reinterpret_cast<const trlb::zd *>(val), sigma, where, 3,
                                 out);
}

extern "C" void trlx_operator_destroy(trlx_operator *A) {
    if (!A) return;
    // Like cudaFree: work still running on any stream of the device may read
    // the operator, so wait for the device before the memory is reused.
    int prev = current_device();
    if (A->device >= 0 && A->device != prev) cudaSetDevice(A->device);
    cudaDeviceSynchronize();
    op_free(A->row_ptr);
    op_free(A->col);
    op_free(A->val);
    op_free(A->slice_ptr);
    op_free(A->perm);
    if (A->halo) {
        op_free(A->halo->send_idx);
        op_free(A->halo->send_buf);
        op_free(A->halo->x_ext);
        delete A->halo;
    }
    cudaStreamSynchronize(0);
    if (A->device >= 0 && A->device != prev) cudaSetDevice(prev);
    delete A;
}

namespace trlb {

void trim_operator_pools() {
    std::lock_guard<std::mutex> g(g_pool_mu);
    for (int d = 0; d < kMaxDevices; ++d)
        if (g_pool[d]) cudaMemPoolTrimTo(g_pool[d], 0);
}

}  // namespace trlb

extern "C" long long trlx_operator_nnz(const trlx_operator *A) { return A ? A->nnz : 0; }
extern "C" int trlx_operator_nrow(const trlx_operator *A) { return A ? A->nrow : 0; }

extern "C" long long trlx_operator_halo(const trlx_operator *A) { return A && A->halo ? A->halo->nhalo : 0; }

namespace {

// Block-row operator of this rank (reference model: SRC/trl_comm_mpi.c
// distributes rows the same way; its user operator does the exchange).
// Every rank takes part in every collective below, also on bad input, so
// that no rank is left waiting.
int dist_create(trlx_comm *comm, int nloc, const long long *row_ptr, const int *col_idx, const double *val,
                int sigma, bool sell, int where, trlx_operator **out) {
    if (!out || !comm || !comm->impl || nloc <= 0 || !row_ptr || !col_idx || !val) return -1;
    trlb::Comm *cm = comm->impl;
    const int P = cm->size, me = cm->rank;
    const bool dev = where == TRLX_DEVICE_ARRAYS;
    // Row ranges of all ranks.
    std::vector<double> cnt(P, 0.0);
    cnt[me] = nloc;
    if (int e = cm->reduce_host(cnt.data(), P, trlb::kOpSum)) return e;
    std::vector<long long> start(P + 1, 0);
    for (int p = 0; p < P; ++p) start[p + 1] = start[p] + (long long)cnt[p];
    const long long row0 = start[me], ntot = start[P], row1 = row0 + nloc;
    std::vector<long long> rp = to_host(row_ptr, (size_t)nloc + 1, where);
    int bad = rp[0] != 0 || rp[nloc] < 0;
    const long long nnz = bad ? 0 : rp[nloc];
    // Column indices and values on the device (the caller's device arrays
    // are read, never changed); the scan over all entries runs there.
    int *d_ci = dev ? const_cast<int *>(col_idx) : nullptr;
    double *d_va = dev ? const_cast<double *>(val) : nullptr;
    int *d_new = nullptr, *d_ext = nullptr, *d_raw = nullptr;
    long long *d_rp = nullptr;
    unsigned long long *d_cnt = nullptr;
    auto cleanup = [&] {
        if (!dev) {
            op_free(d_ci);
            op_free(d_va);
        }
        op_free(d_new);
        op_free(d_ext);
        op_free(d_raw);
        op_free(d_rp);
        op_free(d_cnt);
    };
    std::vector<int> ext;
    if (!bad && nnz > 0) {
        int rc = 0;
        if (!dev) {
            rc = to_device(col_idx, (size_t)nnz, where, &d_ci);
            if (!rc) rc = to_device(val, (size_t)nnz, where, &d_va);
        }
        // d_cnt[0]: out-of-range count, d_cnt[1] (as int): bad column flag.
        if (!rc && op_alloc(reinterpret_cast<void **>(&d_cnt), 2 * sizeof(unsigned long long)) != cudaSuccess)
            rc = -2;
        unsigned long long hc[2] = {0, 0};
        if (!rc && cudaMemset(d_cnt, 0, sizeof(hc)) != cudaSuccess) rc = -3;
        int *d_bad = reinterpret_cast<int *>(d_cnt + 1);
        if (!rc) {
            trlb::launch_halo_scan(d_ci, nnz, row0, row1, ntot, d_cnt, nullptr, 0, d_bad);
            if (cudaMemcpy(hc, d_cnt, sizeof(hc), cudaMemcpyDeviceToHost) != cudaSuccess) rc = -3;
        }
        const unsigned long long nraw = hc[0];
        if (!rc && (int)hc[1] != 0) bad = 1;
        if (!rc && !bad && nraw > 0) {
            if (op_alloc(reinterpret_cast<void **>(&d_raw), sizeof(int) * nraw) != cudaSuccess) rc = -2;
            if (!rc && cudaMemset(d_cnt, 0, sizeof(unsigned long long)) != cudaSuccess) rc = -3;
            if (!rc) {
                trlb::launch_halo_scan(d_ci, nnz, row0, row1, ntot, d_cnt, d_raw, nraw, d_bad);
                ext.resize(nraw);
                if (cudaMemcpy(ext.data(), d_raw, sizeof(int) * nraw, cudaMemcpyDeviceToHost) != cudaSuccess)
                    rc = -3;
            }
        }
        if (rc) bad = 1;
    }
    // Every rank takes part in every collective below, also on bad input.
    double flag = bad;
    if (int e = cm->reduce_host(&flag, 1, trlb::kOpMax)) {
        cleanup();
        return e;
    }
    if (flag != 0.0) {
        cleanup();
        return -1;
    }
    // Columns owned by other ranks, ascending (hence grouped by owner).
    std::sort(ext.begin(), ext.end());
    ext.erase(std::unique(ext.begin(), ext.end()), ext.end());
    const int nhalo = (int)ext.size();
    std::vector<long> roff(P + 1, 0);
    for (int c : ext) {
        const int p = (int)(std::upper_bound(start.begin(), start.end(), (long long)c) - start.begin()) - 1;
        roff[p + 1]++;
    }
    for (int p = 0; p < P; ++p) roff[p + 1] += roff[p];
    // counts[p * P + q]: values p sends to q.
    std::vector<double> cm_counts((size_t)P * P, 0.0);
    for (int p = 0; p < P; ++p) cm_counts[(size_t)p * P + me] = (double)(roff[p + 1] - roff[p]);
    if (int e = cm->reduce_host(cm_counts.data(), cm_counts.size(), trlb::kOpSum)) {
        cleanup();
        return e;
    }
    std::vector<long> counts(cm_counts.size());
    for (size_t k = 0; k < counts.size(); ++k) counts[k] = (long)cm_counts[k];
    // The requested global indices, on a board with one segment per
    // (owner, requester) pair.
    std::vector<long> bo(counts.size() + 1, 0);
    for (size_t k = 0; k < counts.size(); ++k) bo[k + 1] = bo[k] + counts[k];
    std::vector<double> board((size_t)bo.back(), 0.0);
    for (int p = 0; p < P; ++p)
        for (long k = roff[p]; k < roff[p + 1]; ++k) board[(size_t)bo[(size_t)p * P + me] + (k - roff[p])] = ext[k];
    if (int e = cm->reduce_host(board.data(), board.size(), trlb::kOpSum)) {
        cleanup();
        return e;
    }
    std::vector<long> soff(P + 1, 0);
    std::vector<int> sidx;
    for (int q = 0; q < P; ++q) {
        const long c = counts[(size_t)me * P + q];
        for (long k = 0; k < c; ++k)
            sidx.push_back((int)((long long)board[(size_t)bo[(size_t)me * P + q] + k] - row0));
        soff[q + 1] = soff[q] + c;
    }
    // Local numbering on the device: own rows first, then the halo in
    // receive order; the local operator is built from device arrays.
    int rc = to_device(rp.data(), rp.size(), TRLX_HOST_ARRAYS, &d_rp);
    if (!rc && nnz > 0) {
        if (op_alloc(reinterpret_cast<void **>(&d_new), sizeof(int) * (size_t)nnz) != cudaSuccess) rc = -2;
        if (!rc && nhalo > 0) rc = to_device(ext.data(), ext.size(), TRLX_HOST_ARRAYS, &d_ext);
        if (!rc) trlb::launch_halo_renumber(d_ci, nnz, row0, row1, nloc, d_ext, nhalo, d_new);
    }
    trlx_operator *A = nullptr;
    if (!rc)
        rc = sell ? trlx_sell_create(nloc, d_rp, d_new, d_va, sigma, TRLX_DEVICE_ARRAYS, &A)
                  : trlx_csr_create(nloc, d_rp, d_new, d_va, TRLX_DEVICE_ARRAYS, &A);
    cleanup();
    if (rc) return rc;
    auto *h = new trlb::Halo();
    A->halo = h;
    h->comm = cm;
    h->row0 = row0;
    h->nhalo = nhalo;
    h->nsend = (long long)sidx.size();
    h->soff = soff;
    h->roff = roff;
    h->counts = counts;
    const long n_pad = ((long)nloc + 255) / 256 * 256;
    h->ext_len = std::max<long>(n_pad, (long)nloc + nhalo);
    if (h->nsend > 0) {
        rc = to_device(sidx.data(), sidx.size(), TRLX_HOST_ARRAYS, &h->send_idx);
        if (!rc && op_alloc(reinterpret_cast<void **>(&h->send_buf), sizeof(double) * sidx.size()) != cudaSuccess)
            rc = -2;
    }
    if (!rc && op_alloc(reinterpret_cast<void **>(&h->x_ext), sizeof(double) * h->ext_len) != cudaSuccess) rc = -2;
    // Entries past nloc + nhalo are only ever multiplied by zero; keep them zero.
    if (!rc && (cudaMemsetAsync(h->x_ext, 0, sizeof(double) * h->ext_len, 0) != cudaSuccess ||
                cudaStreamSynchronize(0) != cudaSuccess))
        rc = -3;
    if (rc) {
        trlx_operator_destroy(A);
        return rc;
    }
    *out = A;
    return 0;
}

}  // namespace

extern "C" int trlx_dist_csr_create(trlx_comm *comm, int nloc, const long long *row_ptr, const int *col_idx,
                                    const double *val, int where, trlx_operator **out) {
    return dist_create(comm, nloc, row_ptr, col_idx, val, 1, false, where, out);
}

extern "C" int trlx_dist_sell_create(trlx_comm *comm, int nloc, const long long *row_ptr, const int *col_idx,
                                     const double *val, int sigma, int where, trlx_operator **out) {
    return dist_create(comm, nloc, row_ptr, col_idx, val, sigma, true, where, out);
}

extern "C" void trlx_matvec(const int nrow, const int ncol, const double *x, const int ldx, double *y,
                            const int ldy, void *mvparam) {
    auto *A = static_cast<trlx_operator *>(mvparam);
    if (!A || trlb::op_complex(A) || nrow != A->nrow) return;
    for (int j = 0; j < ncol; ++j) trlb::spmv_plain(A, x + (long)j * ldx, y + (long)j * ldy, 0);
}

extern "C" void trlx_zmatvec(const int nrow, const int ncol, const trl_dcomplex *x, const int ldx,
                             trl_dcomplex *y, const int ldy, void *mvparam) {
    auto *A = static_cast<trlx_operator *>(mvparam);
    if (!A || !trlb::op_complex(A) || nrow != A->nrow) return;
    for (int j = 0; j < ncol; ++j) trlb::spmv_plain(A, x + (long)j * ldx, y + (long)j * ldy, 0);
}

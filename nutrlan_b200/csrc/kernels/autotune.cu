// trlx_operator_autotune: the single-solve autotuner (no counterpart in the
// reference, whose user operator is opaque).  For a built-in operator
// created in CSR form (real or complex) it measures, on this GPU and this
// matrix:
//
//  * one fused product y = A x, alpha = Re(x^H y) (the kernel every Lanczos
//    step starts with) in the CSR form and in the SELL-C-32 form built from
//    the same device arrays;
//  * Gram-Schmidt projections h = V^T r over maxlan / 4, maxlan / 2 and
//    3 maxlan / 4 basis columns of this operator's row count (a thick-restart
//    cycle's range of widths) in each form of the projection kernel (8, 12, 16 columns per
//    warp; 16 with the pointer table in shared memory; 16 with the basis
//    staged through shared memory by cp.async), once over FP64 columns and
//    once over FP32 columns (the two basis storage widths);
//
// and keeps the faster of each: the operator's storage is switched in place
// to the faster form (the handle stays valid; the other form is freed) and
// the two projection forms are stored in the operator, where solves with it
// read the one for their basis width.  Every candidate is timed with CUDA events over `kReps` launches after
// a warm-up launch, and the median is kept.  Products are checked against
// each other (the same alpha up to summation order) before a form is adopted.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../../include/trlx.h"
#include "lanczos_kernels.h"
#include "spmv.h"

namespace {

constexpr int kReps = 5;

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    bool alloc(size_t bytes) {
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return false;
        }
        return true;
    }
};

template <class V>
__global__ void k_fill_pattern(V *v, long n, long n_pad, unsigned salt) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad; i += stride) {
        // Deterministic values in [-1, 1); padding rows stay zero as the
        // kernels require.
        unsigned x = (unsigned)(i * 2654435761u) ^ (salt * 0x9E3779B9u);
        x ^= x >> 15;
        x *= 0x2c1b3c6du;
        x ^= x >> 12;
        v[i] = i < n ? (V)((double)(x & 0xFFFFFF) / 8388608.0 - 1.0) : (V)0;
    }
}

template <class F>
double median_ms(F launch, cudaStream_t st) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch();  // warm-up
    std::vector<float> t(kReps);
    for (int r = 0; r < kReps; ++r) {
        cudaEventRecord(a, st);
        launch();
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&t[r], a, b);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    std::sort(t.begin(), t.end());
    return t[kReps / 2];
}

void move_storage(trlx_operator *dst, trlx_operator *src) {
    std::swap(dst->kind, src->kind);
    std::swap(dst->nnz, src->nnz);
    std::swap(dst->row_ptr, src->row_ptr);
    std::swap(dst->col, src->col);
    std::swap(dst->val, src->val);
    std::swap(dst->nslice, src->nslice);
    std::swap(dst->sigma, src->sigma);
    std::swap(dst->slice_ptr, src->slice_ptr);
    std::swap(dst->perm, src->perm);
}

// Refills the first mp columns of the basis buffer as storage type V
// (vw scalars per element) and returns their column table, copied to
// `table` on the device.
template <class V>
void fill_columns(void *basis, void *table, int mp, long n, long n_pad, int vw, cudaStream_t st) {
    std::vector<V *> cols(mp);
    for (int c = 0; c < mp; ++c) {
        cols[c] = static_cast<V *>(basis) + (size_t)c * vw * n_pad;
        k_fill_pattern<V><<<592, 256, 0, st>>>(cols[c], vw * n, vw * n_pad, 7u + c);
    }
    cudaMemcpyAsync(table, cols.data(), sizeof(V *) * mp, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
}

// Index of the fastest of the timed forms (negative times: not timed),
// starting from `dflt`, which stays unless another form measured faster.
int fastest(const double (&ms)[trlb::kProjectForms], int dflt) {
    int best = dflt;
    for (int k = 0; k < trlb::kProjectForms; ++k)
        if (ms[k] >= 0.0 && ms[k] < ms[best]) best = k;
    return best;
}

}  // namespace

extern "C" int trlx_operator_autotune(trlx_operator *A, int maxlan, trlx_tune_result *out) {
    if (!A || !out) return -1;
    *out = trlx_tune_result{};
    // Real CSR-created or complex CSR operators, not distributed ones.
    if ((A->kind != 0 && A->kind != 2) || A->halo) return -1;
    const bool cplx = A->kind == 2;
    const int vw = cplx ? 2 : 1;  // doubles per vector element
    const auto t0 = std::chrono::steady_clock::now();
    int prev = 0;
    cudaGetDevice(&prev);
    if (A->device >= 0 && A->device != prev) cudaSetDevice(A->device);
    int rc = 0;
    const long n = A->nrow;
    const long n_pad = (n + 255) / 256 * 256;
    // The projection is timed at three basis widths spread over a cycle,
    // mp / 3, 2 mp / 3 and mp with mp = 3 maxlan / 4 (at most 128), and a
    // form's time is their sum: the forms' efficiency depends on how the
    // width splits into column groups, so one width would favour whichever
    // form divides it evenly.
    const int m = std::max(8, std::min(128, 3 * maxlan / 4));
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    // Vectors, reduction scratch and the projection's basis columns.
    trlb::Scratch s;
    s.max_blocks = 148 * 8;
    s.max_cols = m;
    DevBuf x, y, part, tick, dsc, basis, table;
    const size_t vec = sizeof(double) * vw * (size_t)n_pad;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    // The widest timing uses m columns when they fit in a quarter of the
    // free memory, else as many as fit (at least 8).
    int mp = (int)std::min<size_t>((size_t)m, free_b / 4 / std::max<size_t>(vec, 1));
    if (mp < 8 || !x.alloc(vec) || !y.alloc(vec) || !part.alloc((size_t)s.max_blocks * (m + 2) * 16) ||
        !tick.alloc(sizeof(unsigned) * trlb::kNumTickets) || !dsc.alloc(sizeof(double) * vw * (m + 4)) ||
        !basis.alloc(vec * mp) || !table.alloc(sizeof(double *) * mp)) {
        rc = -2;
    }
    trlx_operator *other = nullptr;
    const int widths[3] = {std::max(1, mp / 3), std::max(1, 2 * mp / 3), mp};
    auto over_widths = [&](auto launch_at) {
        double t = 0.0;
        for (int w : widths) t += median_ms([&] { launch_at(w); }, st);
        return t;
    };
    if (!rc) {
        s.partials = part.p;
        s.tickets = static_cast<unsigned *>(tick.p);
        cudaMemsetAsync(tick.p, 0, sizeof(unsigned) * trlb::kNumTickets, st);
        // Complex vectors are filled as interleaved (re, im) doubles.
        k_fill_pattern<double><<<592, 256, 0, st>>>(static_cast<double *>(x.p), vw * n, vw * n_pad, 1u);
        fill_columns<double>(basis.p, table.p, mp, n, n_pad, vw, st);
    }
    if (!rc && cplx) {
        // Complex CSR against complex SELL-C-32; the projection keeps its
        // pointer table in registers (form 3) or in shared memory (form 4),
        // or stages the basis through shared memory (form 5).
        using trlb::zd;
        double *alpha = static_cast<double *>(dsc.p);
        auto product = [&](const trlx_operator *op) {
            trlb::spmv_fused_cplx(op, static_cast<zd *>(x.p), static_cast<zd *>(y.p), n_pad, alpha, &s, st);
        };
        out->spmv_ms[0] = median_ms([&] { product(A); }, st);
        out->format = 0;
        out->spmv_ms[1] = -1.0;
        double a_csr = 0.0, a_sell = 0.0;
        cudaMemcpy(&a_csr, alpha, sizeof(double), cudaMemcpyDeviceToHost);
        if (trlx_zsell_create((int)n, A->row_ptr, A->col, static_cast<const trl_dcomplex *>(A->val), 1,
                              TRLX_DEVICE_ARRAYS, &other) == 0) {
            out->spmv_ms[1] = median_ms([&] { product(other); }, st);
            cudaMemcpy(&a_sell, alpha, sizeof(double), cudaMemcpyDeviceToHost);
            const bool same = std::fabs(a_sell - a_csr) <= 1e-13 * (double)n + 1e-12 * std::fabs(a_csr);
            out->format = (same && out->spmv_ms[1] < out->spmv_ms[0]) ? 1 : 0;
            if (out->format == 1) move_storage(A, other);
        }
        trlb::Recur<zd> none;
        out->project_ms[0] = out->project_ms[1] = -1.0;
        for (int k = 2; k < trlb::kProjectForms; ++k) {
            out->project_ms[k] = over_widths([&](int w) {
                trlb::launch_project<zd>(static_cast<zd *const *>(table.p), w, n_pad, static_cast<const zd *>(x.p),
                                         none, static_cast<zd *>(dsc.p), static_cast<double *>(dsc.p) + 2 * (m + 1),
                                         s, st, trlb::kProject8 + k);
            });
        }
        const int best = trlb::kProject8 + fastest(out->project_ms, trlb::kProject16 - trlb::kProject8);
        A->project_form = best;
        out->project_form = best;
        // The same forms over complex64 columns.
        using trlb::zf;
        fill_columns<float>(basis.p, table.p, mp, n, n_pad, vw, st);
        out->project32_ms[0] = out->project32_ms[1] = -1.0;
        for (int k = 2; k < trlb::kProjectForms; ++k) {
            out->project32_ms[k] = over_widths([&](int w) {
                trlb::launch_project<zf>(static_cast<zf *const *>(table.p), w, n_pad, static_cast<const zd *>(x.p),
                                         none, static_cast<zd *>(dsc.p), static_cast<double *>(dsc.p) + 2 * (m + 1),
                                         s, st, trlb::kProject8 + k);
            });
        }
        const int best32 = trlb::kProject8 + fastest(out->project32_ms, trlb::kProject16 - trlb::kProject8);
        A->project_form32 = best32;
        out->project_form32 = best32;
        out->columns = widths[1];
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -3;
    } else if (!rc) {
        // ---- operator form ----------------------------------------------
        double *alpha = static_cast<double *>(dsc.p);
        out->spmv_ms[0] = median_ms(
            [&] {
                trlb::spmv_fused_real(A, static_cast<double *>(x.p), static_cast<double *>(y.p), n_pad, alpha, &s,
                                      st);
            },
            st);
        double a_csr = 0.0, a_sell = 0.0;
        cudaMemcpy(&a_csr, alpha, sizeof(double), cudaMemcpyDeviceToHost);
        rc = trlx_sell_create((int)n, A->row_ptr, A->col, static_cast<const double *>(A->val), 1,
                              TRLX_DEVICE_ARRAYS, &other);
        if (rc == 0) {
            out->spmv_ms[1] = median_ms(
                [&] {
                    trlb::spmv_fused_real(other, static_cast<double *>(x.p), static_cast<double *>(y.p), n_pad,
                                          alpha, &s, st);
                },
                st);
            cudaMemcpy(&a_sell, alpha, sizeof(double), cudaMemcpyDeviceToHost);
            // Same product up to the summation order of n terms of order one.
            const bool same = std::fabs(a_sell - a_csr) <= 1e-13 * (double)n + 1e-12 * std::fabs(a_csr);
            out->format = (same && out->spmv_ms[1] < out->spmv_ms[0]) ? 1 : 0;
            if (out->format == 1) move_storage(A, other);  // A takes the SELL arrays, `other` the CSR ones
        } else {
            rc = 0;  // keep CSR when SELL cannot be built (memory)
            out->format = 0;
            out->spmv_ms[1] = -1.0;
        }
        // ---- projection kernel form -------------------------------------
        trlb::Recur<double> none;
        for (int k = 0; k < trlb::kProjectForms; ++k) {
            out->project_ms[k] = over_widths([&](int w) {
                trlb::launch_project<double>(static_cast<double *const *>(table.p), w, n_pad,
                                             static_cast<const double *>(x.p), none, static_cast<double *>(dsc.p),
                                             static_cast<double *>(dsc.p) + m + 1, s, st, trlb::kProject8 + k);
            });
        }
        const int best = fastest(out->project_ms, trlb::kProject16 - trlb::kProject8);
        A->project_form = trlb::kProject8 + best;
        out->project_form = trlb::kProject8 + best;
        // The same forms over FP32 columns (the first half of the buffer).
        fill_columns<float>(basis.p, table.p, mp, n, n_pad, vw, st);
        for (int k = 0; k < trlb::kProjectForms; ++k) {
            out->project32_ms[k] = over_widths([&](int w) {
                trlb::launch_project<float>(static_cast<float *const *>(table.p), w, n_pad,
                                            static_cast<const double *>(x.p), none, static_cast<double *>(dsc.p),
                                            static_cast<double *>(dsc.p) + m + 1, s, st, trlb::kProject8 + k);
            });
        }
        const int best32 = fastest(out->project32_ms, trlb::kProject16 - trlb::kProject8);
        A->project_form32 = trlb::kProject8 + best32;
        out->project_form32 = trlb::kProject8 + best32;
        out->columns = widths[1];
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -3;
    }
    if (other) trlx_operator_destroy(other);
    cudaStreamDestroy(st);
    cudaGetLastError();
    if (A->device >= 0 && A->device != prev) cudaSetDevice(prev);
    out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

extern "C" int trlx_operator_set_project_form(trlx_operator *A, int form) {
    if (!A || form < trlb::kProjectDefault || form > trlb::kProjectAsync) return -1;
    A->project_form = form;
    return 0;
}

extern "C" int trlx_operator_set_project_form32(trlx_operator *A, int form) {
    if (!A || form < trlb::kProjectDefault || form > trlb::kProjectAsync) return -1;
    A->project_form32 = form;
    return 0;
}

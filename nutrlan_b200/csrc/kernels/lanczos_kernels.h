// Host-side launch API for the Lanczos vector kernels (lanczos_kernels.cu).
//
// Basis storage: every basis vector ("column") is a separate, 256-element
// padded device allocation slot addressed through a device table of column
// pointers.  Padding rows are kept at zero by every kernel, so the kernels
// run over n_pad rows without tail checks.  T is the storage type (double,
// float, zd, zf); the compute type C (double or zd) is FP64 throughout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace trlb {

// Reduction scratch shared by the kernels of one solver instance.
struct Scratch {
    void *partials = nullptr;  // >= max_blocks * (max_cols + 2) * 16 bytes
    unsigned *tickets = nullptr;  // kNumTickets counters, zero between launches
    int max_blocks = 0;
    int max_cols = 0;
};
constexpr int kNumTickets = 8;

// r = y - alpha*x - beta*xp, applied on the fly when `on` is set.
template <class C>
struct Recur {
    const C *x = nullptr;
    const C *xp = nullptr;
    const double *alpha = nullptr;  // device scalar
    double beta = 0.0;
    const double *beta_r2 = nullptr;  // when set: beta = sqrt(*beta_r2) (device)
    int on = 0;
};

// Number of row blocks used by the streaming kernels for n_pad rows.
int stream_blocks(long n_pad, int rows_per_thread_group);

// alpha = Re(x^H y) -> *out (device).  Deterministic.
template <class C>
void launch_dot(const C *x, const C *y, long n_pad, double *out, Scratch &s,
                cudaStream_t st);

// Forms of the projection kernel: for real storage (FP64 or FP32) 8, 12 or
// 16 columns per warp, or 16 with the column-pointer table in shared memory;
// for complex storage 8 columns per warp with the table in registers
// (kProject8 .. kProject16) or in shared memory (kProject16Shared); for
// every storage type, 16 warps of 8 columns with the basis staged through a
// shared-memory ring by cp.async, one block per SM (kProjectAsync).
enum ProjectForm {
    kProjectDefault = 0,
    kProject8 = 1,
    kProject12 = 2,
    kProject16 = 3,
    kProject16Shared = 4,
    kProjectAsync = 5,
    kProjectForms = 5
};

// h[c] = V[:,c]^H r for c < m; out2[0] = ||r||^2, out2[1] = ||h||^2.
// form: a ProjectForm (kProjectDefault: 16 columns, or TRLX_PROJECT_CPW).
template <class T>
void launch_project(T *const *cols, int m, long n_pad,
                    const typename Store<T>::C *r,
                    Recur<typename Store<T>::C> rec, typename Store<T>::C *h,
                    double *out2, Scratch &s, cudaStream_t st, int form = kProjectDefault);

// r_out = r - V h (r computed with the recurrence if rec.on);
// *out_r2 = ||r_out||^2.  r_out may alias r.
template <class T>
void launch_update(T *const *cols, int m, long n_pad,
                   const typename Store<T>::C *r,
                   Recur<typename Store<T>::C> rec,
                   const typename Store<T>::C *h, typename Store<T>::C *r_out,
                   double *out_r2, Scratch &s, cudaStream_t st);

// q = r * scale (scale = 1/sqrt(*r2) when r2 != null, else `fixed`);
// writes q (FP64, may alias r) and, if vcol != null, the stored copy.
template <class T>
void launch_normalize(typename Store<T>::C *r, long n_pad, const double *r2,
                      double fixed, typename Store<T>::C *q, T *vcol,
                      cudaStream_t st);

// out[:,k] = sum_c in[:,c] * Y[c + k*ldy] for k < kept, c < jml (Y real,
// device).  out and in must not overlap.
template <class T>
void launch_ritz(T *const *in_cols, int jml, long n_pad, const double *Y,
                 int ldy, int kept, T *const *out_cols, cudaStream_t st);

// Same, but writing FP64 compute-type output columns (user eigenvectors).
template <class T>
void launch_ritz_out(T *const *in_cols, int jml, long n_pad, const double *Y,
                     int ldy, int kept, typename Store<T>::C *out, long ldo,
                     long n, cudaStream_t st);

// Elementwise conversions between storage and compute vectors.
template <class T>
void launch_store(const typename Store<T>::C *src, long n_pad, T *dst,
                  cudaStream_t st);
template <class T>
void launch_load(const T *src, long n, typename Store<T>::C *dst,
                 cudaStream_t st);

// *out = sum of v[i]^2 for i < n (short vectors: one block, fixed order).
void launch_sumsq(const double *v, long n, double *out, cudaStream_t st);

// out = a * (ay - c * y) + b * yp (yp may be null; out may alias yp): one
// step of the scaled Chebyshev filter of the FP64 refinement.
void launch_cheb(const double *ay, const double *y, const double *yp, long n_pad, double a, double c, double b,
                 double *out, cudaStream_t st);
void launch_cheb(const zd *ay, const zd *y, const zd *yp, long n_pad, double a, double c, double b, zd *out,
                 cudaStream_t st);

// Smoothed uniform random vector (the breakdown restart of Gram-Schmidt);
// rows >= n are set to zero.
template <class C>
void launch_random(C *dst, long n, long n_pad, uint64_t seed, cudaStream_t st);

}  // namespace trlb

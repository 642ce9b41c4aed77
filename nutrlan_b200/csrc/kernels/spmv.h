// Built-in sparse operators (CSR and SELL-C-sigma, real and complex) and their
// fused product kernels.  The engine calls spmv_fused() when the user's
// `op` is trlx_matvec / trlx_zmatvec; the fused kernel produces y = A x and
// alpha = Re(x^H y) in one pass over the matrix (the reference computes the
// alpha dot separately after the callback, SRC/trlcore.c:1098-1108).
#pragma once

#include <cuda_runtime.h>

#include "lanczos_kernels.h"

namespace trlb {
struct Halo;
}

struct trlx_operator {
    int kind = 0;  // 0 real CSR, 1 real SELL-C-32, 2 complex CSR, 3 complex SELL-C-32
    int nrow = 0;
    long long nnz = 0;
    // CSR
    long long *row_ptr = nullptr;
    int *col = nullptr;
    void *val = nullptr;  // double or zd
    // SELL-C-32
    int nslice = 0;
    int sigma = 1;
    long long *slice_ptr = nullptr;  // offset of slice s (entries), nslice+1
    int *perm = nullptr;             // stored row -> original row (nullptr = identity)
    int device = -1;
    // Block-row distribution (trlx_dist_*_create): columns [0, nrow) are
    // this rank's rows, [nrow, nrow + halo entries) values received from
    // other ranks before every product.
    trlb::Halo *halo = nullptr;
    // Form of the Gram-Schmidt projection kernel (trlb::ProjectForm) for
    // solves with this operator over a 64-bit basis (FP64 / complex128) and
    // over a 32-bit basis (FP32 / complex64), set by trlx_operator_autotune
    // (0: the default form).
    int project_form = 0;
    int project_form32 = 0;
};

namespace trlb {

inline bool op_complex(const trlx_operator *A) { return A->kind == 2 || A->kind == 3; }
inline bool op_sell(const trlx_operator *A) { return A->kind == 1 || A->kind == 3; }

// y = A x and, if alpha_out != null, *alpha_out = Re(x^H y) (deterministic).
// x, y are compute vectors of n_pad rows (padding rows of y are written 0).
void spmv_fused_real(const trlx_operator *A, const double *x, double *y, long n_pad,
                     double *alpha_out, Scratch *s, cudaStream_t st);
void spmv_fused_cplx(const trlx_operator *A, const zd *x, zd *y, long n_pad,
                     double *alpha_out, Scratch *s, cudaStream_t st);

// Plain product with leading dimensions (used by trlx_matvec called directly).
void spmv_plain(const trlx_operator *A, const void *x, void *y, cudaStream_t st);

// Algorithmic bytes of one product (values + indices + row pointers + x + y).
double spmv_bytes(const trlx_operator *A);

// Returns the unused memory of the operators' device pools.
void trim_operator_pools();

// Distributed operators: gathers the values other ranks need from x (this
// rank's n_pad-row vector), exchanges halos over the operator's
// communicator and returns in *x_ext the vector to multiply (x's rows, then
// the halo), all ordered on st.  0 or an error code.
int halo_exchange(const trlx_operator *A, const double *x, cudaStream_t st, const double **x_ext);

}  // namespace trlb

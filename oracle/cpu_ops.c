/*
 * CPU operators for the reference library (test infrastructure / CPU
 * baseline only).  The reference's examples pass a C matvec callback; this
 * is the same kind of callback for CSR matrices, OpenMP-parallel over rows,
 * so the CPU baseline spends its time in the reference's own Lanczos code
 * and BLAS rather than in a Python callback.
 *
 * Usage: info.mvparam = &csr (struct cpu_csr); op = cpu_csr_matvec.
 */
#include <omp.h>

struct cpu_csr {
    int n;
    const long long *row_ptr;
    const int *col;
    const double *val; /* real: n values; complex: interleaved (re, im) */
};

void cpu_csr_matvec(const int nrow, const int ncol, const double *x, const int ldx,
                    double *y, const int ldy, void *mvparam) {
    const struct cpu_csr *A = (const struct cpu_csr *)mvparam;
    for (int j = 0; j < ncol; ++j) {
        const double *xj = x + (long)j * ldx;
        double *yj = y + (long)j * ldy;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nrow; ++i) {
            double s = 0.0;
            for (long long k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k) s += A->val[k] * xj[A->col[k]];
            yj[i] = s;
        }
    }
}

void cpu_zcsr_matvec(const int nrow, const int ncol, const double *x, const int ldx,
                     double *y, const int ldy, void *mvparam) {
    const struct cpu_csr *A = (const struct cpu_csr *)mvparam;
    for (int j = 0; j < ncol; ++j) {
        const double *xj = x + 2L * j * ldx;
        double *yj = y + 2L * j * ldy;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nrow; ++i) {
            double sr = 0.0, si = 0.0;
            for (long long k = A->row_ptr[i]; k < A->row_ptr[i + 1]; ++k) {
                const double ar = A->val[2 * k], ai = A->val[2 * k + 1];
                const double xr = xj[2 * A->col[k]], xi = xj[2 * A->col[k] + 1];
                sr += ar * xr - ai * xi;
                si += ar * xi + ai * xr;
            }
            yj[2 * i] = sr;
            yj[2 * i + 1] = si;
        }
    }
}

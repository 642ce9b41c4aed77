/* Complex BLAS-1 helpers that the reference's example programs call for
 * their own set-up (examples/test_ztrlan.c:rankk_init uses trl_zdotc,
 * trl_zaxpy and trl_zscal, which the reference declares in its internal
 * header INC/trl_map.h and defines in SRC/trlmap.c).  They are not part of
 * the solver's public API, so libtrlan_b200.so does not export them; the
 * examples are linked with this file instead.  Plain loops, host memory. */
typedef struct { double r, i; } trl_dcomplex;

void trl_zdotc(trl_dcomplex *ret, int n, trl_dcomplex *x, int incx, trl_dcomplex *y, int incy) {
    double sr = 0.0, si = 0.0;
    for (int k = 0; k < n; ++k) {
        const trl_dcomplex a = x[k * incx], b = y[k * incy];
        sr += a.r * b.r + a.i * b.i;
        si += a.r * b.i - a.i * b.r;
    }
    ret->r = sr;
    ret->i = si;
}

void trl_zaxpy(int n, trl_dcomplex a, trl_dcomplex *x, int incx, trl_dcomplex *y, int incy) {
    for (int k = 0; k < n; ++k) {
        const trl_dcomplex v = x[k * incx];
        y[k * incy].r += a.r * v.r - a.i * v.i;
        y[k * incy].i += a.r * v.i + a.i * v.r;
    }
}

void trl_zscal(int n, trl_dcomplex a, trl_dcomplex *x, int incx) {
    for (int k = 0; k < n; ++k) {
        const trl_dcomplex v = x[k * incx];
        x[k * incx].r = a.r * v.r - a.i * v.i;
        x[k * incx].i = a.r * v.i + a.i * v.r;
    }
}

"""ctypes driver for the reference library built under oracle/_ref.

Test infrastructure: runs the unmodified reference ``trlan``/``ztrlan`` with
numpy operators so that tests can compare the B200 engine against the
reference on identical inputs.  Parity is pinned by the reference's own
examples (examples/simple.c: diag((i+1)^2), n=1897, ned=5, maxlan=200;
examples/test_ztrlan.c: complex diag((i+1)^2)) and by analytic spectra.
"""
import ctypes as C
import os
import subprocess
import time

import numpy as np

from nutrlan_b200._abi import TrlInfo, MATVEC, declare_common

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libnutrlan_ref.so")
# Where the reference checkout lives: $TRLAN_REFERENCE, else the default path.
REF_ROOT = os.environ.get("TRLAN_REFERENCE", "/root/reference")
_LIB = None


def available():
    return os.path.exists(REF_SO)


def build(ref_root=None):
    """Compile the reference from its sources (only where they exist)."""
    ref_root = ref_root or REF_ROOT
    if os.path.isdir(ref_root):
        subprocess.run(["make", "-C", HERE, f"REF={ref_root}", "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    return available()


def load():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError(f"reference oracle not built: {REF_SO}")
        lib = C.CDLL(REF_SO)
        declare_common(lib)
        # Internal routines used for building-block parity tests.
        lib.dstqrb_.argtypes = [C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.POINTER(C.c_int)]
        lib.dstqrb_.restype = None
        lib.trl_get_eval.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        lib.trl_get_eval.restype = None
        lib.trl_tridiag.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        lib.trl_tridiag.restype = None
        lib.trl_shuffle_eig.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                        C.POINTER(TrlInfo), C.POINTER(C.c_int), C.c_int]
        lib.trl_shuffle_eig.restype = None
        lib.trl_convergence_test.argtypes = [C.c_int, C.c_void_p, C.c_void_p,
                                             C.POINTER(TrlInfo), C.c_void_p]
        lib.trl_convergence_test.restype = None
        lib.trl_sort_eig.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                     C.c_void_p]
        lib.trl_sort_eig.restype = None
        lib.trl_set_locking.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_double, C.POINTER(C.c_int)]
        lib.trl_set_locking.restype = None
        lib.dsort2.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        lib.dsort2.restype = None
        _LIB = lib
    return _LIB


def _real_op(matvec):
    def op(nrow, ncol, x, ldx, y, ldy, mvparam):
        for j in range(ncol):
            xv = np.ctypeslib.as_array(C.cast(x + 8 * j * ldx, C.POINTER(C.c_double)), (nrow,))
            yv = np.ctypeslib.as_array(C.cast(y + 8 * j * ldy, C.POINTER(C.c_double)), (nrow,))
            yv[:] = matvec(xv)
    return MATVEC(op)


def _cplx_op(matvec):
    def op(nrow, ncol, x, ldx, y, ldy, mvparam):
        for j in range(ncol):
            xv = np.ctypeslib.as_array(C.cast(x + 16 * j * ldx, C.POINTER(C.c_double)),
                                       (2 * nrow,)).view(np.complex128)
            yv = np.ctypeslib.as_array(C.cast(y + 16 * j * ldy, C.POINTER(C.c_double)),
                                       (2 * nrow,)).view(np.complex128)
            yv[:] = matvec(xv)
    return MATVEC(op)


def trlan(matvec, n, ned, maxlan, lohi=-1, tol=1.4901e-8, restart=1, maxmv=0, start=None,
          mev=None, lwrk=None, rfact=None, lib=None):
    """Reference trlan on a numpy operator; returns dict with eval, evec,
    res (wrk on exit), info and wall seconds."""
    lib = lib or load()
    mev = mev or ned + 1
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, lohi, ned, tol, restart, maxmv, None)
    if rfact is not None:
        lib.trl_set_restart(C.byref(info), rfact)
    evec = np.zeros((mev, n))
    if start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        evec[0] = start
    eval_ = np.zeros(mev)
    lwrk = lwrk if lwrk is not None else maxlan * (maxlan + 10)
    wrk = np.zeros(max(lwrk, 1))
    cb = _real_op(matvec)
    t0 = time.perf_counter()
    lib.trlan(cb, None, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, n, lwrk,
              wrk.ctypes.data)
    dt = time.perf_counter() - t0
    return dict(eval=eval_, evec=evec, res=wrk[:mev].copy(), info=info, seconds=dt)


def ztrlan(matvec, n, ned, maxlan, lohi=-1, tol=1.4901e-8, restart=1, maxmv=0, start=None,
           mev=None, lib=None):
    lib = lib or load()
    mev = mev or ned + 1
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, lohi, ned, tol, restart, maxmv, None)
    evec = np.zeros((mev, n), dtype=np.complex128)
    if start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        evec[0] = start
    eval_ = np.zeros(mev)
    nmis = maxlan * (maxlan + 10) + n * maxlan
    misc = np.zeros(nmis, dtype=np.complex128)
    ldwrk = maxlan * (maxlan + 10)
    dwrk = np.zeros(ldwrk)
    cb = _cplx_op(matvec)
    t0 = time.perf_counter()
    lib.ztrlan(cb, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, n,
               misc.ctypes.data, nmis, dwrk.ctypes.data, ldwrk)
    dt = time.perf_counter() - t0
    return dict(eval=eval_, evec=evec, res=misc[:mev].real.copy(), info=info, seconds=dt)


# ---------------------------------------------------------------------------
# Reference trlan with a compiled (OpenMP) CSR operator: the CPU baseline.
class _CpuCSR(C.Structure):
    _fields_ = [("n", C.c_int), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
                ("val", C.c_void_p)]


_OPS = None


def cpu_ops():
    global _OPS
    if _OPS is None:
        _OPS = C.CDLL(os.path.join(HERE, "_ref", "libcpuops.so"))
    return _OPS


def trlan_csr(A, ned, maxlan, lohi=-1, tol=1.4901e-8, restart=1, maxmv=0, start=None,
              mev=None, lib=None):
    """Reference trlan/ztrlan on a CSR operator applied by compiled C code."""
    lib = lib or load()
    ops = cpu_ops()
    cplx = np.iscomplexobj(A.val)
    val = np.ascontiguousarray(A.val)
    st = _CpuCSR(A.n, A.row_ptr.ctypes.data, A.col.ctypes.data, val.ctypes.data)
    fn = C.cast(ops.cpu_zcsr_matvec if cplx else ops.cpu_csr_matvec, MATVEC)
    mev = mev or ned + 1
    n = A.n
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, lohi, ned, tol, restart, maxmv, None)
    info.mvparam = C.addressof(st)
    dtype = np.complex128 if cplx else np.float64
    evec = np.zeros((mev, n), dtype=dtype)
    if start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        evec[0] = start
    eval_ = np.zeros(mev)
    t0 = time.perf_counter()
    if cplx:
        nmis = maxlan * (maxlan + 10) + n * maxlan
        misc = np.zeros(nmis, dtype=np.complex128)
        ldwrk = maxlan * (maxlan + 10)
        dwrk = np.zeros(ldwrk)
        lib.ztrlan(fn, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, n,
                   misc.ctypes.data, nmis, dwrk.ctypes.data, ldwrk)
    else:
        lwrk = maxlan * (maxlan + 10)
        wrk = np.zeros(lwrk)
        lib.trlan(fn, None, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, n,
                  lwrk, wrk.ctypes.data)
    dt = time.perf_counter() - t0
    res = None if cplx else wrk[:mev].copy()  # ztrlan keeps its residual norms internal
    return dict(eval=eval_, evec=evec, res=res, info=info, seconds=dt)

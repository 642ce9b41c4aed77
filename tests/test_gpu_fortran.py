"""trlan_ / ztrlan_ (include/ftrlan.h) called the way a Fortran program calls
them: scalars by reference and an operator op(nrow, ncol, x, ldx, y, ldy)
whose arguments are all pointers.  Operator: the diagonal matrix of the
reference's examples (diag((i+1)^2), n = 1000), smallest eigenvalues
(i+1)^2."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import TrlInfo, load

pytestmark = pytest.mark.gpu

P = C.POINTER
FOP = C.CFUNCTYPE(None, P(C.c_int), P(C.c_int), C.c_void_p, P(C.c_int), C.c_void_p, P(C.c_int))


def _i(v):
    return C.byref(C.c_int(v))


def _declare(lib):
    lib.trl_init_info_.argtypes = [P(TrlInfo), P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_double),
                                   P(C.c_int), P(C.c_int)]
    lib.trl_init_info_.restype = None
    lib.trl_set_iguess_.argtypes = [P(TrlInfo), P(C.c_int), P(C.c_int), P(C.c_int), C.c_char_p, C.c_size_t]
    lib.trl_set_iguess_.restype = None
    lib.trlan_.argtypes = [FOP, P(TrlInfo), P(C.c_int), P(C.c_int), C.c_void_p, C.c_void_p, P(C.c_int),
                           P(C.c_int), C.c_void_p]
    lib.trlan_.restype = None
    lib.ztrlan_.argtypes = [FOP, P(TrlInfo), P(C.c_int), P(C.c_int), C.c_void_p, C.c_void_p, P(C.c_int),
                            C.c_void_p, P(C.c_int), C.c_void_p, P(C.c_int)]
    lib.ztrlan_.restype = None
    return lib


@pytest.mark.parametrize("cplx", [False, True])
def test_fortran_solver_entry_points(cplx):
    lib = _declare(load())
    n, ned, mev = 1000, 6, 8
    d = (np.arange(n) + 1.0) ** 2
    seen = []

    def op(nrow, ncol, x, ldx, y, ldy):
        nr, nc, lx, ly = nrow[0], ncol[0], ldx[0], ldy[0]
        seen.append((nr, nc, lx, ly))
        dt = np.complex128 if cplx else np.float64
        w = 16 if cplx else 8
        for j in range(nc):
            xv = np.ctypeslib.as_array(C.cast(x + w * j * lx, P(C.c_double)), (nr * (2 if cplx else 1),)).view(dt)
            yv = np.ctypeslib.as_array(C.cast(y + w * j * ly, P(C.c_double)), (nr * (2 if cplx else 1),)).view(dt)
            yv[:] = d * xv

    cb = FOP(op)
    info = TrlInfo()
    lib.trl_init_info_(C.byref(info), _i(n), _i(40), _i(-1), _i(ned), C.byref(C.c_double(1e-9)), _i(1),
                       _i(20000))
    blank = b" " * 8
    lib.trl_set_iguess_(C.byref(info), _i(0), _i(1), _i(0), blank, len(blank))
    rng = np.random.default_rng(3)
    eval_ = np.zeros(mev)
    if cplx:
        evec = np.zeros((mev, n), dtype=np.complex128)
        evec[0] = rng.random(n) + 1j * rng.random(n)
        misc = np.zeros(mev, dtype=np.complex128)
        lib.ztrlan_(cb, C.byref(info), _i(n), _i(mev), eval_.ctypes.data, evec.ctypes.data, _i(n),
                    misc.ctypes.data, _i(mev), None, _i(0))
    else:
        evec = np.zeros((mev, n))
        evec[0] = rng.random(n)
        wrk = np.zeros(mev)
        lib.trlan_(cb, C.byref(info), _i(n), _i(mev), eval_.ctypes.data, evec.ctypes.data, _i(n), _i(mev),
                   wrk.ctypes.data)
    assert info.stat == 0 and info.nec >= ned
    np.testing.assert_allclose(np.sort(eval_[:ned]), d[:ned], rtol=1e-9)
    assert seen and all(s[0] == n and s[1] == 1 for s in seen)
    for lam, v in zip(eval_[:ned], evec[:ned]):
        assert np.linalg.norm(d * v - lam * v) <= 1e-9 * d[-1] * 1.01

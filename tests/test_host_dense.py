"""The engine's host FP64 building blocks against the reference's own
routines (dstqrb_, trl_get_eval, trl_tridiag, trl_shuffle_eig,
trl_convergence_test, trl_sort_eig, trl_set_locking, dsort2), called in the
reference library built under oracle/_ref.  CPU only."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import TrlInfo


def P(a):
    return a.ctypes.data


@pytest.mark.parametrize("nd,locked", [(2, 0), (5, 0), (20, 3), (64, 0), (128, 7)])
def test_get_eval_matches_dstqrb(lib, reflib, nd, locked):
    rng = np.random.default_rng(nd + locked)
    a = rng.standard_normal(nd)
    b = np.abs(rng.standard_normal(nd))
    lam1, res1, lam2, res2 = (np.zeros(nd) for _ in range(4))
    w = np.zeros(10 * nd)
    ierr = C.c_int(0)
    reflib.trl_get_eval(nd, locked, P(a), P(b), P(lam1), P(res1), P(w), 10 * nd, C.byref(ierr))
    assert ierr.value == 0
    assert lib.trlx_host_get_eval(nd, locked, P(a), P(b), P(lam2), P(res2)) == 0
    scale = np.max(np.abs(lam1)) + 1
    np.testing.assert_allclose(lam2, lam1, atol=1e-13 * scale * nd)
    np.testing.assert_allclose(res2, res1, atol=1e-13 * scale * nd)


def test_get_eval_degenerate_and_split(lib, reflib):
    # Repeated diagonal entries and zero couplings (invariant subspaces).
    a = np.array([1.0, 1.0, 2.0, 2.0, 2.0, 3.0, 1.0, 5.0])
    b = np.array([0.0, 0.5, 0.0, 1e-12, 0.3, 0.0, 0.7, 0.2])
    nd = a.size
    lam1, res1, lam2, res2 = (np.zeros(nd) for _ in range(4))
    w = np.zeros(10 * nd)
    ierr = C.c_int(0)
    reflib.trl_get_eval(nd, 0, P(a), P(b), P(lam1), P(res1), P(w), 10 * nd, C.byref(ierr))
    lib.trlx_host_get_eval(nd, 0, P(a), P(b), P(lam2), P(res2))
    np.testing.assert_allclose(lam2, lam1, atol=1e-13)
    np.testing.assert_allclose(res2, res1, atol=1e-13)


@pytest.mark.parametrize("nd", [1, 2, 3, 10, 33, 64])
def test_arrow_to_tridiag_matches_dsytrd(lib, reflib, nd):
    rng = np.random.default_rng(100 + nd)
    a = rng.standard_normal(nd)
    b = rng.standard_normal(nd)
    rot1, rot2 = np.zeros(nd * nd), np.zeros(nd * nd)
    af1, bf1, af2, bf2 = (np.zeros(nd) for _ in range(4))
    w = np.zeros(64 * nd)
    ierr = C.c_int(0)
    reflib.trl_tridiag(nd, P(a), P(b), P(rot1), P(af1), P(bf1), P(w), 64 * nd, C.byref(ierr))
    assert lib.trlx_host_arrow_to_tridiag(nd, P(a), P(b), P(rot2), P(af2), P(bf2)) == 0
    np.testing.assert_allclose(af2, af1, atol=1e-11)
    np.testing.assert_allclose(np.abs(bf2), np.abs(bf1), atol=1e-11)
    Q = rot2.reshape(nd, nd).T
    # Rotation fixes the last coordinate and reproduces the arrow matrix.
    assert np.allclose(Q[-1], np.eye(nd)[-1]) and np.allclose(Q[:, -1], np.eye(nd)[-1])
    Aarr = np.diag(a)
    Aarr[-1, :-1] = b[:-1]
    Aarr[:-1, -1] = b[:-1]
    T = np.diag(af2) + np.diag(bf2[:-1], 1) + np.diag(bf2[:-1], -1)
    np.testing.assert_allclose(Q @ T @ Q.T, Aarr, atol=1e-12 * (1 + np.abs(Aarr).max()))


def test_sym_eig_against_numpy(lib):
    rng = np.random.default_rng(7)
    for n in (1, 4, 31, 96):
        M = rng.standard_normal((n, n))
        M = M + M.T
        A = np.asfortranarray(M.copy())
        w = np.zeros(n)
        assert lib.trlx_host_sym_eig(n, P(A), n, P(w)) == 0
        np.testing.assert_allclose(w, np.linalg.eigvalsh(M), atol=1e-12 * n)
        np.testing.assert_allclose(M @ A, A * w, atol=1e-11 * n)


def _info(nd, ned, maxlan, lohi, restart, rng, nloop=0):
    info = TrlInfo()
    info.lohi, info.ned, info.maxlan, info.klan = lohi, ned, maxlan, maxlan
    info.nec = int(rng.integers(0, max(1, ned // 2)))
    info.tol, info.anrm = 1e-8, 10.0
    info.matvec, info.maxmv = 500, 100000
    info.restart, info.nloop, info.locked = restart, nloop, 0
    info.crat, info.cfac, info.ptres = 0.9, 0.5, 1e-3
    info.trgt, info.tres, info.avgm, info.k = 0.0, 1e-3, 10.0, 5
    info.rfact = 1.5
    return info


@pytest.mark.parametrize("restart", [0, 1, 2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("lohi", [-1, 1, 0])
def test_shuffle_eig_matches_reference(lib, reflib, restart, lohi):
    rng = np.random.default_rng(1000 * restart + lohi + 5)
    for trial in range(6):
        nd = int(rng.integers(6, 120))
        ned = int(rng.integers(1, max(2, nd // 3)))
        lam = np.sort(rng.standard_normal(nd) * 3)
        res = 10.0 ** rng.uniform(-12, -1, nd)
        tind = int(rng.integers(0, nd))
        for nloop in (0, 3):
            i1 = _info(nd, ned, max(nd, 8), lohi, restart, rng, nloop)
            i1.trgt = lam[tind]
            i2 = TrlInfo.from_buffer_copy(i1)
            l1, r1, l2, r2 = lam.copy(), res.copy(), lam.copy(), res.copy()
            k1, k2 = C.c_int(0), C.c_int(0)
            reflib.trl_shuffle_eig(nd, nd, P(l1), P(r1), C.byref(i1), C.byref(k1), 0)
            lib.trlx_host_shuffle_eig(nd, nd, P(l2), P(r2), C.byref(i2), C.byref(k2), 0)
            assert k1.value == k2.value, (trial, nloop)
            np.testing.assert_array_equal(l1[:k1.value], l2[:k2.value])
            np.testing.assert_array_equal(r1[:k1.value], r2[:k2.value])
            assert i1.klan == i2.klan and i1.lohi == i2.lohi


@pytest.mark.parametrize("lohi", [-1, 1, 0, -2, -3, -4])
def test_convergence_test_matches_reference(lib, reflib, lohi):
    rng = np.random.default_rng(50 + lohi)
    for trial in range(10):
        nd = int(rng.integers(4, 80))
        lam = np.sort(rng.standard_normal(nd))
        res = 10.0 ** rng.uniform(-14, 0, nd)
        res[: int(rng.integers(0, nd))] = 1e-15
        i1 = _info(nd, 5, nd, lohi, 1, rng)
        i1.ref = 0.1
        i1.tmv = 100
        i2 = TrlInfo.from_buffer_copy(i1)
        l1, r1, l2, r2 = lam.copy(), res.copy(), lam.copy(), res.copy()
        w1, w2 = np.zeros(2 * nd), np.zeros(2 * nd)
        reflib.trl_convergence_test(nd, P(l1), P(r1), C.byref(i1), P(w1))
        lib.trlx_host_convergence_test(nd, P(l2), P(r2), C.byref(i2), P(w2))
        for f in ("nec", "trgt", "tres", "anrm", "crat", "cfac", "tmv", "ptres"):
            assert getattr(i1, f) == getattr(i2, f), f
        np.testing.assert_array_equal(w1, w2)


@pytest.mark.parametrize("lohi", [-1, 1, 0, -2, -3, -4])
def test_sort_eig_matches_reference(lib, reflib, lohi):
    rng = np.random.default_rng(9 + lohi)
    nd, nec = 40, 7
    lam = rng.standard_normal(nd)
    res = np.abs(rng.standard_normal(nd))
    l1, r1, l2, r2 = lam.copy(), res.copy(), lam.copy(), res.copy()
    reflib.trl_sort_eig(nd, lohi, nec, 0.3, P(l1), P(r1))
    lib.trlx_host_sort_eig(nd, lohi, nec, 0.3, P(l2), P(r2))
    np.testing.assert_array_equal(l1, l2)
    np.testing.assert_array_equal(r1, r2)


def test_set_locking_matches_reference(lib, reflib):
    rng = np.random.default_rng(3)
    for trial in range(20):
        nlam, jnd = int(rng.integers(2, 30)), 40
        lam = rng.standard_normal(nlam)
        res = np.where(rng.random(nlam) < 0.4, 1e-18, rng.random(nlam))
        yy = rng.standard_normal(jnd * nlam)
        a = [lam.copy(), res.copy(), yy.copy()]
        b = [lam.copy(), res.copy(), yy.copy()]
        k1, k2 = C.c_int(0), C.c_int(0)
        reflib.trl_set_locking(jnd, nlam, P(a[0]), P(a[1]), P(a[2]), 5.0, C.byref(k1))
        lib.trlx_host_set_locking(jnd, nlam, P(b[0]), P(b[1]), P(b[2]), 5.0, C.byref(k2))
        assert k1.value == k2.value
        for u, v in zip(a, b):
            np.testing.assert_array_equal(u, v)


def test_shell_sort_tie_order_matches_reference(lib, reflib):
    rng = np.random.default_rng(11)
    key = rng.integers(0, 5, 57).astype(float)
    other = np.arange(57, dtype=float)
    k1, o1, k2, o2 = key.copy(), other.copy(), key.copy(), other.copy()
    reflib.dsort2(57, P(k1), P(o1))
    lib.trlx_host_sort2(57, P(k2), P(o2))
    np.testing.assert_array_equal(k1, k2)
    np.testing.assert_array_equal(o1, o2)


def test_hermitian_jacobi_matches_numpy(lib):
    """trlx_host_herm_eig (used by the FP64 refinement of complex bases)
    against numpy.linalg.eigh: eigenvalues, unitary eigenvectors, A Z = Z w,
    including a degenerate pair."""
    import ctypes as C
    f = lib.trlx_host_herm_eig
    f.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]
    f.restype = C.c_int
    rng = np.random.default_rng(4)
    for n in (1, 2, 5, 16, 33):
        M = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        A = M + M.conj().T
        if n >= 5:  # a degenerate pair
            Q = np.linalg.qr(M)[0]
            d = np.sort(rng.standard_normal(n))
            d[1] = d[2]
            A = (Q * d) @ Q.conj().T
            A = 0.5 * (A + A.conj().T)
        Af = np.asfortranarray(A)
        w = np.zeros(n)
        Z = np.zeros((n, n), dtype=np.complex128, order="F")
        assert f(n, Af.ctypes.data, n, w.ctypes.data, Z.ctypes.data, n) == 0
        np.testing.assert_allclose(w, np.linalg.eigvalsh(A), rtol=1e-12, atol=1e-12 * np.abs(w).max())
        np.testing.assert_allclose(Z.conj().T @ Z, np.eye(n), atol=1e-12)
        np.testing.assert_allclose(A @ Z, Z * w, atol=1e-11 * max(1.0, np.abs(w).max()))

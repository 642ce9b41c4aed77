"""Kernel-level parity through the C ABI against the numpy oracle
(oracle/kernels_np.py): the Gram-Schmidt projection trlx_g_dot /
trlx_zg_dot (reference trl_g_dot_ / ztrl_g_dot_) on arbitrary leading
dimensions and unaligned columns, and the built-in sparse operators
(CSR, SELL-C-32, complex CSR) against a CSR product.  Tolerance: FP64
reductions in a different order, 1e-13 relative to the operand scale."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import load, operators as ops, DeviceOperator
from oracle import kernels_np as K

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,m1,m2,ld1,ld2,off", [
    (1000, 5, 3, 1000, 1003, 0),
    (4097, 0, 7, 4097, 4100, 1),     # v1 empty, odd leading dimension, unaligned
    (4097, 9, 0, 4101, 4097, 1),
    (65536, 40, 24, 65536, 65540, 0),
    (33, 1, 1, 33, 40, 3),
    (300000, 130, 2, 300000, 300001, 0),   # more than 128 columns
])
def test_g_dot_matches_numpy(n, m1, m2, ld1, ld2, off):
    lib = load()
    rng = np.random.default_rng(n + m1)
    v1 = rng.standard_normal((max(m1, 1), ld1)) if m1 else np.zeros((1, ld1))
    v2 = rng.standard_normal((max(m2, 1), ld2)) if m2 else np.zeros((1, ld2))
    rr = rng.standard_normal(n)
    buf1 = dev(np.concatenate([np.zeros(off), v1.ravel()]))
    buf2 = dev(np.concatenate([np.zeros(off), v2.ravel()]))
    drr = dev(rr)
    dw = torch.zeros(m1 + m2, dtype=torch.float64, device="cuda")
    rc = lib.trlx_g_dot(n, buf1.data_ptr() + 8 * off, ld1, m1, buf2.data_ptr() + 8 * off, ld2, m2,
                        drr.data_ptr(), dw.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    want = K.g_dot(v1[:, :n].T, m1, v2[:, :n].T, m2, rr)
    got = dw.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * np.sqrt(n) * 4)
    # Deterministic: a second call gives identical bits.
    dw2 = torch.zeros_like(dw)
    lib.trlx_g_dot(n, buf1.data_ptr() + 8 * off, ld1, m1, buf2.data_ptr() + 8 * off, ld2, m2,
                   drr.data_ptr(), dw2.data_ptr(), None)
    torch.cuda.synchronize()
    assert torch.equal(dw, dw2)


def test_zg_dot_matches_numpy():
    lib = load()
    rng = np.random.default_rng(5)
    n, m1, m2, ld = 5003, 6, 11, 5010
    v1 = rng.standard_normal((m1, ld)) + 1j * rng.standard_normal((m1, ld))
    v2 = rng.standard_normal((m2, ld)) + 1j * rng.standard_normal((m2, ld))
    rr = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    d1, d2, dr = dev(v1), dev(v2), dev(rr)
    dw = torch.zeros(m1 + m2, dtype=torch.complex128, device="cuda")
    assert lib.trlx_zg_dot(n, d1.data_ptr(), ld, m1, d2.data_ptr(), ld, m2, dr.data_ptr(),
                           dw.data_ptr(), None) == 0
    torch.cuda.synchronize()
    want = K.g_dot(v1[:, :n].T, m1, v2[:, :n].T, m2, rr)
    np.testing.assert_allclose(dw.cpu().numpy(), want, atol=1e-12)


def test_g_dot_argument_errors():
    lib = load()
    x = torch.zeros(100, dtype=torch.float64, device="cuda")
    w = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert lib.trlx_g_dot(100, x.data_ptr(), 50, 2, x.data_ptr(), 100, 0, x.data_ptr(),
                          w.data_ptr(), None) == -201
    assert lib.trlx_g_dot(100, x.data_ptr(), 100, 0, x.data_ptr(), 100, 0, x.data_ptr(),
                          w.data_ptr(), None) == 0
    # A rank with no local rows: the partial products are zeros, not an error
    # (the reference's ddot of length 0 is 0).
    for f in (lib.trlx_g_dot, lib.trlx_zg_dot):
        w.fill_(7.0)
        assert f(0, x.data_ptr(), 0, 1, x.data_ptr(), 0, 1, x.data_ptr(), w.data_ptr(), None) == 0
        torch.cuda.synchronize()
        got = w.cpu().numpy()
        assert np.all(got[:4 if f is lib.trlx_zg_dot else 2] == 0.0)


@pytest.mark.parametrize("fmt", ["csr", "sell"])
@pytest.mark.parametrize("family", ["laplace", "laplace64", "anderson", "ragged"])
def test_builtin_operator_matches_csr_product(fmt, family):
    lib = load()
    if family == "laplace":
        A = ops.laplacian_2d(37)
    elif family == "laplace64":  # n multiple of 256: the row-tile CSR kernel
        A = ops.laplacian_2d(64)
    elif family == "anderson":
        A = ops.anderson_3d(13, seed=3)
    else:  # rows of very different lengths, including empty rows
        rng = np.random.default_rng(2)
        n = 3001
        lens = rng.integers(0, 40, n)
        lens[::97] = 0
        lens[5] = 900
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        col = rng.integers(0, n, rp[-1]).astype(np.int32)
        val = rng.standard_normal(rp[-1])
        A = ops.CSR(n, rp, col, val)
    x = np.random.default_rng(9).standard_normal(A.n)
    want = K.csr_matvec(A.row_ptr, A.col, A.val, x)
    with DeviceOperator(A, fmt=fmt, sigma=64 if family == "ragged" else 1) as op:
        dx, dy = dev(x), torch.zeros(A.n, dtype=torch.float64, device="cuda")
        lib.trlx_matvec.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                    C.c_void_p]
        lib.trlx_matvec(A.n, 1, dx.data_ptr(), A.n, dy.data_ptr(), A.n, op.handle)
        torch.cuda.synchronize()
    np.testing.assert_allclose(dy.cpu().numpy(), want, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("fmt,sigma", [("zcsr", 1), ("zsell", 1), ("zsell", 16)])
def test_complex_operator_matches_csr_product(fmt, sigma):
    lib = load()
    A = ops.peierls_2d(32, phi=1.0 / 8.0)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(A.n) + 1j * rng.standard_normal(A.n)
    want = K.csr_matvec(A.row_ptr, A.col, A.val, x)
    with DeviceOperator(A, fmt=fmt, sigma=sigma) as op:
        assert op.fmt == fmt
        dx, dy = dev(x), torch.zeros(A.n, dtype=torch.complex128, device="cuda")
        lib.trlx_zmatvec.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                     C.c_void_p]
        lib.trlx_zmatvec(A.n, 1, dx.data_ptr(), A.n, dy.data_ptr(), A.n, op.handle)
        torch.cuda.synchronize()
    np.testing.assert_allclose(dy.cpu().numpy(), want, atol=1e-12)
    # Hermitian: x^H A x is real
    assert abs(np.vdot(x, want).imag) < 1e-9 * abs(np.vdot(x, want))


@pytest.mark.parametrize("sigma", [1, 64])
def test_complex_sell_ragged_rows_match_csr_product(sigma):
    """Complex SELL-C-32 on rows of very different lengths (empty rows, one
    row of 900 entries; sigma = 64 sorts rows within windows and stores the
    permutation) against the CSR product on the host."""
    lib = load()
    rng = np.random.default_rng(12)
    n = 2999
    lens = rng.integers(0, 40, n)
    lens[::89] = 0
    lens[7] = 900
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col = rng.integers(0, n, rp[-1]).astype(np.int32)
    val = rng.standard_normal(rp[-1]) + 1j * rng.standard_normal(rp[-1])
    A = ops.CSR(n, rp, col, val)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    want = K.csr_matvec(rp, col, val, x)
    with DeviceOperator(A, fmt="zsell", sigma=sigma) as op:
        assert op.nnz >= rp[-1]
        dx, dy = dev(x), torch.zeros(n, dtype=torch.complex128, device="cuda")
        lib.trlx_zmatvec.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                     C.c_void_p]
        lib.trlx_zmatvec(n, 1, dx.data_ptr(), n, dy.data_ptr(), n, op.handle)
        # A complex operator is not a real one: trlx_matvec leaves y alone.
        dz = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
        lib.trlx_matvec.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        lib.trlx_matvec(n, 1, dz.data_ptr(), n, dz.data_ptr(), n, op.handle)
        torch.cuda.synchronize()
    np.testing.assert_allclose(dy.cpu().numpy(), want, rtol=1e-13, atol=1e-12)
    assert torch.all(dz == 7.0)

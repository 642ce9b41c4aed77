"""Host-buffer paths at sizes that go through the pipelined pinned-staging
copies (copies of 4 MB and more from pageable host memory).

* A solve with a host evec (start vector in, Ritz vectors and the last
  Lanczos vector out, leading dimension larger than nrow) returns exactly
  what the same solve returns with a device evec, and leaves the rows past
  nrow of every column alone: once with columns that fit one staging buffer
  (several whole columns per chunk) and once with columns larger than one
  (each column split over chunks).
* Operators built from host arrays and from device arrays are the same
  operator: identical products, and for SELL-C-32 the padded entry count of
  the layout (slices of 32 rows, width = longest row of the slice, rows
  sorted by decreasing length inside windows of sigma rows).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from nutrlan_b200 import operators as ops, DeviceOperator
from nutrlan_b200._abi import TrlInfo
from nutrlan_b200._lib import load, TrlxOptions
from oracle import kernels_np as K

pytestmark = pytest.mark.gpu

SENTINEL = 7.25


def _solve(op, n, lde, ned, maxlan, maxmv, start, on_device):
    lib = load()
    mev = ned + 1
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, -1, ned, 1e-8, 1, maxmv, None)
    info.mvparam = op.handle.value
    lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
    eval_ = np.zeros(mev)
    wrk = np.zeros(mev)
    opts = TrlxOptions()
    lib.trlx_default_options(C.byref(opts))
    if on_device:
        ev = torch.full((mev, lde), SENTINEL, dtype=torch.float64, device="cuda")
        ev[0, :n] = torch.as_tensor(start, device="cuda")
        torch.cuda.synchronize()
        ptr = ev.data_ptr()
    else:
        ev = np.full((mev, lde), SENTINEL)
        ev[0, :n] = start
        ptr = ev.ctypes.data
    lib.trlx_trlan(op.applier, None, C.byref(info), n, mev, eval_.ctypes.data, ptr, lde, mev,
                   wrk.ctypes.data, C.byref(opts))
    torch.cuda.synchronize()
    if on_device:
        ev = ev.cpu().numpy()
    return info, eval_, ev


@pytest.mark.parametrize("L,ned,maxlan", [(900, 4, 24),     # 6.5 MB columns: whole columns per chunk
                                          (1700, 2, 16)])   # 23 MB columns: split over chunks
def test_host_evec_solve_equals_device_evec_solve(L, ned, maxlan):
    A = ops.laplacian_2d(L)
    n = A.n
    lde = n + 5
    start = ops.start_vector(n, seed=31)
    with DeviceOperator(A, fmt="sell") as op:
        ih, eh, vh = _solve(op, n, lde, ned, maxlan, 2 * maxlan, start, on_device=False)
        idv, ed, vd = _solve(op, n, lde, ned, maxlan, 2 * maxlan, start, on_device=True)
    assert ih.stat == idv.stat
    assert ih.matvec == idv.matvec > 0
    assert ih.nec == idv.nec
    np.testing.assert_array_equal(eh, ed)
    # Column 0..ned: Ritz vectors and, after them, the last Lanczos vector.
    np.testing.assert_array_equal(vh[:, :n], vd[:, :n])
    assert np.all(vh[:, n:] == SENTINEL)
    assert np.all(np.isfinite(vh[:, :n])) and np.linalg.norm(vh[0, :n]) > 0.5


def _padded_sell_entries(rp, sigma):
    lens = np.diff(rp)
    n = lens.size
    order = np.arange(n)
    if sigma > 1:
        for w0 in range(0, n, sigma):
            w = lens[w0:w0 + sigma]
            order[w0:w0 + sigma] = w0 + np.argsort(-w, kind="stable")
    slens = np.zeros(-(-n // 32) * 32, dtype=np.int64)
    slens[:n] = lens[order]
    return int(32 * slens.reshape(-1, 32).max(axis=1).sum())


def _matvec(lib, handle, x):
    dx = torch.as_tensor(x, device="cuda")
    dy = torch.zeros_like(dx)
    lib.trlx_matvec.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    lib.trlx_matvec(x.size, 1, dx.data_ptr(), x.size, dy.data_ptr(), x.size, handle)
    torch.cuda.synchronize()
    return dy.cpu().numpy()


def _ragged(n, seed):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 24, n)
    lens[::101] = 0
    lens[7] = 700
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col = rng.integers(0, n, rp[-1]).astype(np.int32)
    return ops.CSR(n, rp, col, rng.standard_normal(rp[-1]))


@pytest.mark.parametrize("family,sigma", [("anderson", 1), ("ragged", 1), ("ragged", 64)])
def test_operators_from_host_and_device_arrays_agree(family, sigma):
    lib = load()
    A = ops.anderson_3d(100, seed=5) if family == "anderson" else _ragged(1_000_003, 8)
    n = A.n
    rp = np.ascontiguousarray(A.row_ptr, np.int64)
    ci = np.ascontiguousarray(A.col, np.int32)
    va = np.ascontiguousarray(A.val, np.float64)
    drp, dci, dva = (torch.as_tensor(a, device="cuda") for a in (rp, ci, va))
    x = np.random.default_rng(3).standard_normal(n)
    want = K.csr_matvec(rp, ci, va, x)
    ys = {}
    for name, create, args in [
        ("sell_host", lib.trlx_sell_create, (rp.ctypes.data, ci.ctypes.data, va.ctypes.data, sigma, 0)),
        ("sell_dev", lib.trlx_sell_create, (drp.data_ptr(), dci.data_ptr(), dva.data_ptr(), sigma, 1)),
        ("csr_host", lib.trlx_csr_create, (rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 0)),
        ("csr_dev", lib.trlx_csr_create, (drp.data_ptr(), dci.data_ptr(), dva.data_ptr(), 1)),
    ]:
        h = C.c_void_p()
        assert create(n, *args, C.byref(h)) == 0, name
        try:
            if name.startswith("sell"):
                assert lib.trlx_operator_nnz(h) == _padded_sell_entries(rp, sigma), name
            ys[name] = _matvec(lib, h, x)
        finally:
            lib.trlx_operator_destroy(h)
    np.testing.assert_array_equal(ys["sell_host"], ys["sell_dev"])
    np.testing.assert_array_equal(ys["csr_host"], ys["csr_dev"])
    np.testing.assert_allclose(ys["sell_host"], want, rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(ys["csr_host"], want, rtol=1e-13, atol=1e-12)

"""Failure paths of the solve, against the reference library on the same
inputs (host operator, host evec):

* an operator that returns NaN (at its 30th application) or Inf (at its
  first): trl_orth's norm check gives stat -102 after the same number of
  applications (SRC/trlcore.c:1865-1869);
* an invariant subspace: a diagonal operator with only a few distinct
  values and the all-ones start vector spans its Krylov space in a few
  steps, so classical Gram-Schmidt must replace the next vector by a
  random one (SRC/trlcore.c:3049-3086): both libraries report nrand > 0,
  stat 0, nec >= ned, and every converged value is an eigenvalue (the
  random vectors differ: the reference draws them from drand48 seeded by
  clock(), this library from a seeded counter-based stream, so which copies
  of a repeated eigenvalue are found is not compared);
* checkpoint files that cannot be resumed (trl_read_checkpoint,
  SRC/trlaux.c:935-1010): another problem size (-213), more vectors than
  maxlan holds (-214), a truncated file (-215).  The reference looks for
  the file under the rank number alone (its trl_pe_filename passes the
  output buffer as a %s argument of the same sprintf, so the prefix is lost
  with this C library); this library uses prefix + rank.  Both names are
  written."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

from nutrlan_b200 import operators as ops, load
from nutrlan_b200._abi import TrlInfo, MATVEC

pytestmark = pytest.mark.gpu


def host_op(fn):
    def op(nrow, ncol, x, ldx, y, ldy, mvparam):
        for j in range(ncol):
            xv = np.ctypeslib.as_array(C.cast(x + 8 * j * ldx, C.POINTER(C.c_double)), (nrow,))
            yv = np.ctypeslib.as_array(C.cast(y + 8 * j * ldy, C.POINTER(C.c_double)), (nrow,))
            yv[:] = fn(xv)
    return MATVEC(op)


def run(lib, fn, n, ned, maxlan, start, mev=None, maxmv=5000, guess=1, cpf=None):
    mev = mev or ned + 1
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, -1, ned, 1.4901e-8, 1, maxmv, None)
    info.verbose = -1
    lib.trl_set_iguess(C.byref(info), 0, guess, 0, cpf)
    evec = np.zeros((mev, n))
    if start is not None:
        evec[0] = start
    eval_ = np.zeros(mev)
    wrk = np.zeros(maxlan * (maxlan + 10))
    cb = host_op(fn)
    lib.trlan(cb, None, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, n, wrk.size, wrk.ctypes.data)
    return info, eval_


def counting(A, at, value):
    calls = [0]

    def fn(x):
        calls[0] += 1
        y = A.matvec(x)
        if calls[0] == at:
            y[5] = value
        return y
    return fn


@pytest.mark.parametrize("at,value", [(30, np.nan), (1, np.inf), (7, -np.inf)])
def test_non_finite_operator_gives_reference_status(reflib, at, value):
    A = ops.laplacian_2d(40, diag=ops.uniform01(3, np.arange(1600, dtype=np.uint64)))
    x0 = ops.start_vector(A.n)
    got = [run(L, counting(A, at, value), A.n, 6, 40, x0)[0] for L in (reflib, load())]
    assert got[0].stat == got[1].stat == -102, (got[0].stat, got[1].stat)
    assert got[0].matvec == got[1].matvec == at


@pytest.mark.parametrize("nd,ned,maxlan", [(3, 5, 20), (4, 6, 20), (2, 4, 16), (5, 8, 30)])
def test_invariant_subspace_forces_random_restart(reflib, nd, ned, maxlan):
    n = 300
    d = np.arange(n) % nd + 1.0
    got = []
    for L in (reflib, load()):
        info, ev = run(L, lambda x: d * x, n, ned, maxlan, np.ones(n))
        got.append((info.stat, info.nec, info.nrand, ev[:info.nec].copy()))
    for stat, nec, nrand, ev in got:
        assert stat == 0 and nec >= ned and nrand >= 1, (stat, nec, nrand)
        assert np.all(np.min(np.abs(ev[:, None] - np.arange(1.0, nd + 1)[None, :]), axis=1) <= 1e-10)
    # the smallest value is found by both
    assert got[0][3].min() == pytest.approx(1.0, abs=1e-10) == got[1][3].min()


def _write_checkpoint(path, nrow, jnd, nvec, truncate=0):
    rng = np.random.default_rng(1)
    data = struct.pack("ii", nrow, jnd)
    data += rng.standard_normal(jnd).tobytes() + np.abs(rng.standard_normal(jnd)).tobytes()
    data += rng.standard_normal(nvec * nrow).tobytes()
    with open(path, "wb") as f:
        f.write(data[:len(data) - truncate] if truncate else data)


@pytest.mark.parametrize("case,code", [("nrow", -213), ("maxlan", -214), ("short", -215)])
def test_unusable_checkpoint_gives_reference_status(reflib, tmp_path, monkeypatch, case, code):
    monkeypatch.chdir(tmp_path)
    n, ned, maxlan = 200, 4, 16
    jnd = {"nrow": 8, "maxlan": maxlan + 4, "short": 8}[case]
    nrow_file = n + 1 if case == "nrow" else n
    for name in ("0", "cp0"):               # the reference's file name, and prefix + rank
        _write_checkpoint(tmp_path / name, nrow_file, jnd, jnd + 1, truncate=(8 * n + 5) if case == "short" else 0)
    d = np.arange(1.0, n + 1.0)
    got = []
    for L in (reflib, load()):
        info, _ = run(L, lambda x: d * x, n, ned, maxlan, None, guess=2, cpf=b"cp")
        got.append(info.stat)
    assert got[0] == got[1] == code, got

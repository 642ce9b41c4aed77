"""Checkpoint files (trl_set_checkpoint, and trl_set_iguess with guess > 1):
the files this library writes have the reference's layout (int nrow, int
jnd, jnd alphas, jnd betas, jnd + 1 vectors) and hold a valid thick-restart
state (orthonormal vectors with A y_i = alpha_i y_i + beta_i q); a solve
resumed from a checkpoint converges to the eigenpairs of an uninterrupted
solve; the reference resumes from a file written here, and its own reader
and writer agree with these files byte for byte."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import operators as ops, DeviceOperator, load, TrlInfo, MATVEC
from oracle import ref

pytestmark = pytest.mark.gpu

NED, MAXLAN, TOL = 8, 40, 1e-9


def read_checkpoint(path, cplx=False):
    with open(path, "rb") as f:
        nrow, jnd = (int(v) for v in np.fromfile(f, np.int32, 2))
        alpha = np.fromfile(f, np.float64, jnd)
        beta = np.fromfile(f, np.float64, jnd)
        dt = np.complex128 if cplx else np.float64
        V = np.fromfile(f, dt, (jnd + 1) * nrow).reshape(jnd + 1, nrow)
        rest = f.read()
    assert rest == b""
    return nrow, jnd, alpha, beta, V


def b200_solve(A, maxmv, start=None, write=None, read=None, mev=NED + 4):
    lib = load()
    with DeviceOperator(A) as op:
        info = TrlInfo()
        lib.trl_init_info(C.byref(info), A.n, MAXLAN, -1, NED, TOL, 1, maxmv, None)
        info.mvparam = op.handle.value
        cplx = np.iscomplexobj(A.val)
        evec = np.zeros((mev, A.n), dtype=np.complex128 if cplx else np.float64)
        if write:
            lib.trl_set_checkpoint(C.byref(info), 1, write.encode())
        if read:
            lib.trl_set_checkpoint(C.byref(info), 0, read.encode())
            lib.trl_set_iguess(C.byref(info), 0, 2, 0, None)
        elif start is not None:
            lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
            evec[0] = start
        eval_ = np.zeros(mev)
        if cplx:
            misc = np.zeros(mev, dtype=np.complex128)
            lib.ztrlan(op.applier, C.byref(info), A.n, mev, eval_.ctypes.data, evec.ctypes.data, A.n,
                       misc.ctypes.data, mev, None, 0)
        else:
            wrk = np.zeros(mev)
            lib.trlan(op.applier, None, C.byref(info), A.n, mev, eval_.ctypes.data, evec.ctypes.data, A.n,
                      mev, wrk.ctypes.data)
    return info, eval_, evec


def ref_solve(A, maxmv, start=None, write=None, read=None, mev=NED + 4):
    lib = ref.load()
    val = np.ascontiguousarray(A.val)
    st = ref._CpuCSR(A.n, A.row_ptr.ctypes.data, A.col.ctypes.data, val.ctypes.data)
    fn = C.cast(ref.cpu_ops().cpu_csr_matvec, MATVEC)
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), A.n, MAXLAN, -1, NED, TOL, 1, maxmv, None)
    info.mvparam = C.addressof(st)
    evec = np.zeros((mev, A.n))
    if write:
        lib.trl_set_checkpoint(C.byref(info), 1, write.encode())
    if read:
        lib.trl_set_checkpoint(C.byref(info), 0, read.encode())
        lib.trl_set_iguess(C.byref(info), 0, 2, 0, None)
    elif start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        evec[0] = start
    eval_ = np.zeros(mev)
    lwrk = MAXLAN * (MAXLAN + 10)
    wrk = np.zeros(lwrk)
    lib.trlan(fn, None, C.byref(info), A.n, mev, eval_.ctypes.data, evec.ctypes.data, A.n, lwrk,
              wrk.ctypes.data)
    return info, eval_, evec


@pytest.fixture(scope="module")
def problem():
    A = ops.anderson_3d(14, seed=11)
    x0 = ops.start_vector(A.n)
    info, ev, _ = b200_solve(A, 100000, start=x0)
    assert info.nec >= NED
    return A, x0, np.sort(ev[:NED]), info.matvec


def test_written_file_layout_and_state(problem, tmp_path):
    A, x0, _, _ = problem
    prefix = str(tmp_path / "ck")
    info, _, _ = b200_solve(A, 70, start=x0, write=prefix)
    assert info.stat == 0 and info.nec < NED
    nrow, jnd, alpha, beta, V = read_checkpoint(prefix + "0")
    assert nrow == A.n and 1 <= jnd < MAXLAN
    np.testing.assert_allclose(V @ V.T, np.eye(jnd + 1), atol=1e-10)
    S = A.to_scipy()
    for i in range(jnd):
        r = S @ V[i] - alpha[i] * V[i] - beta[i] * V[jnd]
        assert np.linalg.norm(r) <= 1e-9 * 10.0, (i, np.linalg.norm(r))


def test_resume_from_own_checkpoint(problem, tmp_path):
    A, x0, full, full_mv = problem
    prefix = str(tmp_path / "own")
    first, _, _ = b200_solve(A, 70, start=x0, write=prefix)
    info, ev, evec = b200_solve(A, 100000, read=prefix)
    assert info.stat == 0 and info.nec >= NED
    np.testing.assert_allclose(np.sort(ev[:NED]), full, rtol=1e-10)
    S = A.to_scipy()
    for lam, v in zip(ev[:NED], evec[:NED]):
        assert np.linalg.norm(S @ v - lam * v) <= 1.01 * TOL * info.anrm


# The reference's trl_pe_filename (SRC/trlaux.c:1047) passes its output
# buffer as a %s argument of the same sprintf; with this C library the prefix
# is lost and the reference reads and writes a file named after the rank
# alone ("0") in the working directory.  The reference calls below run in a
# scratch directory and the files are copied to and from that name.

def test_reference_resumes_from_our_file(problem, tmp_path, monkeypatch):
    import shutil
    A, x0, full, _ = problem
    prefix = str(tmp_path / "ours")
    b200_solve(A, 70, start=x0, write=prefix)
    work = tmp_path / "ref"
    work.mkdir()
    shutil.copy(prefix + "0", work / "0")
    monkeypatch.chdir(work)
    info, ev, _ = ref_solve(A, 100000, read="unused")
    assert info.stat == 0 and info.nec >= NED
    np.testing.assert_allclose(np.sort(ev[:NED]), full, rtol=1e-10)


def test_reference_reader_and_writer_agree_with_our_file(problem, tmp_path):
    """The reference's own trl_read_checkpoint parses a file written here
    into the same state, and its trl_write_checkpoint, given that state,
    writes a byte-identical file.  (Its solver-driven writer cannot run
    here: write_checkpoint passes 138 as the size of a 132-byte name buffer
    to trl_pe_filename, which the C library's overflow check aborts.)"""
    A, x0, _, _ = problem
    lib = ref.load()
    prefix = str(tmp_path / "ours")
    b200_solve(A, 70, start=x0, write=prefix)
    nrow, jnd, alpha, beta, V = read_checkpoint(prefix + "0")
    # Reader: evec large enough for all jnd + 1 vectors (its j1 < mev branch).
    mev = jnd + 2
    ev = np.zeros((mev, nrow))
    a = np.zeros(jnd + 4)
    b = np.zeros(jnd + 4)
    j1, j2 = C.c_int(0), C.c_int(0)
    rd = lib.trl_read_checkpoint
    rd.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_int,
                   C.c_int, C.POINTER(C.c_int), C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    rd.restype = C.c_int
    assert rd((prefix + "0").encode(), nrow, ev.ctypes.data, nrow, mev, C.byref(j1), None, nrow, 1,
              C.byref(j2), jnd + 4, a.ctypes.data, jnd + 4, b.ctypes.data) == 0
    assert j1.value == jnd and j2.value == 0
    np.testing.assert_array_equal(a[:jnd], alpha)
    np.testing.assert_array_equal(b[:jnd], beta)
    np.testing.assert_array_equal(ev[:jnd + 1], V)
    # Writer: same bytes.
    wr = lib.trl_write_checkpoint
    wr.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                   C.c_int, C.c_int]
    wr.restype = C.c_int
    Vc = np.ascontiguousarray(V)
    out = str(tmp_path / "by_reference")
    assert wr(out.encode(), nrow, alpha.ctypes.data, beta.ctypes.data, Vc.ctypes.data, nrow, jnd + 1, None,
              nrow, 0) == 0
    with open(out, "rb") as f1, open(prefix + "0", "rb") as f2:
        assert f1.read() == f2.read()


def test_complex_checkpoint_roundtrip(tmp_path):
    A = ops.peierls_2d(32, phi=1.0 / 16.0)
    x0 = ops.start_vector(A.n) + 1j * ops.start_vector(A.n, seed=7)
    full_info, full, _ = b200_solve(A, 100000, start=x0)
    prefix = str(tmp_path / "z")
    b200_solve(A, 60, start=x0, write=prefix)
    nrow, jnd, alpha, beta, V = read_checkpoint(prefix + "0", cplx=True)
    assert nrow == A.n
    np.testing.assert_allclose(V.conj() @ V.T, np.eye(jnd + 1), atol=1e-10)
    info, ev, _ = b200_solve(A, 100000, read=prefix)
    assert info.nec >= NED
    np.testing.assert_allclose(np.sort(ev[:NED]), np.sort(full[:NED]), rtol=1e-10)


def test_missing_or_mismatched_file(tmp_path):
    A = ops.laplacian_2d(20)
    info, _, _ = b200_solve(A, 1000, read=str(tmp_path / "none"))
    assert info.stat == -212
    prefix = str(tmp_path / "small")
    b200_solve(ops.laplacian_2d(16), 60, start=ops.start_vector(256), write=prefix)
    info, _, _ = b200_solve(A, 1000, read=prefix)
    assert info.stat == -213

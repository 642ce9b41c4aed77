"""Pins the oracle before it is trusted (CPU only):
  * the reference library reproduces the reference's own example golden
    values (examples/simple.c: exact[i] = (i+1)^2; examples/test_ztrlan.c
    complex diagonal) and the analytic 2D Laplacian spectrum;
  * it reproduces the committed fixtures tests/golden/reference_runs.json;
  * the numpy restatement (oracle/kernels_np.py) agrees with scipy / dense
    linear algebra, including edge cases (empty rows, empty blocks);
  * the seeded operator generators are pinned (counter-based RNG values,
    symmetry / Hermiticity, analytic Laplacian eigenvalues)."""
import json
import os

import numpy as np
import pytest

from nutrlan_b200 import operators as ops
from oracle import kernels_np as K

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_runs.json")))


def _distinct(vals, tol=1e-9):
    out = []
    for v in np.sort(vals):
        if not out or abs(v - out[-1]) > tol * max(1.0, abs(v)):
            out.append(v)
    return np.array(out)


def test_golden_fixtures_are_sane():
    for name, c in GOLD.items():
        assert c["stat"] == 0, name
        assert c["nec"] >= c.get("ned", 1), name
    # The reference's example golden values: exact[i] = (i+1)^2.
    np.testing.assert_allclose(GOLD["simple_diag"]["eval"][:5], (np.arange(5) + 1.0) ** 2, rtol=1e-9)
    np.testing.assert_allclose(GOLD["zdiag1000"]["eval"][:10], (np.arange(10) + 1.0) ** 2, rtol=1e-9)
    exact = ops.laplacian_2d_eigs(128)
    for rs in range(1, 8):
        for v in GOLD[f"laplace128_r{rs}"]["eval"]:
            assert np.min(np.abs(exact - v)) <= 1e-10 * abs(v)


def test_reference_library_reproduces_simple_example(reflib):
    from oracle import ref
    c = GOLD["simple_diag"]
    n = c["n"]
    d = (np.arange(n) + 1.0) ** 2
    r = ref.trlan(lambda x: d * x, n, ned=5, maxlan=200, restart=1, maxmv=2000000,
                  start=np.ones(n), mev=100)
    assert r["info"].stat == 0 and r["info"].nec >= 5
    np.testing.assert_allclose(r["eval"][:5], (np.arange(5) + 1.0) ** 2, rtol=1e-9)
    assert abs(r["info"].matvec - c["matvec"]) <= 0.05 * c["matvec"]


@pytest.mark.parametrize("rs", [1, 3, 6])
def test_reference_library_matches_laplace_fixtures(reflib, rs):
    from oracle import ref
    A = ops.laplacian_2d(128)
    r = ref.trlan(A.matvec, A.n, ned=10, maxlan=64, restart=rs, maxmv=100000,
                  start=ops.start_vector(A.n))
    c = GOLD[f"laplace128_r{rs}"]
    assert r["info"].stat == 0
    got, want = _distinct(r["eval"][: r["info"].nec]), _distinct(c["eval"])
    k = min(len(got), len(want))
    np.testing.assert_allclose(got[:k], want[:k], rtol=1e-10)


def test_reference_library_matches_anderson_fixture(reflib):
    from oracle import ref
    B = ops.anderson_3d(16, W=4.0, seed=11)
    r = ref.trlan(B.matvec, B.n, ned=8, maxlan=40, restart=1, maxmv=100000,
                  start=ops.start_vector(B.n))
    c = GOLD["anderson16_r1"]
    np.testing.assert_allclose(r["eval"][:8], c["eval"][:8], rtol=1e-10)
    dense = np.linalg.eigvalsh(B.to_scipy().toarray())
    np.testing.assert_allclose(r["eval"][:8], dense[:8], rtol=1e-10)
    assert abs(r["info"].matvec - c["matvec"]) <= 0.05 * c["matvec"]


def test_reference_complex_library_matches_fixture(reflib):
    from oracle import ref
    P = ops.peierls_2d(64, phi=1.0 / 16.0)
    xp = ops.start_vector(P.n) + 1j * ops.start_vector(P.n, seed=7)
    r = ref.ztrlan(P.matvec, P.n, ned=8, maxlan=48, restart=1, maxmv=100000, start=xp)
    c = GOLD["peierls64"]
    np.testing.assert_allclose(r["eval"][:8], c["eval"][:8], rtol=1e-10)
    dense = np.linalg.eigvalsh(P.to_scipy().toarray())
    np.testing.assert_allclose(r["eval"][:8], dense[:8], rtol=1e-10, atol=1e-12)


def test_kernels_np_against_dense():
    rng = np.random.default_rng(0)
    V = rng.standard_normal((500, 12))
    r = rng.standard_normal(500)
    h = K.g_dot(V[:, :7], 7, V[:, 7:], 5, r)
    np.testing.assert_allclose(h, V.T @ r, rtol=1e-13)
    assert K.g_dot(V, 0, V, 0, r).size == 0
    h2, rn, hh, rr2 = K.cgs_pass(V, r)
    np.testing.assert_allclose(rn, r - V @ (V.T @ r))
    assert hh == pytest.approx(float(h2 @ h2)) and rr2 == pytest.approx(float(rn @ rn))
    Y = rng.standard_normal((12, 4))
    np.testing.assert_allclose(K.ritz_vectors(V, Y), V @ Y)


def test_csr_matvec_with_empty_rows_against_scipy():
    import scipy.sparse as sp
    rng = np.random.default_rng(1)
    n = 700
    lens = rng.integers(0, 9, n)
    lens[0] = 0
    lens[-1] = 0
    lens[::13] = 0
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    col = rng.integers(0, n, rp[-1]).astype(np.int32)
    val = rng.standard_normal(rp[-1])
    x = rng.standard_normal(n)
    M = sp.csr_matrix((val, col, rp), shape=(n, n))
    np.testing.assert_allclose(K.csr_matvec(rp, col, val, x), M @ x, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(ops.CSR(n, rp, col, val).matvec(x), M @ x, rtol=1e-13, atol=1e-13)


def test_counter_rng_is_pinned():
    def splitmix(seed, i):
        m = (1 << 64) - 1
        z = (seed + 0x9E3779B97F4A7C15 * (i + 1)) & m
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & m
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & m
        z ^= z >> 31
        return (z >> 11) / 2.0 ** 53
    got = ops.uniform01(12345, np.arange(6, dtype=np.uint64))
    want = [splitmix(12345, i) for i in range(6)]
    np.testing.assert_array_equal(got, want)


def test_operator_families():
    L = 8
    A = ops.laplacian_2d(L).to_scipy().toarray()
    np.testing.assert_allclose(np.linalg.eigvalsh(A), ops.laplacian_2d_eigs(L), atol=1e-12)
    B = ops.anderson_3d(6, seed=5).to_scipy().toarray()
    assert np.allclose(B, B.T) and B.shape == (216, 216)
    assert np.all(np.abs(np.diag(B)) <= 2.0) and np.count_nonzero(B[0]) == 7
    P = ops.peierls_2d(16, phi=1.0 / 8.0).to_scipy().toarray()
    assert np.allclose(P, P.conj().T)
    # Flux per plaquette: product of hoppings around a unit square.
    x, y = 3, 4
    s = lambda i, j: (i % 16) + 16 * (j % 16)  # noqa: E731
    loop = (P[s(x + 1, y), s(x, y)] * P[s(x + 1, y + 1), s(x + 1, y)] *
            P[s(x, y + 1), s(x + 1, y + 1)] * P[s(x, y), s(x, y + 1)])
    assert np.angle(loop) == pytest.approx(2 * np.pi / 8.0, abs=1e-12) or \
        np.angle(loop) == pytest.approx(-2 * np.pi / 8.0, abs=1e-12)
    W, V = ops.wells_2d(32, seed=1)
    assert V.shape == (32, 32) and V.max() <= 0 and W.n == 1024
    sizes = ops.batched_sizes(4096)
    assert sizes.min() >= 48 and sizes.max() <= 256


def test_ritz_projection_restatement_against_dense():
    """The numpy restatement of trl_ritz_projection's documented steps gives
    the eigenpairs of a subspace that is an invariant subspace up to 1e-8,
    whatever the (non-orthonormal, condition ~80) basis of it: eigenvalues
    to 1e-10, residuals at the perturbation times the basis condition."""
    A = ops.laplacian_2d(16, diag=ops.uniform01(4, np.arange(256, dtype=np.uint64)))
    w, U = np.linalg.eigh(A.to_scipy().toarray())
    rng = np.random.default_rng(1)
    V = (U[:, :7] @ rng.standard_normal((7, 7))).T + 1e-8 * rng.standard_normal((7, 256))
    d, X, res = K.ritz_projection(V, A.matvec, lohi=-1)
    np.testing.assert_allclose(d, w[:6], rtol=1e-10)
    assert np.all(res < 1e-5)
    np.testing.assert_allclose(np.abs(np.sum(X * U[:, :6].T, axis=1)) / np.linalg.norm(X, axis=1), 1.0,
                               atol=1e-9)


def test_reference_ritz_projection_defect(reflib):
    """The reference's trl_ritz_projection copies the lower triangle of V^T A V
    from the wrong column (SRC/trlan.c:1589-1593, 1602-1606): on an exactly
    orthonormal invariant subspace its smallest reported value is 0, not the
    smallest eigenvalue.  This pins why the library's routine is checked
    against the restatement of the documented steps instead."""
    import ctypes as C
    from nutrlan_b200._abi import TrlInfo, MATVEC
    A = ops.laplacian_2d(16, diag=1.0 + ops.uniform01(4, np.arange(256, dtype=np.uint64)))
    w, U = np.linalg.eigh(A.to_scipy().toarray())
    n, mev = A.n, 8
    V = np.ascontiguousarray(U[:, :mev].T)

    def op(nrow, ncol, x, ldx, y, ldy, mvparam):
        xv = np.ctypeslib.as_array(C.cast(x, C.POINTER(C.c_double)), (nrow,))
        yv = np.ctypeslib.as_array(C.cast(y, C.POINTER(C.c_double)), (nrow,))
        yv[:] = A.matvec(xv)
    cb = MATVEC(op)
    info = TrlInfo()
    reflib.trl_init_info(C.byref(info), n, 32, -1, 6, 1e-8, 1, 1000, None)
    info.verbose = -1
    eres, base, wrk = np.zeros(2 * mev), np.zeros(n), np.zeros(256)
    reflib.trl_ritz_projection(cb, C.byref(info), mev, V.ctypes.data, n, eres.ctypes.data, wrk.ctypes.data,
                               wrk.size, base.ctypes.data)
    assert info.stat == 0
    assert eres[0] == 0.0 and w[0] > 1.0
    d, _, _ = K.ritz_projection(U[:, :7].T, A.matvec, lohi=-1)
    np.testing.assert_allclose(d, w[:6], rtol=1e-12)

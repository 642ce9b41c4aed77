"""Parity with the reference library at the benchmark configurations' stated
sizes, against tests/golden/config_runs.json (the reference's own results on
the same seeded operators and start vectors, made by
tests/golden/make_config_golden.py from the reference built under
oracle/_ref).

* Anderson 256^3 (n = 16,777,216), smallest 32, maxlan = maxmv = 128: one
  thick-restart cycle, CSR and SELL-C-32 operators.  The 32 Ritz values
  after the cycle agree with the reference's, and so do the residual
  estimates, nec and the matvec count.
* Anderson 64^3, smallest 32, maxlan 128, tol 1e-8: the full solve returns
  the reference's eigenvalues (1e-10 relative, with multiplicity: the
  disorder breaks degeneracy), true residuals <= tol * ||A||
  (SRC/trlcore.c:2230-2232), matvecs within 5%.
* Peierls 2048^2 (complex Hermitian, n = 4,194,304), smallest 16,
  maxlan = maxmv = 96: one ztrlan cycle; Peierls 256^2 full solve.
* 16 problems of the 4096-problem batch, spread over the size range, solved
  in one batched launch against the reference solving each one.
* Gaussian wells 256^2 (4 held-out operators), plain solve, smallest 16.

Tolerances: 1e-10 relative on eigenvalues, as the task's correctness bar
states.  After a single cycle, Ritz values that have not converged are
still functions of the Krylov subspace alone, so they agree to about the
rounding level of the basis; the test states how far they are allowed to
move (RITZ_RTOL) and the residual estimates (|beta * y_last|, values near
1e-2..1e-4 after one cycle) to 1e-6 relative."""
import json
import os

import numpy as np
import pytest

from nutrlan_b200 import operators as ops, DeviceOperator, solve, residual_norms
from nutrlan_b200.batched import Batch, seeded_start

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))
RITZ_RTOL = 1e-10
RES_RTOL = 1e-6


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.fixture(scope="module")
def anderson256():
    g = GOLD["anderson256_cycle"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    x0 = ops.start_vector(A.n, seed=g["start_seed"])
    yield g, A, x0
    torch.cuda.empty_cache()


@pytest.mark.parametrize("fmt", ["sell", "csr"])
def test_anderson256_one_cycle_matches_reference(anderson256, fmt):
    g, A, x0 = anderson256
    k = g["ned"]
    with DeviceOperator(A, fmt=fmt) as op:
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=g["maxmv"], tol=1e-8, restart=g["restart"],
                  start=x0, mev=g["mev"], device=True)
    del r.evec
    assert r.stat == g["stat"]
    assert (r.nec, r.info.matvec, r.info.nloop) == (g["nec"], g["matvec"], g["nloop"])
    rel = _rel(r.eval[:k], g["eval"])
    print(f"anderson256 {fmt}: max rel Ritz-value diff {rel:.2e}, "
          f"max rel residual-estimate diff {_rel(r.res[:k], g['res']):.2e}")
    assert rel <= RITZ_RTOL
    np.testing.assert_allclose(r.res[:k], g["res"], rtol=RES_RTOL)


def _full_solve_check(g, A, x0, cplx=False, fmt="csr", basis_bits=64):
    with DeviceOperator(A, fmt=fmt) as op:
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=x0, mev=g["mev"], device=True, basis_bits=basis_bits)
        assert r.stat == 0 and r.nec >= g["ned"], (r.stat, r.nec)
        k = r.nec
        res = residual_norms(op, r.eval[:k], r.evec[:k])
    got = np.sort(r.eval[:g["ned"]])
    want = np.sort(np.array(g["eval"])[:g["ned"]])
    rel = _rel(got, want)
    print(f"max rel eigenvalue diff {rel:.2e}; matvecs {r.info.matvec} vs reference {g['matvec']}; "
          f"max true residual {res.max():.2e} (tol*anrm {g['tol'] * r.info.anrm:.2e})")
    assert rel <= 1e-10
    assert np.all(res <= g["tol"] * r.info.anrm * 1.01)
    # A 32-bit basis adds the FP64 refinement's applications (9 per pair per pass).
    extra = 0 if basis_bits == 64 else 9 * 3 * g["ned"]
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"] + extra


def test_anderson64_fp32_basis_full_solve_matches_reference():
    """FP32 basis storage (FP64 recurrence, dots and projected problem) with
    the FP64 refinement of the converged pairs: the reference's eigenvalues
    to 1e-10 and true residuals <= tol * ||A||."""
    g = GOLD["anderson64_full"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    _full_solve_check(g, A, ops.start_vector(A.n, seed=g["start_seed"]), fmt="sell", basis_bits=32)


def test_peierls256_c64_basis_full_solve_matches_reference():
    g = GOLD["peierls256_full"]
    A = ops.peierls_2d(g["L"], phi=g["phi"], W=g["W"], seed=g["pot_seed"])
    _full_solve_check(g, A, _peierls_start(A.n), cplx=True, basis_bits=32)


def test_anderson64_full_solve_matches_reference():
    g = GOLD["anderson64_full"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    _full_solve_check(g, A, ops.start_vector(A.n, seed=g["start_seed"]))


def _peierls_start(n):
    return ops.start_vector(n) + 1j * ops.start_vector(n, seed=99)


@pytest.mark.parametrize("fmt", ["zcsr", "zsell"])
def test_peierls2048_one_cycle_matches_reference(fmt):
    g = GOLD["peierls2048_cycle"]
    A = ops.peierls_2d(g["L"], phi=g["phi"], W=g["W"], seed=g["pot_seed"])
    with DeviceOperator(A, fmt=fmt) as op:
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=g["maxmv"], tol=1e-8, restart=g["restart"],
                  start=_peierls_start(A.n), mev=g["mev"], device=True)
    del r.evec
    torch.cuda.empty_cache()
    k = g["ned"]
    assert r.stat == g["stat"]
    assert (r.nec, r.info.matvec, r.info.nloop) == (g["nec"], g["matvec"], g["nloop"])
    rel = _rel(r.eval[:k], g["eval"])
    print(f"peierls2048 {fmt}: max rel Ritz-value diff {rel:.2e}")
    assert rel <= RITZ_RTOL


@pytest.mark.parametrize("fmt", ["zcsr", "zsell"])
def test_peierls256_full_solve_matches_reference(fmt):
    g = GOLD["peierls256_full"]
    A = ops.peierls_2d(g["L"], phi=g["phi"], W=g["W"], seed=g["pot_seed"])
    _full_solve_check(g, A, _peierls_start(A.n), cplx=True, fmt=fmt)


def test_batched_sample_matches_reference():
    """16 problems of the config-4 batch, each with the start vector the
    batched solver would give it at its position in the full batch."""
    g = GOLD["batched_sample"]
    Ls_all = ops.batched_sizes(g["count"], seed=g["sizes_seed"])
    probs = g["problems"]
    Ls, diags, starts = [], [], []
    for p in probs:
        L = int(Ls_all[p["index"]])
        assert L == p["L"]
        Ls.append(L)
        diags.append(2.0 * ops.uniform01(1000 + p["index"], np.arange(L * L, dtype=np.uint64)))
        starts.append(seeded_start(g["start_seed"], p["index"], L * L))
    b = Batch.stencil5(Ls, diags)
    try:
        b.set_start(starts)
        r = b.solve(ned=g["ned"], maxlan=g["maxlan"], tol=g["tol"], restart=g["restart"], maxmv=100000)
        worst, mv_dev = 0.0, []
        for i, p in enumerate(probs):
            stat, nec, mv, nloop = r.info[i]
            assert stat == 0 and nec >= g["ned"], (i, r.info[i])
            worst = max(worst, _rel(np.sort(r.eval[i]), np.sort(p["eval"][:g["ned"]])))
            mv_dev.append((mv - p["matvec"]) / p["matvec"])
            A = ops.laplacian_2d(p["L"], diag=diags[i])
            V = b.eigenvectors(i)
            for lam, v in zip(r.eval[i], V):
                assert np.linalg.norm(A.matvec(v) - lam * v) <= g["tol"] * p["anrm"] * 1.01
        print(f"batched sample: max rel eigenvalue diff {worst:.2e}; matvec deviations "
              f"{min(mv_dev):+.3f}..{max(mv_dev):+.3f}")
        assert worst <= 1e-10
        assert max(abs(d) for d in mv_dev) <= 0.05
    finally:
        b.close()


def test_wells256_plain_matches_reference():
    g = GOLD["wells256"]
    for p in g["problems"]:
        A, _ = ops.wells_2d(g["L"], seed=p["seed"])
        with DeviceOperator(A) as op:
            r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                      start=ops.start_vector(A.n), device=True)
            assert r.stat == 0 and r.nec >= g["ned"]
            res = residual_norms(op, r.eval[:r.nec], r.evec[:r.nec])
        rel = _rel(np.sort(r.eval[:g["ned"]]), np.sort(p["eval"][:g["ned"]]))
        print(f"wells seed {p['seed']}: rel {rel:.2e}, matvecs {r.info.matvec} vs {p['matvec']}")
        assert rel <= 1e-10
        assert np.all(res <= g["tol"] * r.info.anrm * 1.01)
        assert abs(r.info.matvec - p["matvec"]) <= 0.05 * p["matvec"] + 2

"""Batched persistent solver (trlx_batch_*) on the GPU: each problem's
smallest eigenpairs against dense eigvalsh (small grids) and against the
single-problem engine run on the same operator and start vector (same
algorithm: eigenvalues within 1e-10, matvec counts within a few percent);
residuals of the returned eigenvectors <= tol * ||A||; every thread-group
size and operator format gives the same answers."""
import numpy as np
import pytest

from nutrlan_b200 import operators as ops, DeviceOperator, solve
from nutrlan_b200.batched import Batch, seeded_start

pytestmark = pytest.mark.gpu

SEED = 0x1234567


def make_batch(Ls, seed=5):
    diags = [2.0 * ops.uniform01(seed + k, np.arange(L * L, dtype=np.uint64)) for k, L in enumerate(Ls)]
    return Batch.stencil5(Ls, diags), diags


@pytest.fixture(scope="module")
def small():
    Ls = [12, 17, 24, 31, 40, 9, 26, 35]
    b, diags = make_batch(Ls)
    yield Ls, b, diags
    b.close()


@pytest.mark.parametrize("threads,fmt,cta", [(256, 0, 1024), (512, 0, 1024), (1024, 0, 1024), (256, 1, 1024),
                                             (1024, 1, 1024), (512, 0, 512), (256, 0, 512), (128, 0, 512),
                                             (128, 1, 512)])
def test_batched_small_against_dense(small, threads, fmt, cta):
    Ls, b, diags = small
    r = b.solve(ned=6, maxlan=24, tol=1e-8, seed=SEED, threads=threads, fmt=fmt, cta=cta)
    assert r.config.cta_threads == cta
    for p, L in enumerate(Ls):
        stat, nec, mv, nloop = r.info[p]
        assert stat == 0 and nec >= 6, (p, r.info[p])
        A = ops.laplacian_2d(L, diag=diags[p])
        dense = np.linalg.eigvalsh(A.to_scipy().toarray())
        np.testing.assert_allclose(r.eval[p], dense[:6], rtol=1e-10, atol=1e-12)
        V = b.eigenvectors(p)
        anrm = np.max(np.abs(dense))
        for lam, v in zip(r.eval[p], V):
            assert np.linalg.norm(A.matvec(v) - lam * v) <= 1e-8 * anrm * 1.01


def test_batched_matches_single_engine_on_mixed_sizes():
    Ls = [48, 64, 96, 128, 181, 200, 256, 50, 100, 150]
    b, diags = make_batch(Ls, seed=77)
    try:
        r = b.solve(ned=8, maxlan=32, tol=1e-8, seed=SEED)
        for p, L in enumerate(Ls):
            A = ops.laplacian_2d(L, diag=diags[p])
            x0 = seeded_start(SEED, p, A.n)
            with DeviceOperator(A) as op:
                e = solve(op, ned=8, maxlan=32, tol=1e-8, restart=1, maxmv=100000, start=x0)
            assert r.info[p][0] == 0 and r.info[p][1] >= 8
            np.testing.assert_allclose(r.eval[p], e.eval[:8], rtol=1e-10)
            assert abs(r.info[p][2] - e.info.matvec) <= 0.05 * e.info.matvec + 8, (p, r.info[p], e.info.matvec)
            V = b.eigenvectors(p)
            for lam, v in zip(r.eval[p], V):
                assert np.linalg.norm(A.matvec(v) - lam * v) <= 1e-8 * (8.0 + 2.0) * 1.01
        cfg = r.config
        assert all(t in (256, 512, 1024) for t in cfg.bucket_threads)
    finally:
        b.close()


def test_batched_caller_start_vectors(small):
    Ls, b, diags = small
    starts = [None] * len(Ls)
    starts[2] = np.ones(Ls[2] ** 2)
    b.set_start(starts)
    try:
        r = b.solve(ned=6, maxlan=24, tol=1e-8, seed=SEED, threads=512, fmt=0)
        A = ops.laplacian_2d(Ls[2], diag=diags[2])
        with DeviceOperator(A) as op:
            e = solve(op, ned=6, maxlan=24, tol=1e-8, restart=1, maxmv=100000, start=np.ones(A.n))
        np.testing.assert_allclose(r.eval[2], e.eval[:6], rtol=1e-10)
        assert abs(r.info[2][2] - e.info.matvec) <= 0.05 * e.info.matvec + 8
    finally:
        b.set_start([None] * len(Ls))


def test_batched_large_maxlan_uses_fitting_splits():
    """maxlan 48, ned 16 (the learned-seed training configuration): the
    autotuner only uses thread splits whose shared memory fits, and an
    explicit split that does not fit is rejected up front."""
    Ls = [48, 64, 40]
    diags = [ops.wells_potential(L, 900 + k).reshape(-1) for k, L in enumerate(Ls)]
    b = Batch.stencil5(Ls, diags)
    try:
        r = b.solve(ned=16, maxlan=48, tol=1e-8, seed=SEED)
        for p, L in enumerate(Ls):
            assert r.info[p][0] == 0 and r.info[p][1] >= 16
            A = ops.laplacian_2d(L, diag=diags[p])
            dense = np.linalg.eigvalsh(A.to_scipy().toarray())
            np.testing.assert_allclose(r.eval[p], dense[:16], rtol=1e-10, atol=1e-12)
        with pytest.raises(RuntimeError):
            b.solve(ned=16, maxlan=48, tol=1e-8, seed=SEED, threads=256)
    finally:
        b.close()


def test_batched_cta_sizes_agree():
    """The 512-thread CTA form (16-column projection passes, twice the
    registers) runs the same algorithm as the 1024-thread form: the same
    eigenvalues to 1e-12 and the same matvec counts, problem by problem."""
    Ls = [48, 96, 150, 200, 256, 60, 120, 181]
    b, _ = make_batch(Ls, seed=91)
    try:
        r1 = b.solve(ned=8, maxlan=32, tol=1e-8, seed=SEED, threads=512, cta=1024)
        r2 = b.solve(ned=8, maxlan=32, tol=1e-8, seed=SEED, threads=512, cta=512)
        assert r1.config.cta_threads == 1024 and r2.config.cta_threads == 512
        np.testing.assert_allclose(r2.eval, r1.eval, rtol=1e-12)
        assert np.all(np.abs(r2.info[:, 2] - r1.info[:, 2]) <= 0.02 * r1.info[:, 2] + 2), (r1.info, r2.info)
        assert np.all(r2.info[:, 1] >= 8)
    finally:
        b.close()


def test_batched_solve_replays_its_captured_graph(small):
    """A solve's launch sequence is a CUDA graph captured once per launch
    configuration: the same configuration again replays it (with the same
    results), a different one captures a new graph."""
    Ls, b, diags = small
    kw = dict(ned=6, maxlan=24, tol=1e-8, seed=SEED, threads=512, fmt=0, cta=1024)
    r1 = b.solve(**kw)
    r2 = b.solve(**kw)
    assert r2.config.graph_replays == r1.config.graph_replays + 1 >= 2
    np.testing.assert_array_equal(r1.eval, r2.eval)
    np.testing.assert_array_equal(r1.info, r2.info)
    r3 = b.solve(**dict(kw, threads=256))
    assert r3.config.graph_replays == 1
    np.testing.assert_allclose(r3.eval, r1.eval, rtol=1e-10)

"""Block-row solves on the GPU.

Two ranks run as two processes on the one GPU of the test machine with a
gloo group behind the library's host-callback communicator: every sum and
halo exchange waits on the host, no kernel waits for the other process.
Each rank owns an uneven block of rows of a 3D Anderson operator (the split
falls inside a lattice plane, so the halo has entries from both
neighbours' planes) as a distributed CSR or SELL operator:

* the distributed product equals the global CSR product on every row;
* the block-row solve (FP64 basis, and FP32 basis with the FP64
  refinement, whose Gram matrices are summed over the ranks too) returns
  the single-GPU solve's eigenvalues to 1e-10 relative, with residuals of
  the assembled eigenvectors <= tol * ||A||, in about as many matvecs;
* every rank returns the same eigenvalues.

An NCCL communicator of one rank (the NCCL calls run, as copies) gives the
single-GPU eigenvalues.  NCCL with two ranks needs two GPUs and is not run
here: ranks whose collective kernels wait on each other must not share a GPU.
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

from nutrlan_b200 import operators as ops, DeviceOperator, solve

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L, NED, MAXLAN, TOL = 16, 8, 40, 1e-8
SPLIT = 1700  # rows of rank 0 (inside plane 6 of 16)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        from nutrlan_b200 import operators as ops
        from nutrlan_b200.dist import Comm, DistOperator, local_rows, solve as dsolve
        A = ops.anderson_3d(L, seed=11)
        x0 = ops.start_vector(A.n, seed=5)
        row0, nloc = (0, SPLIT) if rank == 0 else (SPLIT, A.n - SPLIT)
        x = np.random.default_rng(2).standard_normal(A.n)
        out = {"rank": rank}
        with Comm.from_process_group() as comm:
            for fmt in ("csr", "sell"):
                with DistOperator(comm, *local_rows(A, row0, nloc), fmt=fmt) as op:
                    out[f"halo_{fmt}"] = op.halo
                    out[f"y_{fmt}"] = op.matvec(x[row0:row0 + nloc])
                    for bits in (64, 32):
                        r = dsolve(comm, op, ned=NED, maxlan=MAXLAN, tol=TOL, start=x0[row0:row0 + nloc],
                                   basis_bits=bits)
                        out[f"solve_{fmt}_{bits}"] = dict(
                            stat=r.stat, nec=r.nec, matvec=r.info.matvec, eval=r.eval[:r.nec].copy(),
                            evec=np.array(r.evec[:r.nec]), anrm=r.info.anrm, ntot=r.info.ntot)
        q.put(out)
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put({"rank": rank, "error": repr(e)})
    finally:
        dist.destroy_process_group()


@pytest.fixture(scope="module")
def two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
    for o in out:
        assert "error" not in o, o
    for p in procs:
        assert p.exitcode == 0
    return sorted(out, key=lambda o: o["rank"])


@pytest.fixture(scope="module")
def single():
    A = ops.anderson_3d(L, seed=11)
    x0 = ops.start_vector(A.n, seed=5)
    res = {}
    with DeviceOperator(A, fmt="sell") as op:
        for bits in (64, 32):
            r = solve(op, ned=NED, maxlan=MAXLAN, tol=TOL, start=x0, basis_bits=bits)
            res[bits] = (r.eval[:r.nec].copy(), r.info.matvec)
    return A, res


def test_distributed_product_matches_global(two_ranks, single):
    A, _ = single
    x = np.random.default_rng(2).standard_normal(A.n)
    want = A.matvec(x)
    for fmt in ("csr", "sell"):
        assert two_ranks[0][f"halo_{fmt}"] > 0 and two_ranks[1][f"halo_{fmt}"] > 0
        y = np.concatenate([two_ranks[0][f"y_{fmt}"], two_ranks[1][f"y_{fmt}"]])
        np.testing.assert_allclose(y, want, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("fmt", ["csr", "sell"])
@pytest.mark.parametrize("bits", [64, 32])
def test_block_row_solve_matches_single_gpu(two_ranks, single, fmt, bits):
    A, res = single
    want, mv1 = res[bits]
    r0, r1 = two_ranks[0][f"solve_{fmt}_{bits}"], two_ranks[1][f"solve_{fmt}_{bits}"]
    assert r0["stat"] == r1["stat"] == 0
    assert r0["ntot"] == A.n
    assert r0["nec"] == r1["nec"] >= NED
    np.testing.assert_array_equal(r0["eval"], r1["eval"])
    k = min(NED, len(want))
    np.testing.assert_allclose(np.sort(r0["eval"])[:k], np.sort(want)[:k], rtol=1e-10)
    assert abs(r0["matvec"] - mv1) <= 0.1 * mv1, (r0["matvec"], mv1)
    z = np.concatenate([r0["evec"], r1["evec"]], axis=1)
    for lam, v in zip(r0["eval"], z):
        res_norm = np.linalg.norm(A.matvec(v) - lam * v) / np.linalg.norm(v)
        assert res_norm <= 1.01 * TOL * r0["anrm"], (lam, res_norm)


def test_nccl_single_rank_solve(single):
    from nutrlan_b200.dist import Comm, DistOperator, local_rows, solve as dsolve
    A, res = single
    x0 = ops.start_vector(A.n, seed=5)
    try:
        uid = Comm.nccl_unique_id()
    except RuntimeError as e:
        pytest.skip(f"NCCL not loadable: {e}")
    with Comm.nccl(1, 0, uid) as comm:
        with DistOperator(comm, *local_rows(A, 0, A.n), fmt="sell") as op:
            assert op.halo == 0
            r = dsolve(comm, op, ned=NED, maxlan=MAXLAN, tol=TOL, start=x0)
    assert r.stat == 0 and r.nec >= NED
    want, mv1 = res[64]
    np.testing.assert_allclose(np.sort(r.eval[:NED]), np.sort(want)[:NED], rtol=1e-12)
    assert abs(r.info.matvec - mv1) <= 0.05 * mv1

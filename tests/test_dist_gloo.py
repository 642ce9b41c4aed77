"""Block-row communicators on CPU: two and three gloo ranks (127.0.0.1) drive
the library's host-callback communicator (trlx_comm_create_host), which
needs no GPU for host reductions:

* trlx_comm_allreduce sums / maxes / mins host doubles over the ranks;
* trlx_init_info_comm gives every rank ntot = sum of the local row counts
  (uneven blocks), its own my_pe, npes, and the reference maxmv default
  from the global ntot (SRC/trl_comm_mpi.c trl_init_info);
* the row-block helpers split a global CSR matrix into the blocks the
  distributed operators take (global column indices, row_ptr from 0).
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import ctypes as C
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from nutrlan_b200 import TrlInfo, load
        from nutrlan_b200.dist import Comm, SUM, MAX, MIN
        lib = load()
        with Comm.from_process_group() as comm:
            v = np.array([1.0 + rank, -2.0 * rank, 10.0 ** rank])
            out = {"rank": comm.rank, "size": comm.size,
                   "sum": comm.allreduce(v, SUM), "max": comm.allreduce(v, MAX), "min": comm.allreduce(v, MIN)}
            nloc = 1000 + 7 * rank
            info = TrlInfo()
            rc = lib.trlx_init_info_comm(C.byref(info), comm.handle, nloc, 40, -1, 5, 1e-8, 1, 0)
            out.update(rc=rc, ntot=info.ntot, nloc=info.nloc, my_pe=info.my_pe, npes=info.npes,
                       maxmv=info.maxmv, mpicomp=bool(info.mpicomp))
            # An op outside SUM/MAX/MIN is refused before any communication.
            out["bad_op"] = lib.trlx_comm_allreduce(comm.handle, v.ctypes.data, 3, 7)
        q.put(out)
    finally:
        dist.destroy_process_group()


def _run(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out, key=lambda o: o["rank"])


def test_host_communicator_reductions_and_info():
    for world in (2, 3):
        res = _run(world)
        vs = np.array([[1.0 + r, -2.0 * r, 10.0 ** r] for r in range(world)])
        ntot = sum(1000 + 7 * r for r in range(world))
        for r, o in enumerate(res):
            assert o["rank"] == r and o["size"] == world
            np.testing.assert_array_equal(o["sum"], vs.sum(axis=0))
            np.testing.assert_array_equal(o["max"], vs.max(axis=0))
            np.testing.assert_array_equal(o["min"], vs.min(axis=0))
            assert o["rc"] == 0 and o["ntot"] == ntot and o["nloc"] == 1000 + 7 * r
            assert o["my_pe"] == r and o["npes"] == world and o["mpicomp"]
            assert o["maxmv"] == min(max(ntot, 1000), 1000 * 5)
            assert o["bad_op"] == -1


def test_row_blocks_cover_and_local_rows_keep_global_columns():
    sys.path.insert(0, ROOT)
    from nutrlan_b200 import operators as ops
    from nutrlan_b200.dist import row_blocks, local_rows
    A = ops.anderson_3d(6, seed=4)
    blocks = row_blocks(A.n, 5)
    assert blocks[0][0] == 0 and sum(nl for _, nl in blocks) == A.n
    assert all(b[0] + b[1] == c[0] for b, c in zip(blocks, blocks[1:]))
    assert max(nl for _, nl in blocks) - min(nl for _, nl in blocks) <= 1
    x = np.random.default_rng(0).standard_normal(A.n)
    y = A.matvec(x)
    parts = []
    for row0, nloc in blocks:
        rp, ci, va = local_rows(A, row0, nloc)
        assert rp[0] == 0 and len(rp) == nloc + 1 and ci.max() < A.n
        parts.append(np.array([va[rp[i]:rp[i + 1]] @ x[ci[rp[i]:rp[i + 1]]] for i in range(nloc)]))
    np.testing.assert_allclose(np.concatenate(parts), y, rtol=1e-14, atol=1e-13)

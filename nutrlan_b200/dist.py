"""Block-row solves over several ranks, one GPU each.

The reference's parallel build gives every MPI rank a contiguous block of
rows of every vector and sums the partial dot products over the ranks
(SRC/trl_comm_mpi.c).  The library does the same with a ``trlx_comm``:

* ``Comm.from_process_group(pg)`` wraps a ``torch.distributed`` group: a
  gloo group becomes a host-callback communicator (each sum is a
  ``dist.all_reduce`` of a CPU tensor), an NCCL group becomes an NCCL
  communicator of the library (rank 0 makes the NCCL id, the group
  broadcasts it);
* ``row_blocks(n, nranks)`` / ``local_rows(csr, row0, nloc)`` split a
  global CSR matrix into the rows a rank owns (column indices stay global);
* ``DistOperator(comm, rp, ci, va)`` is the rank's block of a distributed
  built-in operator (halo exchange before every product);
* ``solve(comm, op, ...)`` runs trlan on the rank's rows: every rank gets the
  same eigenvalues and its rows of the eigenvectors.

Example (torchrun, one process per GPU)::

    comm = Comm.from_process_group()
    row0, nloc = row_blocks(A.n, comm.size)[comm.rank]
    with DistOperator(comm, *local_rows(A, row0, nloc), fmt="sell") as op:
        r = solve(comm, op, ned=32, maxlan=128, start=x0[row0:row0 + nloc])
"""
import ctypes as C

import numpy as np

from ._abi import TrlInfo, MATVEC
from ._lib import load, TrlxOptions, TrlxStats, ALLREDUCE_FN
from .solver import SolveResult

SUM, MAX, MIN = 0, 1, 2


class Comm:
    """A library communicator (trlx_comm) of this rank."""

    def __init__(self, handle, keep=None):
        self.lib = load()
        self.handle = handle
        self._keep = keep  # the ctypes callback must outlive the communicator
        self.rank = self.lib.trlx_comm_rank(handle)
        self.size = self.lib.trlx_comm_size(handle)

    @classmethod
    def host(cls, nranks, rank, allreduce):
        """Host-callback communicator; ``allreduce(array, op)`` reduces a
        float64 numpy array in place over all ranks (op: SUM, MAX, MIN)."""
        lib = load()

        def cb(buf, count, op, ctx):
            try:
                allreduce(np.ctypeslib.as_array(buf, shape=(count,)), op)
                return 0
            except Exception:  # noqa: BLE001 - reported as a library error code
                return 1

        fn = ALLREDUCE_FN(cb)
        h = C.c_void_p()
        rc = lib.trlx_comm_create_host(nranks, rank, fn, None, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"trlx_comm_create_host failed ({rc})")
        return cls(h, keep=fn)

    @classmethod
    def nccl(cls, nranks, rank, unique_id):
        lib = load()
        h = C.c_void_p()
        idb = (C.c_ubyte * 128).from_buffer_copy(bytes(unique_id))
        rc = lib.trlx_comm_create_nccl(nranks, rank, idb, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"trlx_comm_create_nccl failed ({rc})")
        return cls(h)

    @staticmethod
    def nccl_unique_id():
        idb = (C.c_ubyte * 128)()
        rc = load().trlx_comm_nccl_id(idb)
        if rc != 0:
            raise RuntimeError(f"trlx_comm_nccl_id failed ({rc})")
        return bytes(idb)

    @classmethod
    def from_process_group(cls, group=None):
        """Communicator over a torch.distributed group (default: WORLD)."""
        import torch
        import torch.distributed as dist
        rank, size = dist.get_rank(group), dist.get_world_size(group)
        if dist.get_backend(group) == "nccl":
            box = [cls.nccl_unique_id() if rank == 0 else None]
            src = dist.get_global_rank(group, 0) if group is not None else 0
            dist.broadcast_object_list(box, src=src, group=group)
            return cls.nccl(size, rank, box[0])
        ops = {SUM: dist.ReduceOp.SUM, MAX: dist.ReduceOp.MAX, MIN: dist.ReduceOp.MIN}

        def allreduce(arr, op):
            dist.all_reduce(torch.from_numpy(arr), op=ops[op], group=group)

        return cls.host(size, rank, allreduce)

    def allreduce(self, values, op=SUM):
        """Reduced copy of ``values`` (float64) through the library."""
        a = np.ascontiguousarray(values, dtype=np.float64).copy()
        rc = self.lib.trlx_comm_allreduce(self.handle, a.ctypes.data, a.size, op)
        if rc != 0:
            raise RuntimeError(f"trlx_comm_allreduce failed ({rc})")
        return a

    def close(self):
        if self.handle:
            self.lib.trlx_comm_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def row_blocks(n, nranks):
    """[(row0, nloc)] of ``nranks`` contiguous blocks covering n rows, the
    first n % nranks blocks one row longer."""
    base, extra = divmod(n, nranks)
    out, r0 = [], 0
    for p in range(nranks):
        nl = base + (1 if p < extra else 0)
        out.append((r0, nl))
        r0 += nl
    return out


def local_rows(csr, row0, nloc):
    """Rows row0 .. row0+nloc-1 of a global CSR matrix as (row_ptr, col, val)
    with row_ptr starting at 0 and global column indices."""
    rp = np.asarray(csr.row_ptr, dtype=np.int64)
    b, e = int(rp[row0]), int(rp[row0 + nloc])
    return (np.ascontiguousarray(rp[row0:row0 + nloc + 1] - b),
            np.ascontiguousarray(np.asarray(csr.col, dtype=np.int32)[b:e]),
            np.ascontiguousarray(np.asarray(csr.val, dtype=np.float64)[b:e]))


class DistOperator:
    """This rank's block rows of a distributed real operator (CSR or
    SELL-C-32 locally, halo values received before every product)."""

    def __init__(self, comm, row_ptr, col, val, fmt="csr", sigma=1):
        lib = load()
        self.lib, self.comm = lib, comm
        self.n = len(row_ptr) - 1
        self.complex = False
        rp = np.ascontiguousarray(row_ptr, np.int64)
        ci = np.ascontiguousarray(col, np.int32)
        va = np.ascontiguousarray(val, np.float64)
        self.handle = C.c_void_p()
        if fmt == "sell":
            rc = lib.trlx_dist_sell_create(comm.handle, self.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                           int(sigma), 0, C.byref(self.handle))
        else:
            rc = lib.trlx_dist_csr_create(comm.handle, self.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                          0, C.byref(self.handle))
        if rc != 0:
            raise RuntimeError(f"distributed operator creation failed ({rc})")
        self.fmt = fmt
        self.halo = lib.trlx_operator_halo(self.handle)
        self.applier = C.cast(lib.trlx_matvec, MATVEC)

    def matvec(self, x_local):
        """y = A x for this rank's rows (a collective: every rank calls it)."""
        import torch
        x = torch.as_tensor(np.asarray(x_local, dtype=np.float64), device="cuda")
        y = torch.zeros_like(x)
        f = self.lib.trlx_matvec
        f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        f.restype = None
        f(self.n, 1, x.data_ptr(), self.n, y.data_ptr(), self.n, self.handle)
        torch.cuda.synchronize()
        return y.cpu().numpy()

    def close(self):
        if self.handle:
            self.lib.trlx_operator_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def solve(comm, op, ned, maxlan, lohi=-1, tol=1.4901e-8, restart=1, maxmv=0, start=None, mev=None,
          basis_bits=64, seed=0, refine=None, profile=False, evec=None):
    """trlan on this rank's rows (``op``: a DistOperator, or anything with
    ``n``, ``handle`` and ``applier`` of a built-in operator).  ``start`` is
    this rank's rows of the start vector; ``evec`` (optional) a C-contiguous
    mev x n float64 torch CUDA tensor (device-resident eigenvectors) or numpy
    array.  A collective: every
    rank calls it with the same parameters."""
    lib = load()
    n = op.n
    mev = mev or ned + 1
    info = TrlInfo()
    rc = lib.trlx_init_info_comm(C.byref(info), comm.handle, n, maxlan, lohi, ned, tol, restart, maxmv)
    if rc != 0:
        raise RuntimeError(f"trlx_init_info_comm failed ({rc})")
    info.mvparam = op.handle.value
    eval_ = np.zeros(mev)
    if evec is not None and hasattr(evec, "data_ptr"):
        import torch
        ev = evec
        if start is not None:
            ev[0].copy_(torch.as_tensor(np.asarray(start, dtype=np.float64)))
        torch.cuda.synchronize()
        ptr = ev.data_ptr()
    else:
        ev = evec if evec is not None else np.zeros((mev, n))
        if start is not None:
            ev[0] = start
        ptr = ev.ctypes.data
    if start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
    wrk = np.zeros(mev)
    opts = TrlxOptions()
    lib.trlx_default_options(C.byref(opts))
    opts.basis_bits = basis_bits
    opts.seed = seed
    if refine is not None:
        opts.refine = 1 if refine else 0
    opts.profile = 1 if profile else 0
    lib.trlx_trlan(op.applier, None, C.byref(info), n, mev, eval_.ctypes.data, ptr, n, mev, wrk.ctypes.data,
                   C.byref(opts))
    stats = TrlxStats()
    lib.trlx_get_last_stats(C.byref(stats))
    return SolveResult(eval=eval_, evec=ev, res=wrk, info=info, stats=stats)

"""Python front end of the batched solver (trlx_batch_* in include/trlx.h).

    from nutrlan_b200.batched import Batch
    b = Batch.stencil5(Ls, diags)           # L x L Laplacians + diagonals
    r = b.solve(ned=8, maxlan=32, tol=1e-8)  # one persistent launch
    r.eval[p], r.info[p], b.eigenvectors(p)
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import load


class BatchOptions(C.Structure):
    _fields_ = [("ned", C.c_int), ("maxlan", C.c_int), ("lohi", C.c_int), ("restart", C.c_int),
                ("maxmv", C.c_int), ("tol", C.c_double), ("seed", C.c_ulonglong),
                ("threads", C.c_int), ("format", C.c_int), ("cta_threads", C.c_int)]


class BatchConfig(C.Structure):
    _fields_ = [("bucket_threads", C.c_int * 3), ("bucket_format", C.c_int * 3),
                ("tune_seconds", C.c_double), ("cta_threads", C.c_int), ("graph_replays", C.c_int)]


def _declare(lib):
    P = C.POINTER
    lib.trlx_batch_create_stencil5.argtypes = [C.c_int, C.c_void_p, C.c_void_p, P(C.c_void_p)]
    lib.trlx_batch_create_stencil5.restype = C.c_int
    lib.trlx_batch_set_start.argtypes = [C.c_void_p, C.c_void_p]
    lib.trlx_batch_set_start.restype = C.c_int
    lib.trlx_batch_default_options.argtypes = [P(BatchOptions)]
    lib.trlx_batch_default_options.restype = None
    lib.trlx_batch_autotune.argtypes = [C.c_void_p, P(BatchOptions), P(BatchConfig)]
    lib.trlx_batch_autotune.restype = C.c_int
    lib.trlx_batch_solve.argtypes = [C.c_void_p, P(BatchOptions), C.c_void_p, C.c_void_p, C.c_void_p,
                                     P(BatchConfig)]
    lib.trlx_batch_solve.restype = C.c_int
    lib.trlx_batch_eigenvectors.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    lib.trlx_batch_eigenvectors.restype = C.c_int
    lib.trlx_batch_size.argtypes = [C.c_void_p, C.c_int]
    lib.trlx_batch_size.restype = C.c_int
    lib.trlx_batch_destroy.argtypes = [C.c_void_p]
    lib.trlx_batch_destroy.restype = None
    return lib


@dataclass
class BatchResult:
    eval: np.ndarray   # (nprob, ned)
    res: np.ndarray    # (nprob, ned) residual estimates
    info: np.ndarray   # (nprob, 4): stat, nec, matvec, restarts
    config: BatchConfig


class Batch:
    def __init__(self, handle, nprob, lib):
        self.handle, self.nprob, self.lib = handle, nprob, lib
        self.ned = None

    @classmethod
    def stencil5(cls, Ls, diags):
        lib = _declare(load())
        Ls = np.ascontiguousarray(Ls, dtype=np.int32)
        keep = [np.ascontiguousarray(d, dtype=np.float64) for d in diags]
        ptrs = (C.c_void_p * len(keep))(*[d.ctypes.data for d in keep])
        h = C.c_void_p()
        rc = lib.trlx_batch_create_stencil5(len(keep), Ls.ctypes.data, ptrs, C.byref(h))
        if rc:
            raise RuntimeError(f"trlx_batch_create_stencil5 failed ({rc})")
        b = cls(h, len(keep), lib)
        b.Ls = Ls
        return b

    def set_start(self, starts):
        keep = [None if s is None else np.ascontiguousarray(s, dtype=np.float64) for s in starts]
        ptrs = (C.c_void_p * len(keep))(*[None if s is None else s.ctypes.data for s in keep])
        rc = self.lib.trlx_batch_set_start(self.handle, ptrs)
        if rc:
            raise RuntimeError(f"trlx_batch_set_start failed ({rc})")

    def options(self, ned=8, maxlan=32, tol=1e-8, restart=1, maxmv=100000, seed=None, threads=0,
                fmt=-1, lohi=-1, cta=0):
        o = BatchOptions()
        self.lib.trlx_batch_default_options(C.byref(o))
        o.ned, o.maxlan, o.tol, o.restart, o.maxmv, o.lohi = ned, maxlan, tol, restart, maxmv, lohi
        if seed is not None:
            o.seed = seed
        o.threads, o.format, o.cta_threads = threads, fmt, cta
        return o

    def autotune(self, **kw):
        o = self.options(**kw)
        cfg = BatchConfig()
        rc = self.lib.trlx_batch_autotune(self.handle, C.byref(o), C.byref(cfg))
        if rc:
            raise RuntimeError(f"trlx_batch_autotune failed ({rc})")
        return cfg

    def solve(self, **kw):
        o = self.options(**kw)
        ev = np.zeros((self.nprob, o.ned))
        rs = np.zeros((self.nprob, o.ned))
        info = np.zeros((self.nprob, 4), dtype=np.int32)
        cfg = BatchConfig()
        rc = self.lib.trlx_batch_solve(self.handle, C.byref(o), ev.ctypes.data, rs.ctypes.data,
                                       info.ctypes.data, C.byref(cfg))
        if rc:
            raise RuntimeError(f"trlx_batch_solve failed ({rc})")
        self.ned = o.ned
        return BatchResult(ev, rs, info, cfg)

    def eigenvectors(self, p, out=None):
        """(ned, n) eigenvectors of problem p: a new numpy array, or `out`
        (a contiguous float64 numpy array or CUDA tensor of that size)."""
        n = self.lib.trlx_batch_size(self.handle, p)
        if out is None:
            out = np.zeros((self.ned, n))
        if hasattr(out, "data_ptr"):
            import torch
            if out.dtype != torch.float64 or not out.is_contiguous() or out.numel() != self.ned * n:
                raise ValueError("out must be a contiguous float64 tensor of ned * n elements")
            ptr = out.data_ptr()
        else:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self.ned * n:
                raise ValueError("out must be a contiguous float64 array of ned * n elements")
            ptr = out.ctypes.data
        rc = self.lib.trlx_batch_eigenvectors(self.handle, p, ptr)
        if rc:
            raise RuntimeError(f"trlx_batch_eigenvectors failed ({rc})")
        return out

    def close(self):
        if self.handle:
            self.lib.trlx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def seeded_start(seed, pid, n):
    """The start vector the batched solver uses for problem pid."""
    from .operators import uniform01
    s = (int(seed) + 0x9E3779B97F4A7C15 * (pid + 1)) & 0xFFFFFFFFFFFFFFFF
    return 2.0 * uniform01(s, np.arange(n, dtype=np.uint64)) - 1.0


def main(argv=None):
    """Solve a seeded batch of the benchmark family (L uniform in [48, 256],
    5-point Laplacian + U[0, 2] diagonal) and print throughput; used for
    profiling the persistent kernel."""
    import argparse
    import json
    import time
    from . import operators as ops
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--problems", type=int, default=512)
    ap.add_argument("--threads", type=int, default=0, help="0: autotuned; else the group size (128..1024)")
    ap.add_argument("--format", type=int, default=-1, help="-1: autotuned; 0 stencil, 1 CSR")
    ap.add_argument("--cta", type=int, default=0, help="0: autotuned; 1024 or 512 threads per CTA")
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args(argv)
    Ls = ops.batched_sizes(a.problems, seed=777)
    diags = [2.0 * ops.uniform01(1000 + k, np.arange(int(L) * int(L), dtype=np.uint64)) for k, L in enumerate(Ls)]
    b = Batch.stencil5(Ls, diags)
    kw = dict(ned=8, maxlan=32, tol=1e-8, restart=1, maxmv=100000, seed=4242, threads=a.threads, fmt=a.format,
              cta=a.cta)
    for _ in range(a.repeat):
        t0 = time.perf_counter()
        r = b.solve(**kw)
        dt = time.perf_counter() - t0
    print(json.dumps({"problems": a.problems, "seconds": dt, "problems_per_s": a.problems / dt,
                      "matvecs": int(r.info[:, 2].sum()), "solved": int((r.info[:, 1] >= 8).sum()),
                      "bucket_threads": list(r.config.bucket_threads),
                      "bucket_format": list(r.config.bucket_format), "cta_threads": r.config.cta_threads}))
    b.close()


if __name__ == "__main__":
    main()

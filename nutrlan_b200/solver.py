"""Python front end over the C ABI: built-in device operators and solves.

Example::

    from nutrlan_b200 import operators, DeviceOperator, solve
    A = operators.laplacian_2d(128)
    with DeviceOperator(A) as op:
        r = solve(op, ned=10, maxlan=64, lohi=-1, tol=1.4901e-8,
                  start=operators.start_vector(A.n))
    r.eval[:r.nec]

``evec`` placement decides residency: a torch CUDA tensor keeps everything on
the device (``device=True``), a numpy array gets the eigenvectors copied back
to the host.  The basis itself is always resident in GPU memory.
"""
import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._abi import TrlInfo, MATVEC
from ._lib import load, TrlxStats, TrlxOptions, TrlxTuneResult


class DeviceOperator:
    """A trlx_operator (CSR or SELL-C-32, real or complex) resident on the
    GPU.

    ``fmt="auto"`` creates the CSR form and runs trlx_operator_autotune
    (``maxlan`` sets the projection width it times): the operator keeps the
    faster of CSR and SELL-C-32 and the faster projection kernel forms for
    its solves; ``self.tune`` holds what was measured.  ``self.fmt`` is
    "csr"/"sell" for real and "zcsr"/"zsell" for complex operators."""

    def __init__(self, csr, fmt="csr", sigma=1, maxlan=128):
        lib = load()
        self.tune = None
        auto = fmt == "auto"
        if auto:
            fmt = "csr"
        self.lib = lib
        self.n = csr.n
        self.complex = np.iscomplexobj(csr.val)
        self.handle = C.c_void_p()
        rp = np.ascontiguousarray(csr.row_ptr, np.int64)
        ci = np.ascontiguousarray(csr.col, np.int32)
        if self.complex and fmt in ("sell", "zsell"):
            va = np.ascontiguousarray(csr.val, np.complex128)
            rc = lib.trlx_zsell_create(csr.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                       int(sigma), 0, C.byref(self.handle))
        elif self.complex:
            va = np.ascontiguousarray(csr.val, np.complex128)
            rc = lib.trlx_zcsr_create(csr.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 0,
                                      C.byref(self.handle))
        elif fmt == "sell":
            va = np.ascontiguousarray(csr.val, np.float64)
            rc = lib.trlx_sell_create(csr.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data,
                                      int(sigma), 0, C.byref(self.handle))
        else:
            va = np.ascontiguousarray(csr.val, np.float64)
            rc = lib.trlx_csr_create(csr.n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 0,
                                     C.byref(self.handle))
        if rc != 0:
            raise RuntimeError(f"trlx operator creation failed ({rc})")
        fmt = "sell" if fmt == "zsell" else ("csr" if fmt == "zcsr" else fmt)
        self.fmt = ("z" + fmt) if self.complex else fmt
        if auto:
            res = TrlxTuneResult()
            rc = lib.trlx_operator_autotune(self.handle, int(maxlan), C.byref(res))
            if rc != 0:
                self.close()
                raise RuntimeError(f"trlx_operator_autotune failed ({rc})")
            self.tune = res.as_dict()
            self.fmt = ("z" if self.complex else "") + self.tune["format"]
        self.nnz = lib.trlx_operator_nnz(self.handle)
        # The exported applier, used as `op` so the engine takes its fused path.
        name = "trlx_zmatvec" if self.complex else "trlx_matvec"
        self.applier = C.cast(getattr(lib, name), MATVEC)

    def close(self):
        if self.handle:
            self.lib.trlx_operator_destroy(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def residual_norms(op, evals, evecs):
    """||A z_i - lambda_i z_i|| / ||z_i|| for device eigenvectors (rows of a
    torch CUDA tensor), recomputed in FP64 with the built-in operator."""
    import torch
    lib = op.lib
    name = "trlx_zmatvec" if op.complex else "trlx_matvec"
    f = getattr(lib, name)
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    f.restype = None
    out = []
    y = torch.empty_like(evecs[0])
    for lam, z in zip(evals, evecs):
        z = z.contiguous()
        f(op.n, 1, z.data_ptr(), op.n, y.data_ptr(), op.n, op.handle)
        torch.cuda.synchronize()
        out.append(float(torch.linalg.vector_norm(y - float(lam) * z) / torch.linalg.vector_norm(z)))
    return np.array(out)


@dataclass
class SolveResult:
    eval: np.ndarray
    evec: object
    res: np.ndarray
    info: TrlInfo
    stats: TrlxStats = field(default=None)

    @property
    def nec(self):
        return self.info.nec

    @property
    def stat(self):
        return self.info.stat


def solve(op, ned, maxlan, lohi=-1, tol=1.4901e-8, restart=1, maxmv=0, start=None, mev=None,
          basis_bits=64, device=False, seed=0, evec=None, refine=None, profile=False):
    """Run trlan/ztrlan on a DeviceOperator through the C ABI.

    ``start`` (length n, numpy or CUDA tensor) becomes the initial vector
    (guess = 1); otherwise the reference's default ones vector is used.  ``device=True`` passes a torch
    CUDA tensor as evec, so the solver never copies vectors to the host.
    """
    lib = load()
    n = op.n
    mev = mev or ned + 1
    dtype = np.complex128 if op.complex else np.float64
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, lohi, ned, tol, restart, maxmv, None)
    info.mvparam = op.handle.value
    if start is not None:
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
    eval_ = np.zeros(mev)
    if device:
        import torch
        tdt = torch.complex128 if op.complex else torch.float64
        ev = evec if evec is not None else torch.zeros((mev, n), dtype=tdt, device="cuda")
        if start is not None:
            if hasattr(start, "data_ptr"):
                if start.data_ptr() != ev[0].data_ptr():
                    ev[0].copy_(start)
            else:
                ev[0].copy_(torch.as_tensor(np.asarray(start, dtype=dtype)))
        torch.cuda.synchronize()
        evec_ptr = ev.data_ptr()
    else:
        ev = np.zeros((mev, n), dtype=dtype)
        if start is not None:
            ev[0] = start.cpu().numpy() if hasattr(start, "data_ptr") else start
        evec_ptr = ev.ctypes.data
    wrk = np.zeros(mev)
    opts = TrlxOptions()
    lib.trlx_default_options(C.byref(opts))
    opts.basis_bits = basis_bits
    opts.seed = seed
    if refine is not None:
        opts.refine = 1 if refine else 0
    opts.profile = 1 if profile else 0
    if op.complex:
        misc = np.zeros(mev, dtype=np.complex128)
        lib.trlx_ztrlan(op.applier, C.byref(info), n, mev, eval_.ctypes.data, evec_ptr, n,
                        misc.ctypes.data, mev, None, 0, C.byref(opts))
        wrk = misc.real.copy()
    else:
        lib.trlx_trlan(op.applier, None, C.byref(info), n, mev, eval_.ctypes.data, evec_ptr, n,
                       mev, wrk.ctypes.data, C.byref(opts))
    stats = TrlxStats()
    lib.trlx_get_last_stats(C.byref(stats))
    return SolveResult(eval=eval_, evec=ev, res=wrk, info=info, stats=stats)

"""Loader for the in-tree libtrlan_b200.so.

The library must have been built (``python -c "import __graft_entry__ as g;
g.build()"`` or ``make -C nutrlan_b200/csrc``).  There is no fallback: a
missing or unloadable library raises ImportError.
"""
import ctypes as C
import os

from ._abi import (TrlInfo, MATVEC, USER_ORTHO, declare_common, c_int, c_double,
                   c_void_p)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                        "libtrlan_b200.so")


class TrlxStats(C.Structure):
    _fields_ = [
        ("seconds_total", c_double), ("seconds_op", c_double),
        ("seconds_orth", c_double), ("seconds_restart", c_double),
        ("basis_bytes", c_double), ("op_bytes", c_double),
        ("kernel_launches", C.c_longlong), ("cgs_passes", c_int),
        ("host_syncs", c_int), ("max_true_residual", c_double),
        ("kernel_seconds", c_double * 8), ("kernel_bytes", c_double * 8),
        ("kernel_count", C.c_longlong * 8), ("seconds_setup", c_double),
        ("speculative_steps", C.c_longlong), ("speculative_discarded", C.c_longlong),
    ]

    KERNEL_CLASSES = ("spmv", "project", "update", "normalize", "ritz", "dot", "other")

    def kernels(self):
        """{class: (seconds, bytes, launches)} for the profiled classes."""
        return {name: (self.kernel_seconds[i], self.kernel_bytes[i], self.kernel_count[i])
                for i, name in enumerate(self.KERNEL_CLASSES) if self.kernel_count[i]}


# int (*)(double *buf, long long count, int op, void *ctx)
ALLREDUCE_FN = C.CFUNCTYPE(c_int, C.POINTER(C.c_double), C.c_longlong, c_int, c_void_p)


class TrlxOptions(C.Structure):
    _fields_ = [("basis_bits", c_int), ("seed", C.c_ulonglong),
                ("stream", c_void_p), ("refine", c_int), ("profile", c_int)]


class TrlxTuneResult(C.Structure):
    """trlx_tune_result: what trlx_operator_autotune measured and kept."""
    _fields_ = [("format", c_int), ("project_form", c_int), ("spmv_ms", c_double * 2),
                ("project_ms", c_double * 5), ("columns", c_int), ("seconds", c_double),
                ("project_form32", c_int), ("project32_ms", c_double * 5)]

    FORMS = ("cpw8", "cpw12", "cpw16", "cpw16_shared_ptrs", "cpw8_staged")

    def as_dict(self):
        return {"format": ("csr", "sell")[self.format], "project_form": self.FORMS[self.project_form - 1],
                "spmv_forms_timed": 2 if self.spmv_ms[1] >= 0 else 1,
                "spmv_ms": {"csr": self.spmv_ms[0], "sell": self.spmv_ms[1]},
                "project_ms": {f: self.project_ms[i] for i, f in enumerate(self.FORMS) if self.project_ms[i] >= 0},
                "project_form32": self.FORMS[self.project_form32 - 1],
                "project32_ms": {f: self.project32_ms[i] for i, f in enumerate(self.FORMS)
                                 if self.project32_ms[i] >= 0},
                "columns": self.columns, "seconds": self.seconds}


def _declare(lib):
    declare_common(lib)
    P = C.POINTER
    lib.trlx_trlan.argtypes = list(lib.trlan.argtypes) + [P(TrlxOptions)]
    lib.trlx_trlan.restype = None
    lib.trlx_ztrlan.argtypes = list(lib.ztrlan.argtypes) + [P(TrlxOptions)]
    lib.trlx_ztrlan.restype = None
    lib.trlx_default_options.argtypes = [P(TrlxOptions)]
    lib.trlx_default_options.restype = None
    lib.trlx_get_last_stats.argtypes = [P(TrlxStats)]
    lib.trlx_get_last_stats.restype = None
    lib.trlx_version.restype = C.c_char_p
    for name in ("trlx_g_dot", "trlx_zg_dot", "trlx_g_dot_noalloc"):
        f = getattr(lib, name)
        f.argtypes = [c_int, c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_void_p, c_void_p,
                      c_void_p]
        f.restype = c_int
    lib.trlx_release_workspace.argtypes = []
    lib.trlx_release_workspace.restype = None
    for name in ("trlx_csr_create", "trlx_zcsr_create"):
        f = getattr(lib, name)
        f.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_int, P(c_void_p)]
        f.restype = c_int
    for name in ("trlx_sell_create", "trlx_zsell_create"):
        f = getattr(lib, name)
        f.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, P(c_void_p)]
        f.restype = c_int
    lib.trlx_operator_destroy.argtypes = [c_void_p]
    lib.trlx_operator_destroy.restype = None
    lib.trlx_operator_nnz.argtypes = [c_void_p]
    lib.trlx_operator_nnz.restype = C.c_longlong
    lib.trlx_operator_nrow.argtypes = [c_void_p]
    lib.trlx_operator_nrow.restype = c_int
    lib.trlx_operator_autotune.argtypes = [c_void_p, c_int, P(TrlxTuneResult)]
    lib.trlx_operator_autotune.restype = c_int
    for name in ("trlx_operator_set_project_form", "trlx_operator_set_project_form32"):
        getattr(lib, name).argtypes = [c_void_p, c_int]
        getattr(lib, name).restype = c_int
    # Block-row communicators and distributed operators.
    lib.trlx_comm_create_host.argtypes = [c_int, c_int, ALLREDUCE_FN, c_void_p, P(c_void_p)]
    lib.trlx_comm_create_host.restype = c_int
    lib.trlx_comm_nccl_id.argtypes = [c_void_p]
    lib.trlx_comm_nccl_id.restype = c_int
    lib.trlx_comm_create_nccl.argtypes = [c_int, c_int, c_void_p, P(c_void_p)]
    lib.trlx_comm_create_nccl.restype = c_int
    for name in ("trlx_comm_rank", "trlx_comm_size"):
        getattr(lib, name).argtypes = [c_void_p]
        getattr(lib, name).restype = c_int
    lib.trlx_comm_allreduce.argtypes = [c_void_p, c_void_p, C.c_longlong, c_int]
    lib.trlx_comm_allreduce.restype = c_int
    lib.trlx_comm_destroy.argtypes = [c_void_p]
    lib.trlx_comm_destroy.restype = None
    lib.trlx_init_info_comm.argtypes = [P(TrlInfo), c_void_p, c_int, c_int, c_int, c_int, C.c_double, c_int,
                                        c_int]
    lib.trlx_init_info_comm.restype = c_int
    lib.trlx_dist_csr_create.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int, P(c_void_p)]
    lib.trlx_dist_csr_create.restype = c_int
    lib.trlx_dist_sell_create.argtypes = [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                          P(c_void_p)]
    lib.trlx_dist_sell_create.restype = c_int
    lib.trlx_operator_halo.argtypes = [c_void_p]
    lib.trlx_operator_halo.restype = C.c_longlong
    lib.trlx_host_get_eval.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.trlx_host_get_eval.restype = c_int
    lib.trlx_host_tridiag_eig_last.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p]
    lib.trlx_host_tridiag_eig_last.restype = c_int
    lib.trlx_host_arrow_to_tridiag.argtypes = [c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                               c_void_p]
    lib.trlx_host_arrow_to_tridiag.restype = c_int
    lib.trlx_host_sym_eig.argtypes = [c_int, c_void_p, c_int, c_void_p]
    lib.trlx_host_sym_eig.restype = c_int
    lib.trlx_host_shuffle_eig.argtypes = [c_int, c_int, c_void_p, c_void_p, P(TrlInfo),
                                          P(c_int), c_int]
    lib.trlx_host_shuffle_eig.restype = None
    lib.trlx_host_convergence_test.argtypes = [c_int, c_void_p, c_void_p, P(TrlInfo), c_void_p]
    lib.trlx_host_convergence_test.restype = None
    lib.trlx_host_sort_eig.argtypes = [c_int, c_int, c_int, c_double, c_void_p, c_void_p]
    lib.trlx_host_sort_eig.restype = None
    lib.trlx_host_set_locking.argtypes = [c_int, c_int, c_void_p, c_void_p, c_void_p, c_double,
                                          P(c_int)]
    lib.trlx_host_set_locking.restype = None
    lib.trlx_host_sort2.argtypes = [c_int, c_void_p, c_void_p]
    lib.trlx_host_sort2.restype = None
    return lib


_LIB = None


def load():
    """Return the loaded library (raises ImportError if it is not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libtrlan_b200.so not found at {LIB_PATH}; build it with "
                "`make -C nutrlan_b200/csrc` (the CUDA path has no fallback)")
        _LIB = _declare(C.CDLL(LIB_PATH))
    return _LIB


__all__ = ["load", "LIB_PATH", "TrlInfo", "TrlxStats", "TrlxOptions", "TrlxTuneResult", "MATVEC",
           "USER_ORTHO"]

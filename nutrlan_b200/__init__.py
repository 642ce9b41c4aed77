"""nutrlan_b200: thick-restart Lanczos for NVIDIA B200 behind nuTRLan's C API.

The product is the shared library ``nutrlan_b200/lib/libtrlan_b200.so``
(headers in ``include/``).  This package loads it through ctypes and adds
Python conveniences: ``solve`` runs a real or complex solve on a built-in
device operator with the basis resident in GPU memory, and
``nutrlan_b200.operators`` builds the synthetic operator families.
"""
from ._abi import TrlInfo, TrlDComplex, MATVEC, USER_ORTHO  # noqa: F401
from ._lib import load, LIB_PATH, TrlxStats, TrlxOptions  # noqa: F401
from .solver import DeviceOperator, solve, SolveResult, residual_norms  # noqa: F401

__version__ = "0.1.0"

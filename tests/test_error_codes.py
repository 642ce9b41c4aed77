"""Argument errors of trlan() (reference trl_clear_counter,
SRC/trlan.c:1217-1349): on the same bad inputs this library returns the
reference's info->stat codes, before any device work (so no GPU is needed),
and leaves the same adjusted fields (ned, maxlan, klan, tol) in trl_info:

* -1: nrow differs from the nloc the info was set up with;
* -2: evec leading dimension below nrow;
* -4: fewer than 10 rows;
* -5: fewer than 5 basis vectors after the maxlan adjustments
  (maxlan < ned + 3 resets it to ned + min(ned, 20) + log(ntot)).

A non-error combination is included only through its field adjustments,
which trl_clear_counter makes before the solve starts (checked with an
error-code case that triggers the same adjustments: ned reduced to mev)."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import TrlInfo, MATVEC
from oracle import ref


def _run(lib, n, ned, mev, lde, maxlan=20, init_n=None, tol=1e-8):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), init_n or n, maxlan, -1, ned, tol, 1, 1000, None)
    info.verbose = -1
    evec = np.zeros(max(mev, 1) * max(lde, n) + 8)
    eval_ = np.zeros(max(mev, 1))
    wrk = np.zeros(max(maxlan, 1) * (max(maxlan, 1) + 10))
    cb = MATVEC(lambda *a: None)
    lib.trlan(cb, None, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, lde, wrk.size,
              wrk.ctypes.data)
    return info


CASES = [
    # n, ned, mev, lde, maxlan, init_n, tol, code
    (8, 2, 4, 8, 20, None, 1e-8, -4),
    (100, 4, 6, 90, 20, None, 1e-8, -2),
    (90, 4, 6, 90, 20, 100, 1e-8, -1),
    (10, 1, 1, 10, 2, None, 1e-8, -5),
    (8, 6, 4, 8, 3, None, 2.0, -4),      # ned > mev reduced to mev, tol >= 1 reset, maxlan reset
    (100, 4, 6, 50, 2, None, 0.0, -2),   # tol <= DBL_MIN set to eps, maxlan reset to ned + ned + log(n)
]


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
@pytest.mark.parametrize("n,ned,mev,lde,maxlan,init_n,tol,code", CASES)
def test_error_codes_match_reference(lib, n, ned, mev, lde, maxlan, init_n, tol, code):
    ours = _run(lib, n, ned, mev, lde, maxlan, init_n, tol)
    theirs = _run(ref.load(), n, ned, mev, lde, maxlan, init_n, tol)
    assert ours.stat == theirs.stat == code, (ours.stat, theirs.stat)
    for f in ("ned", "nec", "maxlan", "klan", "tol", "matvec", "locked"):
        assert getattr(ours, f) == getattr(theirs, f), (f, getattr(ours, f), getattr(theirs, f))

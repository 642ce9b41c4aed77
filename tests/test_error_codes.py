"""Argument errors of trlan() (reference trl_clear_counter,
SRC/trlan.c:1217-1349): on the same bad inputs this library returns the
reference's info->stat codes, before any device work (so no GPU is needed):
a problem smaller than 10 rows (-4) and an evec leading dimension below
nrow (-2)."""
import ctypes as C

import numpy as np
import pytest

from nutrlan_b200 import TrlInfo, MATVEC
from oracle import ref


def _run(lib, n, ned, mev, lde, maxlan=20):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), n, maxlan, -1, ned, 1e-8, 1, 1000, None)
    info.verbose = -1
    evec = np.zeros(max(mev, 1) * max(lde, n) + 8)
    eval_ = np.zeros(max(mev, 1))
    wrk = np.zeros(maxlan * (maxlan + 10))
    cb = MATVEC(lambda *a: None)
    lib.trlan(cb, None, C.byref(info), n, mev, eval_.ctypes.data, evec.ctypes.data, lde, wrk.size,
              wrk.ctypes.data)
    return info.stat


@pytest.mark.skipif(not ref.available(), reason="reference oracle not built")
@pytest.mark.parametrize("n,ned,mev,lde,code", [(8, 2, 4, 8, -4), (100, 4, 6, 90, -2)])
def test_error_codes_match_reference(lib, n, ned, mev, lde, code):
    ours = _run(lib, n, ned, mev, lde)
    theirs = _run(ref.load(), n, ned, mev, lde)
    assert ours == theirs == code, (ours, theirs)

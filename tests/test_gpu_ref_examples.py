"""The reference's own example programs, compiled unchanged from the
reference tree and linked against libtrlan_b200.so (tests/ref_examples/
Makefile, run by build()), run on the GPU:

* examples/simple.c (diag((i+1)^2), n = 1897, ned 5, maxlan 200, host evec
  and host operator), built against the reference's INC/ headers and
  against this library's include/: its TRL_CHECK_RITZ table must list
  exact[i] = (i+1)^2 (examples/simple.c:90) for every returned pair, with
  the Ritz values within 10 tol * exact[i] of it and the computed residual
  norms within the tolerance, and the printed MATVEC count close to the
  reference's own 3403 (tests/golden/reference_runs.json "simple_diag").
* examples/test_ztrlan.c (complex diag((i+1)^2), n = 1000, ned 100,
  maxlan 200, restart 7): the program itself must print its SUCCESS line
  (100 converged, ztrl_check_ritz's checks passed).

The binaries exist only where the reference sources were available when
the library was built; without them the test is skipped with that reason.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "ref_examples", "_bin")
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_runs.json")))
FLOAT = re.compile(r"[-+]?\d\.\d+e[-+]\d{2,3}")


def run(name, tmp_path):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference sources: make -C tests/ref_examples)")
    p = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return p.stdout


@pytest.mark.parametrize("name", ["simple", "simple_b200hdr"])
def test_reference_simple_example_runs_unchanged(name, tmp_path):
    out = run(name, tmp_path)
    mv = re.search(r"MATVEC:\s*(\d+)", out)
    assert mv, out[-3000:]
    g = GOLD["simple_diag"]
    assert abs(int(mv.group(1)) - g["matvec"]) <= 0.05 * g["matvec"], (mv.group(1), g["matvec"])
    lines = out.splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.startswith("TRL_CHECK_RITZ"))
    rows = []
    for ln in lines[k + 2:]:
        try:
            alpha = float(ln[:21])
        except ValueError:
            break
        rows.append([alpha] + [float(t) for t in FLOAT.findall(ln[21:])])
    assert len(rows) >= g["ned"], out[-3000:]
    tol = 1.4901e-8
    for i, r in enumerate(rows):
        alpha, res, resdiff, err, rqdiff, acterr, exact = r
        assert exact == pytest.approx((i + 1.0) ** 2, rel=1e-3)        # printed to 4 digits
        assert abs(acterr) <= 10 * tol * (i + 1.0) ** 2, r
        assert res <= tol * 1897.0 ** 2, r
        assert abs(resdiff) <= 1e-5, r
    m = min(len(rows), len(g["eval"]))
    np.testing.assert_allclose([r[0] for r in rows[:m]], g["eval"][:m], rtol=1e-6)


def test_reference_complex_example_runs_unchanged(tmp_path):
    out = run("test_ztrlan", tmp_path)
    assert "SUCCESS (100 converged)" in out, out[-3000:]
    assert "ERROR" not in out

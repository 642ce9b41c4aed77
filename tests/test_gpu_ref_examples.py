"""The reference's own example programs, compiled unchanged from the
reference tree (tests/ref_examples/Makefile, run by build()), linked once
against libtrlan_b200.so and once against the reference library (oracle/_ref),
and run side by side; the B200 build runs on the GPU.

* examples/simple.c (diag((i+1)^2), n = 1897, ned 5, maxlan 200, host evec
  and host operator), built against the reference's INC/ headers and
  against this library's include/: every row of its TRL_CHECK_RITZ table
  has exact[i] = (i+1)^2 (examples/simple.c:90), Ritz values within
  10 tol * exact[i] of it, computed residual norms within tol * ||A|| and
  agreeing with the solver's estimates (the program's own 1e-5 check); the
  operator count of the execution summary within 5% of the reference
  build's, and the Ritz values equal to the reference build's to 1e-6.
* examples/test_ztrlan.c (complex diag((i+1)^2), n = 1000, ned 100,
  maxlan 200, restart 7): both builds report 100 converged pairs with the
  same verdict line (the reference's own build prints "ERROR (100
  converged)" too: its check compares the actual error with ten times an
  estimate floored at machine epsilon times the largest value, which
  1e-10-accurate eigenvalues exceed); the two tables agree row by row
  (Ritz values within the sum of the two builds' actual errors, actual
  errors of this build no larger than 10x the reference's largest).

The binaries exist only where the reference sources were available when
the library was built; without them the test is skipped with that reason.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "ref_examples", "_bin")
FLOAT = re.compile(r"[-+]?\d\.\d+e[-+]\d{2,3}")


def run(name, tmp_path):
    exe = os.path.join(BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (needs the reference sources: make -C tests/ref_examples)")
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
    d = tmp_path / name
    d.mkdir()
    p = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stderr[-2000:]
    # Diagnostics go to stdout, or to the per-process log file a program
    # names with trl_set_debug (the reference's own build names it after the
    # rank alone: its trl_pe_filename loses the prefix with this C library).
    logs = "".join(f.read_text() for f in sorted(d.iterdir()) if f.is_file() and f.name != "error.txt")
    return p.stdout + "\n" + logs


def table(out):
    lines = out.splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.startswith("TRL_CHECK_RITZ"))
    rows = []
    for ln in lines[k + 2:]:
        try:
            alpha = float(ln[:21])
        except ValueError:
            break
        rows.append([alpha] + [float(t) for t in FLOAT.findall(ln[21:])])
    return np.array(rows)


def applied(out):
    m = re.search(r"Times the operator is applied:\s*(\d+)", out)
    assert m, out[-3000:]
    return int(m.group(1))


@pytest.mark.parametrize("name", ["simple", "simple_b200hdr"])
def test_reference_simple_example_runs_unchanged(name, tmp_path):
    ours, theirs = run(name, tmp_path), run("simple_ref", tmp_path)
    mv, mv_ref = applied(ours), applied(theirs)
    assert abs(mv - mv_ref) <= 0.05 * mv_ref, (mv, mv_ref)
    rows, ref_rows = table(ours), table(theirs)
    assert len(rows) >= 5, ours[-3000:]
    tol, anrm = 1.4901e-8, 1897.0 ** 2
    for i, r in enumerate(rows):
        alpha, res, resdiff, err, rqdiff, acterr, exact = r
        assert exact == pytest.approx((i + 1.0) ** 2, rel=1e-3)        # printed to 4 digits
        assert abs(acterr) <= 10 * tol * (i + 1.0) ** 2, r
        assert res <= tol * anrm, r
        assert abs(resdiff) <= 1e-5, r
    m = min(len(rows), len(ref_rows))
    np.testing.assert_allclose(rows[:m, 0], ref_rows[:m, 0], rtol=1e-6)
    print(f"{name}: {mv} applications (reference build {mv_ref}), {len(rows)} pairs "
          f"(reference {len(ref_rows)}), max |actual error| {np.abs(rows[:, 5]).max():.2e} "
          f"(reference {np.abs(ref_rows[:, 5]).max():.2e})")


def test_reference_complex_example_runs_unchanged(tmp_path):
    ours, theirs = run("test_ztrlan", tmp_path), run("test_ztrlan_ref", tmp_path)
    verdict = [ln.strip() for ln in ours.splitlines() if "converged" in ln and ("SUCCESS" in ln or "ERROR" in ln
                                                                               or "only" in ln)]
    verdict_ref = [ln.strip() for ln in theirs.splitlines() if "converged" in ln and
                   ("SUCCESS" in ln or "ERROR" in ln or "only" in ln)]
    assert verdict == verdict_ref and "100 converged" in verdict[0], (verdict, verdict_ref)
    rows, ref_rows = table(ours), table(theirs)
    assert rows.shape == ref_rows.shape == (100, 7)
    # both builds' values carry actual errors up to ~1e-9 (their own
    # "act. error" column): they agree to within the sum of those errors
    np.testing.assert_allclose(rows[:, 0], ref_rows[:, 0], rtol=1e-13,
                               atol=np.abs(rows[:, 5]).max() + np.abs(ref_rows[:, 5]).max())
    np.testing.assert_allclose(rows[:, 6], (np.arange(100) + 1.0) ** 2, rtol=1e-3)
    assert np.abs(rows[:, 5]).max() <= 10 * np.abs(ref_rows[:, 5]).max()
    print(f"test_ztrlan: {verdict[0]} in both builds; max |actual error| {np.abs(rows[:, 5]).max():.2e} "
          f"(reference {np.abs(ref_rows[:, 5]).max():.2e})")

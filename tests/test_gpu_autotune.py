"""Single-solve autotuner (trlx_operator_autotune): it keeps the faster of
the measured CSR / SELL-C-32 forms and of the measured projection forms
(one choice per basis storage width), the tuned operator computes the same
product, and a solve with it returns the reference's eigenvalues (the golden
Anderson 64^3 run of tests/golden/config_runs.json) like the untuned CSR
operator does, over a 64-bit and over a 32-bit basis."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from nutrlan_b200 import operators as ops, DeviceOperator, solve, load
from nutrlan_b200._lib import TrlxTuneResult

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))


def product(op, x):
    lib = load()
    f = lib.trlx_matvec
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    f.restype = None
    xd = torch.as_tensor(x).cuda()
    yd = torch.empty_like(xd)
    f(op.n, 1, xd.data_ptr(), op.n, yd.data_ptr(), op.n, op.handle)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("L", [24, 96])
def test_autotune_keeps_the_faster_measured_forms(L):
    A = ops.anderson_3d(L, W=4.0, seed=5)
    x = ops.start_vector(A.n, seed=3)
    with DeviceOperator(A, fmt="auto", maxlan=64) as op:
        t = op.tune
        print(f"L={L}: {t}")
        assert t["format"] in ("csr", "sell") and op.fmt == t["format"]
        sp = t["spmv_ms"]
        assert min(sp.values()) > 0
        assert sp[t["format"]] == min(sp.values())
        pm = t["project_ms"]
        assert t["project_form"] in pm and pm[t["project_form"]] == min(pm.values())
        pm32 = t["project32_ms"]
        assert len(pm) == 5 and len(pm32) == 5 and min(pm32.values()) > 0
        assert pm32[t["project_form32"]] == min(pm32.values())
        assert t["columns"] == 32
        y = product(op, x)
    np.testing.assert_allclose(y, A.matvec(x), rtol=1e-13, atol=1e-13)


def test_autotuned_solve_matches_reference():
    g = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))["anderson64_full"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    with DeviceOperator(A, fmt="auto", maxlan=g["maxlan"]) as op:
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=ops.start_vector(A.n, seed=g["start_seed"]), mev=g["mev"], device=True)
    assert r.stat == 0 and r.nec >= g["ned"]
    got, want = np.sort(r.eval[:g["ned"]]), np.sort(np.array(g["eval"])[:g["ned"]])
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-10
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"]


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5])
def test_every_projection_form_solves_to_the_reference(form):
    """Each form the autotuner can keep (8, 12, 16 columns per warp; 16 with
    the pointer table in shared memory; 8 per warp over 16 warps, staged
    through shared memory by cp.async), set on the operator, returns the
    reference's Anderson 64^3 eigenvalues."""
    g = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))["anderson64_full"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    lib = load()
    with DeviceOperator(A, fmt="sell") as op:
        assert lib.trlx_operator_set_project_form(op.handle, form) == 0
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=ops.start_vector(A.n, seed=g["start_seed"]), mev=g["mev"], device=True)
    assert r.stat == 0 and r.nec >= g["ned"]
    got, want = np.sort(r.eval[:g["ned"]]), np.sort(np.array(g["eval"])[:g["ned"]])
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-10
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"]


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5])
def test_every_fp32_basis_projection_form_solves_to_the_reference(form):
    """The same over an FP32 basis (FP64 recurrence, dots and refinement),
    the form set with trlx_operator_set_project_form32: the reference's
    eigenvalues to 1e-10 and true residuals <= tol * ||A||; the refinement
    adds up to 9 applications per pair per pass."""
    from nutrlan_b200 import residual_norms
    g = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))["anderson64_full"]
    A = ops.anderson_3d(g["L"], W=g["W"], seed=g["pot_seed"])
    lib = load()
    with DeviceOperator(A, fmt="sell") as op:
        assert lib.trlx_operator_set_project_form32(op.handle, form) == 0
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=ops.start_vector(A.n, seed=g["start_seed"]), mev=g["mev"], device=True, basis_bits=32)
        assert r.stat == 0 and r.nec >= g["ned"]
        res = residual_norms(op, r.eval[:r.nec], r.evec[:r.nec])
    got, want = np.sort(r.eval[:g["ned"]]), np.sort(np.array(g["eval"])[:g["ned"]])
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-10
    assert np.all(res <= g["tol"] * r.info.anrm * 1.01)
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"] + 9 * 3 * g["ned"]


@pytest.mark.parametrize("form", [0, 3, 4, 5])
def test_complex_autotune_and_forms_solve_to_the_reference(form):
    """A complex operator tunes its format (complex CSR or SELL-C-32) and
    its projection form (pointer table in registers or in shared memory, or
    the staged form); with each form, and with the tuned ones, the Peierls
    256^2 solve returns the reference's eigenvalues."""
    g = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))["peierls256_full"]
    P = ops.peierls_2d(g["L"], phi=g["phi"], W=g["W"], seed=g["pot_seed"])
    lib = load()
    fmt = "auto" if form == 0 else "csr"
    with DeviceOperator(P, fmt=fmt, maxlan=g["maxlan"]) as op:
        if form == 0:
            t = op.tune
            print(t)
            forms = {"cpw16", "cpw16_shared_ptrs", "cpw8_staged"}
            assert t["spmv_forms_timed"] == 2 and set(t["project_ms"]) == forms
            assert t["spmv_ms"][t["format"]] == min(t["spmv_ms"].values())
            assert op.fmt == "z" + t["format"]
            assert t["project_ms"][t["project_form"]] == min(t["project_ms"].values())
            assert set(t["project32_ms"]) == forms
            assert t["project32_ms"][t["project_form32"]] == min(t["project32_ms"].values())
        else:
            assert lib.trlx_operator_set_project_form(op.handle, form) == 0
        x0 = ops.start_vector(P.n) + 1j * ops.start_vector(P.n, seed=99)
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=x0, mev=g["mev"], device=True)
    assert r.stat == 0 and r.nec >= g["ned"]
    got, want = np.sort(r.eval[:g["ned"]]), np.sort(np.array(g["eval"])[:g["ned"]])
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-10
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"]


@pytest.mark.parametrize("form", [3, 4, 5])
def test_complex64_basis_forms_solve_to_the_reference(form):
    """Each complex form over a complex64 basis (complex128 recurrence, dots
    and refinement), set with trlx_operator_set_project_form32."""
    from nutrlan_b200 import residual_norms
    g = json.load(open(os.path.join(HERE, "golden", "config_runs.json")))["peierls256_full"]
    P = ops.peierls_2d(g["L"], phi=g["phi"], W=g["W"], seed=g["pot_seed"])
    lib = load()
    with DeviceOperator(P, fmt="csr") as op:
        assert lib.trlx_operator_set_project_form32(op.handle, form) == 0
        x0 = ops.start_vector(P.n) + 1j * ops.start_vector(P.n, seed=99)
        r = solve(op, ned=g["ned"], maxlan=g["maxlan"], maxmv=100000, tol=g["tol"], restart=g["restart"],
                  start=x0, mev=g["mev"], device=True, basis_bits=32)
        assert r.stat == 0 and r.nec >= g["ned"]
        res = residual_norms(op, r.eval[:r.nec], r.evec[:r.nec])
    got, want = np.sort(r.eval[:g["ned"]]), np.sort(np.array(g["eval"])[:g["ned"]])
    assert np.max(np.abs(got - want) / np.abs(want)) <= 1e-10
    assert np.all(res <= g["tol"] * r.info.anrm * 1.01)
    assert abs(r.info.matvec - g["matvec"]) <= 0.05 * g["matvec"] + 9 * 3 * g["ned"]


def test_autotune_rejects_operators_it_does_not_tune():
    lib = load()
    res = TrlxTuneResult()
    A = ops.laplacian_2d(32)
    with DeviceOperator(A, fmt="sell") as op:
        assert lib.trlx_operator_autotune(op.handle, 32, C.byref(res)) == -1
    assert lib.trlx_operator_autotune(None, 32, C.byref(res)) == -1
    assert lib.trlx_operator_set_project_form(None, 1) == -1
    assert lib.trlx_operator_set_project_form32(None, 1) == -1
    with DeviceOperator(A, fmt="csr") as op:
        assert lib.trlx_operator_set_project_form32(op.handle, 6) == -1
        assert lib.trlx_operator_set_project_form(op.handle, -1) == -1

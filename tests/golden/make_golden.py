"""Generate tests/golden/reference_runs.json from the reference nuTRLan
library built under oracle/_ref (run in a checkout where the reference
sources were available: ``make -C oracle`` first).

Each case records the reference's own output on a seeded operator and start
vector: converged eigenvalues, nec, matvec and restart counts.  The operators
are the reference's example operator (examples/simple.c: diag((i+1)^2),
n=1897, ned=5, maxlan=200, restart 1, ones start vector), the complex
diagonal of examples/test_ztrlan.c (reduced to n=1000, ned=10), the
benchmark's 128^2 Laplacian and small Anderson / Peierls instances.

    OPENBLAS_NUM_THREADS=1 python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from nutrlan_b200 import operators as ops  # noqa: E402
from oracle import ref  # noqa: E402


def record(r, extra=None):
    i = r["info"]
    out = {"stat": i.stat, "nec": i.nec, "matvec": i.matvec, "nloop": i.nloop,
           "north": i.north, "eval": [float(v) for v in r["eval"][: max(i.nec, 0)]]}
    out.update(extra or {})
    return out


def main():
    ref.build()
    cases = {}
    n = 1897
    d = (np.arange(n) + 1.0) ** 2
    cases["simple_diag"] = record(
        ref.trlan(lambda x: d * x, n, ned=5, maxlan=200, restart=1, maxmv=2000000,
                  start=np.ones(n), mev=100),
        {"n": n, "ned": 5, "maxlan": 200, "restart": 1, "mev": 100})
    A = ops.laplacian_2d(128)
    x0 = ops.start_vector(A.n)
    for rs in range(1, 8):
        cases[f"laplace128_r{rs}"] = record(
            ref.trlan(A.matvec, A.n, ned=10, maxlan=64, restart=rs, maxmv=100000, start=x0),
            {"L": 128, "ned": 10, "maxlan": 64, "restart": rs, "seed": 12345})
    B = ops.anderson_3d(16, W=4.0, seed=11)
    xb = ops.start_vector(B.n)
    for rs in (1, 7):
        cases[f"anderson16_r{rs}"] = record(
            ref.trlan(B.matvec, B.n, ned=8, maxlan=40, restart=rs, maxmv=100000, start=xb),
            {"L": 16, "W": 4.0, "pot_seed": 11, "ned": 8, "maxlan": 40, "restart": rs})
    nz = 1000
    dz = ((np.arange(nz) + 1.0) ** 2).astype(np.complex128)
    xz = ops.start_vector(nz) + 0.5j * ops.start_vector(nz, seed=99)
    cases["zdiag1000"] = record(
        ref.ztrlan(lambda x: dz * x, nz, ned=10, maxlan=64, restart=7, maxmv=100000, start=xz),
        {"n": nz, "ned": 10, "maxlan": 64, "restart": 7})
    P = ops.peierls_2d(64, phi=1.0 / 16.0)
    xp = ops.start_vector(P.n) + 1j * ops.start_vector(P.n, seed=7)
    cases["peierls64"] = record(
        ref.ztrlan(P.matvec, P.n, ned=8, maxlan=48, restart=1, maxmv=100000, start=xp),
        {"L": 64, "phi": 1.0 / 16.0, "ned": 8, "maxlan": 48, "restart": 1})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_runs.json")
    with open(path, "w") as f:
        json.dump(cases, f, indent=1)
    print(f"wrote {path}: {len(cases)} cases")


if __name__ == "__main__":
    main()

"""Generate tests/golden/config_runs.json: the reference nuTRLan library's
own results at the benchmark configurations' stated sizes.

Run where the reference sources are available (``make -C oracle`` builds
oracle/_ref from them); the GPU tests read only the committed JSON:

    OMP_NUM_THREADS=8 OPENBLAS_NUM_THREADS=8 python tests/golden/make_config_golden.py [case ...]

Cases (operators and start vectors from nutrlan_b200.operators, whose
counter-based random numbers are reproduced bit for bit on the GPU):

* ``anderson256_cycle``  Anderson 256^3 (W = 4, potential seed 2024), smallest
  32, maxlan = maxmv = 128: one thick-restart cycle.  Records the 32 Ritz
  values and residual estimates after the cycle (``trlan`` returns
  min(mev - 1, ned) pairs when maxmv stops it).
* ``anderson64_full``    Anderson 64^3, smallest 32, maxlan 128, tol 1e-8, full
  solve.
* ``peierls2048_cycle``  Peierls 2048^2 (flux 1/64, disorder U[-1, 1], seed
  4242), smallest 16, maxlan = maxmv = 96: one ``ztrlan`` cycle.
* ``peierls256_full``    Peierls 256^2 (same family), smallest 16, maxlan 96,
  tol 1e-8, full solve.
* ``batched_sample``     16 problems of the 4096-problem batch (sizes seed 777,
  diagonals seed 1000 + k, start vector ``seeded_start(4242, k, n)``) spread
  over the size range, smallest 8, maxlan 32, tol 1e-8, each solved by
  ``trlan``.
* ``wells256``           4 held-out Gaussian-well operators (seeds 10^6 ..
  10^6 + 3), smallest 16, maxlan 48, tol 1e-8, plain start vector.

Each record keeps the reference's eigenvalues, residual norms (real
solver), stat / nec / matvec / nloop / north, the wall time and the host
thread count.  A second run of a case with another BLAS thread count
(``--threads``) is stored under ``<case>@<threads>t`` so the tests can see
how far rounding alone moves the reference's own results.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from nutrlan_b200 import operators as ops  # noqa: E402
from nutrlan_b200.batched import seeded_start  # noqa: E402
from oracle import ref  # noqa: E402

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "config_runs.json")


def rec(r, **extra):
    i = r["info"]
    k = i.nec if i.nec > 0 else extra.pop("kept", 0)
    out = {"stat": i.stat, "nec": i.nec, "matvec": i.matvec, "nloop": i.nloop, "north": i.north,
           "nrand": i.nrand, "anrm": i.anrm, "seconds": r["seconds"],
           "eval": [float(v) for v in r["eval"][:k]]}
    if r.get("res") is not None:
        out["res"] = [float(v) for v in r["res"][:k]]
    out.update(extra)
    return out


def anderson256_cycle():
    A = ops.anderson_3d(256, W=4.0, seed=2024)
    r = ref.trlan_csr(A, ned=32, maxlan=128, tol=1e-8, restart=1, maxmv=128,
                      start=ops.start_vector(A.n), mev=33)
    return rec(r, kept=32, L=256, W=4.0, pot_seed=2024, ned=32, maxlan=128, maxmv=128, restart=1,
               start_seed=12345, mev=33)


def anderson64_full():
    A = ops.anderson_3d(64, W=4.0, seed=2024)
    r = ref.trlan_csr(A, ned=32, maxlan=128, tol=1e-8, restart=1, maxmv=100000,
                      start=ops.start_vector(A.n), mev=33)
    return rec(r, L=64, W=4.0, pot_seed=2024, ned=32, maxlan=128, tol=1e-8, restart=1, start_seed=12345,
               mev=33)


def _peierls_start(n):
    return ops.start_vector(n) + 1j * ops.start_vector(n, seed=99)


def peierls2048_cycle():
    A = ops.peierls_2d(2048, phi=1.0 / 64.0, W=2.0, seed=4242)
    r = ref.trlan_csr(A, ned=16, maxlan=96, tol=1e-8, restart=1, maxmv=96, start=_peierls_start(A.n),
                      mev=17)
    return rec(r, kept=16, L=2048, phi=1.0 / 64.0, W=2.0, pot_seed=4242, ned=16, maxlan=96, maxmv=96,
               restart=1, mev=17)


def peierls256_full():
    A = ops.peierls_2d(256, phi=1.0 / 64.0, W=2.0, seed=4242)
    r = ref.trlan_csr(A, ned=16, maxlan=96, tol=1e-8, restart=1, maxmv=100000, start=_peierls_start(A.n),
                      mev=17)
    return rec(r, L=256, phi=1.0 / 64.0, W=2.0, pot_seed=4242, ned=16, maxlan=96, tol=1e-8, restart=1, mev=17)


BATCH_COUNT, BATCH_SAMPLE = 4096, 16


def batched_sample():
    Ls = ops.batched_sizes(BATCH_COUNT, seed=777)
    out = []
    for k in np.linspace(0, BATCH_COUNT - 1, BATCH_SAMPLE).astype(int):
        L = int(Ls[k])
        diag = 2.0 * ops.uniform01(1000 + int(k), np.arange(L * L, dtype=np.uint64))
        A = ops.laplacian_2d(L, diag=diag)
        r = ref.trlan_csr(A, ned=8, maxlan=32, tol=1e-8, restart=1, maxmv=100000,
                          start=seeded_start(4242, int(k), A.n))
        out.append(rec(r, index=int(k), L=L))
    return {"count": BATCH_COUNT, "sizes_seed": 777, "diag_seed": "1000 + index", "start_seed": 4242,
            "ned": 8, "maxlan": 32, "tol": 1e-8, "restart": 1, "problems": out}


def wells256():
    out = []
    for s in range(10 ** 6, 10 ** 6 + 4):
        A, _ = ops.wells_2d(256, seed=s)
        r = ref.trlan_csr(A, ned=16, maxlan=48, tol=1e-8, restart=1, maxmv=100000,
                          start=ops.start_vector(A.n))
        out.append(rec(r, seed=s))
    return {"L": 256, "ned": 16, "maxlan": 48, "tol": 1e-8, "restart": 1, "problems": out}


CASES = {f.__name__: f for f in (anderson256_cycle, anderson64_full, peierls2048_cycle, peierls256_full,
                                 batched_sample, wells256)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*", default=list(CASES))
    ap.add_argument("--suffix", default="", help="store under <case><suffix> (e.g. @1t)")
    a = ap.parse_args()
    ref.build()
    data = {}
    if os.path.exists(PATH):
        with open(PATH) as f:
            data = json.load(f)
    threads = os.environ.get("OPENBLAS_NUM_THREADS", str(os.cpu_count()))
    for name in a.cases:
        t0 = time.perf_counter()
        r = CASES[name]()
        r["host_threads"] = int(threads)
        data[name + a.suffix] = r
        with open(PATH, "w") as f:
            json.dump(data, f, indent=1)
        print(f"{name}{a.suffix}: {time.perf_counter() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()

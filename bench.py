#!/usr/bin/env python
"""Benchmark: thick-restart Lanczos on the 3D Anderson model, 256^3.

Workload (the configuration the headline metric is quoted on): real
symmetric FP64 operator, periodic 7-point stencil with hopping -1 and a
seeded diagonal potential uniform[-2, 2] (W = 4), n = 16,777,216, CSR
(117.4M entries); smallest ned = 32 eigenpairs, maxlan = 128, tol = 1e-8,
start vector seeded uniform[-1, 1].

A step is one trlan() call bounded to one thick-restart cycle
(maxmv = maxlan = 128): 128 Lanczos steps, each one fused SpMV + alpha, one
full classical Gram-Schmidt pass against the growing basis (1..128 vectors),
normalisation, then the Ritz recombination V*Y of the 32 wanted vectors.
The metric is Lanczos steps (matvec + full reorthogonalisation) per second.

* value: device-resident inputs (CSR and evec on the GPU before timing).
* e2e:   the same call through the C ABI with host buffers: the CSR arrays
         and the start vector are copied host->device and the eigenvectors
         device->host inside the timed region, every step; the buffers are
         page-locked host memory, and e2e.pageable repeats the calls with
         pageable numpy arrays (an unchanged nuTRLan program's case).
* roofline: the dominant kernel's algorithmic bytes / its CUDA-event time
         measured inside the engine on its own stream (trlx_options.profile).
* cpu_baseline / --impl reference: the reference nuTRLan library
         (oracle/_ref, built from the reference sources with OpenBLAS) on the
         same operator with a compiled OpenMP CSR callback, on a bounded
         sample: the first 32 Lanczos steps (maxlan = maxmv = 32) of the same
         solve; the reference arm's config.workload says so.  The sample's
         basis is 4x smaller on average than a full cycle's, so per-step CPU
         throughput is overstated, not understated.
* format: by default the operator is created as CSR and
         trlx_operator_autotune keeps the faster of CSR / SELL-C-32 and of
         the projection widths (config.autotune has its measurements; the
         other format is timed as a variant).
* solve: time to solution, the metric's own measure: one solve to
         residual <= 1e-8 with an FP64 basis and one with an FP32 basis plus
         FP64 refinement: seconds, matvecs, true residuals (--no-solve skips).
* batched: the 4096-problem batched configuration, one persistent launch
         per solve, timed with CUDA events (--no-batched skips).

Inputs (basis >= 4 GB, CSR 1.4 GB) exceed the 126 MB L2 between steps.
Multi-GPU (N > 1): every rank solves its own replica (different potential
seed), no collective in the data path ("replicas only", weak scaling).
"""
import os

os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")

import argparse
import ctypes as C
import json
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "anderson256": dict(kind="anderson", L=256, W=4.0, ned=32, maxlan=128, tol=1e-8),
    "batched4096": dict(kind="batched", count=4096, ned=8, maxlan=32, tol=1e-8),
    "batched512": dict(kind="batched", count=512, ned=8, maxlan=32, tol=1e-8),
    "anderson128": dict(kind="anderson", L=128, W=4.0, ned=32, maxlan=128, tol=1e-8),
    "laplace128": dict(kind="laplace", L=128, ned=10, maxlan=64, tol=1.4901e-8),
    "peierls2048": dict(kind="peierls", L=2048, phi=1.0 / 64.0, W=2.0, ned=16, maxlan=96, tol=1e-8),
    "peierls1024": dict(kind="peierls", L=1024, phi=1.0 / 64.0, W=2.0, ned=16, maxlan=96, tol=1e-8),
    "wells256": dict(kind="wells", L=256, ned=16, maxlan=48, tol=1e-8, problems=16),
}


def _form_index(tune, key):
    """A tuned projection form as its trlx value (0: the default form)."""
    if not tune:
        return 0
    from nutrlan_b200._lib import TrlxTuneResult
    return 1 + TrlxTuneResult.FORMS.index(tune[key])


def _forced_forms(args, lib, op, forms, config):
    """--project-form: set one projection form for both basis widths on the
    operator (profiling and A/B runs); returns the (64-bit, 32-bit) forms."""
    from nutrlan_b200._lib import TrlxTuneResult
    if args.project_form == "auto":
        return forms
    f = 1 + TrlxTuneResult.FORMS.index(args.project_form)
    lib.trlx_operator_set_project_form(op.handle, f)
    lib.trlx_operator_set_project_form32(op.handle, f)
    config["project_form_forced"] = args.project_form
    return f, f


def build_operator(w, seed):
    from nutrlan_b200 import operators as ops
    if w["kind"] == "anderson":
        return ops.anderson_3d(w["L"], W=w["W"], seed=seed)
    return ops.laplacian_2d(w["L"])


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference_sample(A, w, x0, sample_steps):
    """Reference trlan (CPU) on the first `sample_steps` Lanczos steps."""
    from oracle import ref
    ref.build()
    r = ref.trlan_csr(A, ned=w["ned"], maxlan=sample_steps, lohi=-1, tol=w["tol"], restart=1,
                      maxmv=sample_steps, start=x0, mev=w["ned"] + 1)
    return r["info"].matvec, r["seconds"]


BATCHED_SAMPLE = ("reference trlan on {n} problems of the batch spread over the size range, "
                  "solved one after another (OpenBLAS + OpenMP CSR callback)")


def batched_problems(w, rank):
    """Sizes (L uniform in [48, 256]) and uniform[0, 2] diagonals of the
    batched configuration's problems."""
    from nutrlan_b200 import operators as ops
    Ls = ops.batched_sizes(w["count"], seed=777 + rank)
    diags = [2.0 * ops.uniform01(1000 + 7919 * rank + k, np.arange(int(L) * int(L), dtype=np.uint64))
             for k, L in enumerate(Ls)]
    return Ls, diags


def batched_reference_sample(w, Ls, diags, rank, nprob=6):
    """The reference library on `nprob` problems of the batch spread over
    the size range, same operators, start vectors and parameters as the
    batched solver; returns (problems, seconds)."""
    from nutrlan_b200 import operators as ops
    from nutrlan_b200.batched import seeded_start
    from oracle import ref
    ref.build()
    t_cpu, n_cpu = 0.0, 0
    for k in np.linspace(0, len(Ls) - 1, nprob).astype(int):
        A = ops.laplacian_2d(int(Ls[k]), diag=diags[k])
        x0 = seeded_start(4242 + rank, int(k), A.n)
        o = ref.trlan_csr(A, ned=w["ned"], maxlan=w["maxlan"], tol=w["tol"], restart=1,
                          maxmv=100000, start=x0)
        t_cpu += o["seconds"]
        n_cpu += 1
    return n_cpu, t_cpu


def run_batched_reference(args, w, world, rank):
    """Reference arm of the batched configuration: problems/s of the
    reference library on a bounded sample of the batch (rank 0 only)."""
    if rank != 0:
        return
    count = w["count"]
    Ls, diags = batched_problems(w, rank)
    times, probs = [], []
    for s in range(args.warmup + args.steps):
        n_cpu, t_cpu = batched_reference_sample(w, Ls, diags, rank)
        if s >= args.warmup:
            times.append(t_cpu)
            probs.append(n_cpu)
    val = sum(probs) / sum(times)
    sample = BATCHED_SAMPLE.format(n=probs[0])
    print(json.dumps({"impl": "reference",
                      "metric": f"batched thick-restart Lanczos, {count} problems (smallest {w['ned']} each)",
                      "value": val, "unit": "problems/s", "n_gpus": world, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic (seeded)",
                      "config": {"workload": f"batched{count}: L~U[48,256], 5-pt Laplacian + U[0,2] diag, "
                                             f"ned={w['ned']}, maxlan={w['maxlan']}, tol={w['tol']}; sample per "
                                             f"step: {probs[0]} problems of the batch spread over the size range, "
                                             "solved one after another by reference trlan"},
                      "cpu_baseline": {"value": val, "unit": "problems/s", "cores": os.cpu_count(),
                                       "kind": "reference", "sample": sample},
                      "e2e": {"value": val, "unit": "problems/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def batched_alg_bytes(info, Ls, w):
    """Algorithmic bytes of one batched solve: per matvec the stencil's x, y
    and diagonal (3 vectors), a Gram-Schmidt pass reading the basis twice at
    the cycle's average size (3/4 maxlan columns) and the recurrence
    vectors (4); per restart the Ritz recombination, reading jml <= maxlan
    columns and writing kept >= ned.  Returns (total, steps only)."""
    sizes = Ls.astype(np.int64) ** 2
    steps = float(np.sum(info[:, 2] * sizes * 8 * (3 + 2 * 0.75 * w["maxlan"] + 4)))
    restarts = float(np.sum(info[:, 3] * sizes * 8 * (w["maxlan"] + w["ned"])))
    return steps + restarts, steps


def batched_record(w, rank, solves=2):
    """The batched configuration measured inside the default line: one
    autotuned persistent launch per solve of all `count` problems, timed with
    CUDA events over `solves` solves after one warm-up solve."""
    import torch
    from nutrlan_b200.batched import Batch
    Ls, diags = batched_problems(w, rank)
    b = Batch.stencil5(Ls, diags)
    try:
        kw = dict(ned=w["ned"], maxlan=w["maxlan"], tol=w["tol"], restart=1, maxmv=100000, seed=4242 + rank)
        t_tune = time.perf_counter()
        cfg = b.autotune(**kw)
        t_tune = time.perf_counter() - t_tune
        b.solve(**kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(solves):
            r = b.solve(**kw)
        e1.record()
        torch.cuda.synchronize()
        dt = e0.elapsed_time(e1) * 1e-3 / solves
        alg, alg_steps = batched_alg_bytes(r.info, Ls, w)
        peak, kind = read_peaks()
        return {"workload": f"batched{w['count']}: L~U[48,256], 5-pt Laplacian + U[0,2] diag, ned={w['ned']}, "
                            f"maxlan={w['maxlan']}, tol={w['tol']}, one persistent launch per solve",
                "problems_per_s": w["count"] / dt, "ms_per_solve": 1e3 * dt, "solves_timed": solves,
                "solved": int(np.sum((r.info[:, 0] == 0) & (r.info[:, 1] >= w["ned"]))),
                "matvecs_total": int(np.sum(r.info[:, 2])), "restarts_total": int(np.sum(r.info[:, 3])),
                "alg_GBps": alg / dt / 1e9, "hbm_frac": alg / dt / 1e9 / peak, "peak_source": kind,
                "alg_GBps_steps_only": alg_steps / dt / 1e9,
                "alg_bytes": "per matvec (3 + 2 * 0.75 maxlan + 4) * 8 n, per restart (maxlan + ned) * 8 n",
                "autotune": {"bucket_threads": list(cfg.bucket_threads), "bucket_format": list(cfg.bucket_format),
                             "cta_threads": cfg.cta_threads, "seconds": t_tune}}
    finally:
        b.close()


def run_batched(args, w, world, rank, local, pg):
    """Batched configuration: `count` problems, L x L Dirichlet Laplacian +
    uniform[0, 2] diagonal, L uniform in [48, 256]; 8 smallest each,
    maxlan 32, tol 1e-8; one persistent launch per step.  Metric:
    problems solved per second."""
    import torch
    from nutrlan_b200.batched import Batch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    count = w["count"]
    Ls, diags = batched_problems(w, rank)
    b = Batch.stencil5(Ls, diags)
    kw = dict(ned=w["ned"], maxlan=w["maxlan"], tol=w["tol"], restart=1, maxmv=100000, seed=4242 + rank)
    t_tune = time.perf_counter()
    cfg = b.autotune(**kw)
    t_tune = time.perf_counter() - t_tune
    for _ in range(args.warmup):
        b.solve(**kw)
    torch.cuda.synchronize()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        r = b.solve(**kw)
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    dt = reduce_max(pg, e0.elapsed_time(e1) * 1e-3, dev)
    solved = int(np.sum((r.info[:, 0] == 0) & (r.info[:, 1] >= w["ned"])))
    n_total = int(np.sum(Ls.astype(np.int64) ** 2))
    matvecs = int(np.sum(r.info[:, 2]))
    alg_bytes, _ = batched_alg_bytes(r.info, Ls, w)   # steps + restart recombinations
    value = count * world * args.steps / dt
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_cpu, t_cpu = batched_reference_sample(w, Ls, diags, rank)
        cpu = {"value": n_cpu / t_cpu, "unit": "problems/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": BATCHED_SAMPLE.format(n=n_cpu)}
    if rank == 0:
        line = {"metric": f"batched thick-restart Lanczos, {count} problems (smallest {w['ned']} each)",
                "value": value, "unit": "problems/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": {"workload": f"batched{count}: L~U[48,256], 5-pt Laplacian + U[0,2] diag, "
                                       f"ned={w['ned']}, maxlan={w['maxlan']}, tol={w['tol']}",
                           "rows_total": n_total, "one_launch_per_step": True},
                "solved": solved, "matvecs_total": matvecs,
                "alg_GBps": alg_bytes / (dt / args.steps) / 1e9,
                "autotune": {"bucket_threads": list(cfg.bucket_threads), "bucket_format": list(cfg.bucket_format),
                             "cta_threads": cfg.cta_threads, "seconds": t_tune},
                "cpu_baseline": cpu, "clocks": clocks}
        print(json.dumps(line), flush=True)
    b.close()


def run_complex(args, w, world, rank, local, pg):
    """Complex Hermitian configuration (ztrlan): 2D tight binding on an
    L x L periodic lattice with Peierls phases for flux phi per plaquette,
    diagonal disorder uniform[-W/2, W/2]; smallest 16, maxlan 96, tol 1e-8.
    A step is one ztrlan() call bounded to one thick-restart cycle (96
    Lanczos steps + Ritz vectors); metric: Lanczos steps/s with a c128 basis
    (c64 basis as a variant)."""
    from nutrlan_b200 import operators as ops
    L, ned, maxlan, tol = w["L"], w["ned"], w["maxlan"], w["tol"]
    seed = 4242 + rank
    metric = f"Lanczos steps/s (SpMV + full CGS reorth), peierls{L} complex Hermitian, smallest {ned}"
    config = {"workload": f"peierls{L}: n={L * L}, flux 1/{int(round(1 / w['phi']))}, disorder "
                          f"U[-{w['W'] / 2:g},{w['W'] / 2:g}], ned={ned}, maxlan={maxlan}, tol={tol}, "
                          f"complex {{fmt}}, basis c128, one thick-restart cycle/step",
              "global_batch": world, "parallelism": f"replicas x{world}"}
    A = ops.peierls_2d(L, phi=w["phi"], W=w["W"], seed=seed)
    n = A.n
    config["l2"] = (f"inputs larger than L2 (basis {maxlan * n * 16 / 1e9:.1f} GB, "
                    f"CSR {(A.nnz * 20 + 8 * n) / 1e6:.0f} MB)")
    x0 = ops.start_vector(n) + 1j * ops.start_vector(n, seed=99)
    cpu_sample = args.cpu_sample

    def reference_sample():
        from oracle import ref
        ref.build()
        r = ref.trlan_csr(A, ned=ned, maxlan=cpu_sample, lohi=-1, tol=tol, restart=1, maxmv=cpu_sample,
                          start=x0, mev=ned + 1)
        return r["info"].matvec, r["seconds"]

    cpu_desc = (f"reference ztrlan, first {cpu_sample} Lanczos steps (maxlan=maxmv={cpu_sample}) of the "
                "same solve, OpenBLAS + OpenMP complex CSR callback")
    if args.impl == "reference":
        if rank != 0:
            return
        times, mvs = [], []
        for s_ in range(args.warmup + args.steps):
            mv, dt = reference_sample()
            if s_ >= args.warmup:
                times.append(dt)
                mvs.append(mv)
        val = sum(mvs) / sum(times)
        ref_config = dict(config, workload=config["workload"].replace(
            "complex {fmt}, basis c128, one thick-restart cycle/step",
            f"complex CSR callback (OpenMP) + OpenBLAS; sample per step: the first {cpu_sample} Lanczos steps "
            f"of the same solve (maxlan=maxmv={cpu_sample}, reference ztrlan)"))
        print(json.dumps({"impl": "reference", "metric": metric, "value": val, "unit": "steps/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                          "config": ref_config,
                          "cpu_baseline": {"value": val, "unit": "steps/s", "cores": os.cpu_count(),
                                           "kind": "reference", "sample": cpu_desc},
                          "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from nutrlan_b200 import load, TrlInfo, TrlxOptions, TrlxStats, DeviceOperator
    lib = load()
    mev = ned + 1
    op = DeviceOperator(A, fmt="auto", maxlan=maxlan)        # tunes the format and projection forms
    tuned_form, tuned_form32 = _forced_forms(
        args, lib, op, (_form_index(op.tune, "project_form"), _form_index(op.tune, "project_form32")), config)
    config["workload"] = config["workload"].replace("{fmt}", "SELL-C-32" if op.fmt == "zsell" else "CSR")
    config["autotune"] = op.tune
    evec = torch.zeros((mev, n), dtype=torch.complex128, device=dev)
    x0_dev = torch.as_tensor(x0, device=dev)
    eval_ = np.zeros(mev)
    misc = np.zeros(mev, dtype=np.complex128)
    stats = TrlxStats()

    def options(bits, profile):
        o = TrlxOptions()
        lib.trlx_default_options(C.byref(o))
        o.basis_bits = bits
        o.profile = profile
        return o

    def call(info, opts, maxmv, evp, opptr, applier):
        lib.trl_init_info(C.byref(info), n, maxlan, -1, ned, tol, 1, maxmv, None)
        info.mvparam = opptr
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        lib.trlx_ztrlan(applier, C.byref(info), n, mev, eval_.ctypes.data, evp, n, misc.ctypes.data, mev,
                        None, 0, C.byref(opts))
        if info.stat != 0:
            raise RuntimeError(f"ztrlan stat {info.stat}")
        return info.matvec

    def timed(bits, profile, oper=None):
        oper = oper or op
        opts = options(bits, profile)
        info = TrlInfo()
        for _ in range(args.warmup):
            evec[0].copy_(x0_dev)
            call(info, opts, maxlan, evec.data_ptr(), oper.handle.value, oper.applier)
        torch.cuda.synchronize()
        barrier(pg)
        sampler = ClockSampler(local) if profile else None
        if sampler:
            sampler.start()
        kt, kb, kc = np.zeros(8), np.zeros(8), np.zeros(8)
        launches, mv = 0, 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            evec[0].copy_(x0_dev)
            mv += call(info, opts, maxlan, evec.data_ptr(), oper.handle.value, oper.applier)
            lib.trlx_get_last_stats(C.byref(stats))
            kt += np.array(stats.kernel_seconds[:])
            kb += np.array(stats.kernel_bytes[:])
            kc += np.array(stats.kernel_count[:])
            launches += stats.kernel_launches
        e1.record()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        dt = reduce_max(pg, e0.elapsed_time(e1) * 1e-3, dev)
        return reduce_max(pg, mv, dev) * world / dt, dt, kt, kb, kc, launches, clocks

    value, dt, kt, kb, kc, launches, clocks = timed(64, 1)
    names = ["spmv", "project", "update", "normalize", "ritz", "dot", "other", "x"]
    dom = int(np.argmax(kt))
    peak, peak_kind = read_peaks()
    achieved = kb[dom] / kt[dom] / 1e9 if kt[dom] > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                "alg_bytes_per_launch": kb[dom] / max(kc[dom], 1), "launches": int(kc[dom]),
                "per_kernel": {names[i]: {"seconds": kt[i], "GB/s": (kb[i] / kt[i] / 1e9) if kt[i] else 0,
                                          "launches": int(kc[i])} for i in range(7) if kc[i]},
                "spmv_plus_reorth_GBps": float((kb[0] + kb[1] + kb[2]) / max(kt[0] + kt[1] + kt[2], 1e-30) / 1e9)}
    variants = {}
    if not args.no_variants:
        variants[f"{op.fmt}_c64"] = timed(32, 0)[0]
        # The format the autotuner did not keep, with the same projection forms.
        other = "zcsr" if op.fmt == "zsell" else "zsell"
        with DeviceOperator(A, fmt=other) as oop:
            lib.trlx_operator_set_project_form(oop.handle, tuned_form)
            lib.trlx_operator_set_project_form32(oop.handle, tuned_form32)
            variants[f"{other}_c128"] = timed(64, 0, oop)[0]

    e2e = None
    if not args.no_e2e:
        opts = options(64, 0)

        def host_buffers(pinned):
            def like(a):
                a = np.ascontiguousarray(a)
                if not pinned:
                    return a
                h = torch.empty(a.shape, dtype=torch.from_numpy(a[:1]).dtype, pin_memory=True).numpy()
                h[...] = a
                return h
            hev = torch.zeros((mev, n), dtype=torch.complex128, pin_memory=pinned).numpy()
            return like(A.row_ptr), like(A.col), like(A.val), hev

        def e2e_call(rp, ci, va, hev):
            h = C.c_void_p()
            if op.fmt == "zsell":
                rc = lib.trlx_zsell_create(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 1, 0, C.byref(h))
            else:
                rc = lib.trlx_zcsr_create(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 0, C.byref(h))
            if rc != 0:
                raise RuntimeError(f"complex operator creation from host arrays failed ({rc})")
            lib.trlx_operator_set_project_form(h, tuned_form)
            lib.trlx_operator_set_project_form32(h, tuned_form32)
            hev[0] = x0
            mv = call(TrlInfo(), opts, maxlan, hev.ctypes.data, h.value, op.applier)
            lib.trlx_operator_destroy(h)
            return mv

        def e2e_rate(pinned, steps):
            bufs = host_buffers(pinned)
            e2e_call(*bufs)
            barrier(pg)
            t0 = time.perf_counter()
            mv = sum(e2e_call(*bufs) for _ in range(steps))
            e_wall = reduce_max(pg, time.perf_counter() - t0, dev)
            return reduce_max(pg, mv, dev) * world / e_wall

        csr_bytes = A.row_ptr.nbytes + A.col.nbytes + A.val.nbytes
        e2e = {"value": e2e_rate(True, args.steps), "unit": "steps/s",
               "h2d_bytes_per_step": int(csr_bytes + 16 * n),
               "d2h_bytes_per_step": int(16 * n * mev + 8 * mev),
               "host_buffers": "page-locked (CSR arrays, start vector, evec)"}
        e2e["pageable"] = {"value": e2e_rate(False, max(3, min(args.steps, 5))), "unit": "steps/s",
                           "host_buffers": "pageable numpy arrays (staged copies)"}

    solve_rec = None
    if not args.no_solve and rank == 0 and world == 1:
        from nutrlan_b200 import residual_norms
        solve_rec = {}
        for bits in (64, 32):
            info = TrlInfo()
            evec[0].copy_(x0_dev)
            torch.cuda.synchronize()
            ts = time.perf_counter()
            call(info, options(bits, 0), args.solve_maxmv, evec.data_ptr(), op.handle.value, op.applier)
            torch.cuda.synchronize()
            ts = time.perf_counter() - ts
            k = max(info.nec, 1)
            res = residual_norms(op, eval_[:k], evec[:k])
            solve_rec[f"c{2 * bits}"] = {"seconds": ts, "matvecs": info.matvec, "restarts": info.nloop,
                                         "nec": info.nec, "max_true_residual": float(res.max()),
                                         "anrm": info.anrm, "evals": [float(v) for v in eval_[:k]]}
        a_, b_ = np.array(solve_rec["c128"]["evals"]), np.array(solve_rec["c64"]["evals"])
        kk = min(len(a_), len(b_))
        solve_rec["c64_vs_c128_max_rel_eval_diff"] = float(np.max(np.abs(np.sort(a_[:kk]) - np.sort(b_[:kk]))
                                                                  / np.abs(np.sort(a_[:kk]))))
    op.close()
    del evec
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            mv, dtc = reference_sample()
            cpu = {"value": mv / dtc, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": cpu_desc, "seconds": dtc}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    if rank == 0:
        print(json.dumps({"metric": metric, "value": value, "unit": "steps/s", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                          "data": "synthetic (seeded disorder and start vector)", "config": config,
                          "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                          "clocks": clocks, "variants": variants, "solve": solve_rec}), flush=True)


def learned_seed_ab(problems, seed0=10 ** 6, log=None):
    """Plain vs learned-seed solves on held-out Gaussian-well operators
    (256 x 256, smallest 16, maxlan 48, tol 1e-8) with the packaged
    weights; per-problem wall time includes the network forward pass and
    the start-vector construction."""
    from nutrlan_b200.seednet import SeedNet
    from nutrlan_b200.seed_train import evaluate, summarize
    net = SeedNet.pretrained()
    try:
        recs = evaluate(net, range(seed0, seed0 + problems), 256, maxlan=48, log=log or (lambda *a: None),
                        subspace=True)
    finally:
        net.close()
    out = summarize(recs)
    out["all_converged"] = bool(all(r["plain_nec"] >= 16 and r["sum_nec"] >= 16 and r["rr_nec"] >= 16
                                    for r in recs))
    out["max_true_residual_over_tol"] = float(max(max(r["sum_max_true_res"], r["rr_max_true_res"]) / r["tol_abs"]
                                                  for r in recs))
    out["max_eval_rel_diff_vs_plain"] = float(max(max(r["sum_eval_rel_diff"], r["rr_eval_rel_diff"])
                                                  for r in recs))
    out["subspace"] = {
        "dense": "restarted dense Rayleigh-Ritz over span(seed Ritz vectors, Krylov block), exact residuals",
        "first": "one dense cycle from the seed, then trlan from the sum of its Ritz vectors",
        "dense_all_converged": bool(all(r["dense_converged"] for r in recs)),
        "dense_max_eval_rel_diff_vs_plain": float(max(r["dense_eval_rel_diff"] for r in recs)),
        "first_all_converged": bool(all(r["first_nec"] >= 16 for r in recs))}
    return out


def wells_reference_sample(seed0, count=2):
    """The reference library's plain solves of `count` held-out well
    operators (same operators, start vector and parameters as the plain arm
    of the A/B test); returns (solves, seconds, matvecs)."""
    from oracle import ref
    from nutrlan_b200 import operators as ops
    ref.build()
    t_cpu, n_cpu, mv = 0.0, 0, 0
    for s_ in range(seed0, seed0 + count):
        A, _ = ops.wells_2d(256, seed=s_)
        o = ref.trlan_csr(A, ned=16, maxlan=48, tol=1e-8, restart=1, maxmv=100000,
                          start=ops.start_vector(A.n))
        t_cpu += o["seconds"]
        n_cpu += 1
        mv += o["info"].matvec
    return n_cpu, t_cpu, mv


WELLS_METRIC = "learned-seed solves/s to residual <= 1e-8 (Gaussian wells 256x256, smallest 16)"
WELLS_WORKLOAD = ("wells256: n=65536, 8 Gaussian wells, ned=16, maxlan=48, tol=1e-8, "
                  "CSR, seed = sum of network outputs (guess=1)")


def run_wells(args, w, world, rank, local, pg):
    """Learned-seed configuration: time to residual <= 1e-8 on held-out
    Gaussian-well operators, seeded by the packaged network (start vector =
    sum of its normalised outputs) against the plain solve.  Metric: seeded
    solves per second (whole job); the plain rate and matvec counts beside it.
    The reference arm times the reference's plain solves of the same held-out
    operators (the learned seed has no counterpart there), rank 0 only."""
    seed0 = 10 ** 6 + 1000 * rank
    if args.impl == "reference":
        if rank != 0:
            return
        times, solves, mvs = [], [], []
        for s in range(args.warmup + args.steps):
            n_cpu, t_cpu, mv = wells_reference_sample(seed0)
            if s >= args.warmup:
                times.append(t_cpu)
                solves.append(n_cpu)
                mvs.append(mv)
        val = sum(solves) / sum(times)
        sample = (f"reference trlan, plain solves of {solves[0]} of the held-out operators per step "
                  f"({sum(mvs) / sum(solves):.0f} matvecs each), OpenBLAS + OpenMP CSR callback")
        print(json.dumps({"impl": "reference", "metric": WELLS_METRIC, "value": val, "unit": "solves/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic (seeded well potentials, held-out seeds)",
                          "config": {"workload": WELLS_WORKLOAD, "parallelism": f"replicas x{world}",
                                     "reference": "plain solve (no learned seed), start vector uniform[-1,1]"},
                          "cpu_baseline": {"value": val, "unit": "solves/s", "cores": os.cpu_count(),
                                           "kind": "reference", "sample": sample},
                          "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_prob = w["problems"]
    learned_seed_ab(2, seed0=seed0 + 500)  # warm-up (workspace, library, network)
    for _ in range(max(args.warmup - 1, 0)):
        learned_seed_ab(1, seed0=seed0 + 600)
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    t0 = time.perf_counter()
    ab = learned_seed_ab(n_prob, seed0=seed0)
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    seeded_s = reduce_max(pg, ab["sum_s"], dev)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        n_cpu, t_cpu, mv = wells_reference_sample(seed0)
        cpu = {"value": n_cpu / t_cpu, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": f"reference trlan, plain solves of {n_cpu} of the held-out operators "
                         f"({mv / n_cpu:.0f} matvecs each), OpenBLAS + OpenMP CSR callback"}
    if rank == 0:
        print(json.dumps({
            "metric": WELLS_METRIC,
            "value": world / seeded_s, "unit": "solves/s", "n_gpus": world, "steps": n_prob,
            "warmup": args.warmup, "ms_per_step": 1e3 * seeded_s, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 solver, bf16 network",
            "data": "synthetic (seeded well potentials, held-out seeds)",
            "config": {"workload": WELLS_WORKLOAD,
                       "problems_per_rank": n_prob, "parallelism": f"replicas x{world}",
                       "l2": "operator and basis fit in L2 (latency-bound regime)"},
            "plain_solves_per_s": world / reduce_max(pg, ab["plain_s"], dev),
            "learned_seed": ab, "cpu_baseline": cpu, "clocks": clocks, "host_wall_s": wall}), flush=True)


def run_dist(args, w, world, rank, local, pg):
    """One Anderson/Laplace solve split into block rows over the ranks (the
    reference's parallel model): NCCL sums and halo exchanges between the
    GPUs.  Strong scaling: the global problem is the named workload; value =
    Lanczos steps of the one global solve per second (max over ranks)."""
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from nutrlan_b200 import operators as ops
    from nutrlan_b200.dist import Comm, DistOperator, row_blocks, local_rows, solve as dsolve
    A = build_operator(w, 2024)
    n = A.n
    ned, maxlan, tol = w["ned"], w["maxlan"], w["tol"]
    mev = ned + 1
    row0, nloc = row_blocks(n, world)[rank]
    rp, ci, va = local_rows(A, row0, nloc)
    x0 = ops.start_vector(n)[row0:row0 + nloc]
    comm = Comm.from_process_group() if pg is not None else Comm.nccl(1, 0, Comm.nccl_unique_id())
    dist_fmt = "sell" if args.format == "auto" else args.format   # block rows: no autotuner
    op = DistOperator(comm, rp, ci, va, fmt=dist_fmt)
    evec = torch.zeros((mev, nloc), dtype=torch.float64, device=dev)

    def one_call(profile=True):
        r = dsolve(comm, op, ned, maxlan, tol=tol, maxmv=maxlan, start=x0, evec=evec,
                   basis_bits=args.basis_bits, profile=profile)
        if r.stat != 0:
            raise RuntimeError(f"trlan stat {r.stat}")
        return r

    for _ in range(args.warmup):
        one_call()
    torch.cuda.synchronize()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    kt, kb, kc = np.zeros(8), np.zeros(8), np.zeros(8)
    launches = mv = 0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        r = one_call()
        st = r.stats
        kt += np.array(st.kernel_seconds[:])
        kb += np.array(st.kernel_bytes[:])
        kc += np.array(st.kernel_count[:])
        launches += st.kernel_launches
        mv += r.info.matvec
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    elapsed = reduce_max(pg, e0.elapsed_time(e1) * 1e-3, dev)
    value = mv / elapsed
    names = ["spmv", "project", "update", "normalize", "ritz", "dot", "other", "x"]
    dom = int(np.argmax(kt))
    peak, peak_kind = read_peaks()
    achieved = kb[dom] / kt[dom] / 1e9 if kt[dom] > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None, "peak_source": peak_kind,
                "alg_bytes_per_launch": kb[dom] / max(kc[dom], 1), "launches": int(kc[dom]),
                "note": "rank 0's kernels on its own rows"}
    e2e = None
    if not args.no_e2e:
        hev = np.zeros((mev, nloc))

        def e2e_call():
            with DistOperator(comm, rp, ci, va, fmt=dist_fmt) as hop:
                r = dsolve(comm, hop, ned, maxlan, tol=tol, maxmv=maxlan, start=x0, basis_bits=args.basis_bits,
                           evec=hev)
                return r.info.matvec

        e2e_call()
        barrier(pg)
        t0 = time.perf_counter()
        emv = sum(e2e_call() for _ in range(args.steps))
        e_wall = reduce_max(pg, time.perf_counter() - t0, dev)
        e2e = {"value": emv / e_wall, "unit": "steps/s",
               "h2d_bytes_per_step": int(rp.nbytes + ci.nbytes + va.nbytes + 8 * nloc),
               "d2h_bytes_per_step": int(8 * nloc * mev + 8 * mev)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cmv, cdt = run_reference_sample(A, w, ops.start_vector(n), args.cpu_sample)
        cpu = {"value": cmv / cdt, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
               "sample": f"reference trlan, first {args.cpu_sample} Lanczos steps of the same solve"}
    op.close()
    comm.close()
    if rank == 0:
        print(json.dumps({
            "metric": f"Lanczos steps/s (SpMV + full CGS reorth), {args.workload}, smallest {ned}",
            "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if args.basis_bits == 64 else "f32 basis / f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{args.workload}: n={n}, ned={ned}, maxlan={maxlan}, tol={tol}, "
                                   f"{dist_fmt.upper()} block rows, basis fp{args.basis_bits}, "
                                   "one thick-restart cycle/step",
                       "parallelism": f"block rows x{world} (NCCL sums + halo exchange)",
                       "l2": "inputs larger than L2"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks}), flush=True)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if args.impl == "b200" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value, device):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="anderson256")
    ap.add_argument("--basis-bits", type=int, choices=[64, 32], default=64)
    ap.add_argument("--format", choices=["auto", "csr", "sell"], default="auto",
                    help="operator format; auto: trlx_operator_autotune picks CSR or SELL-C-32 "
                         "and the projection width by measurement")
    ap.add_argument("--project-form", default="auto",
                    choices=["auto", "cpw8", "cpw12", "cpw16", "cpw16_shared_ptrs", "cpw8_staged"],
                    help="projection kernel form for both basis widths (auto: the autotuner's choice)")
    ap.add_argument("--cpu-sample", type=int, default=32,
                    help="Lanczos steps in the bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the secondary timings (other format, 32-bit basis)")
    ap.add_argument("--no-solve", action="store_true",
                    help="skip the solves to convergence (time to solution, FP64 and FP32 basis)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-solver record of the default line")
    ap.add_argument("--solve-maxmv", type=int, default=20000)
    ap.add_argument("--no-learned-seed", action="store_true",
                    help="skip the learned-seed A/B record of the default line")
    ap.add_argument("--dist", action="store_true",
                    help="one solve split into block rows over the ranks (NCCL), strong scaling; "
                         "default for --gpus N: independent replicas")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    world, rank, local, pg = dist_setup(args)
    if w["kind"] == "wells":
        run_wells(args, w, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if w["kind"] == "peierls":
        run_complex(args, w, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.dist and args.impl == "b200" and w["kind"] in ("anderson", "laplace"):
        run_dist(args, w, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if w["kind"] == "batched":
        if args.impl == "reference":
            run_batched_reference(args, w, world, rank)
            if pg is not None:
                pg.destroy_process_group()
            return
        run_batched(args, w, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    seed = 2024 + rank
    metric = f"Lanczos steps/s (SpMV + full CGS reorth), {args.workload}, smallest {w['ned']}"
    nrows = w['L'] ** (3 if w['kind'] == 'anderson' else 2)

    def workload(fmt, what):
        return (f"{args.workload}: n={nrows}, ned={w['ned']}, maxlan={w['maxlan']}, tol={w['tol']}, "
                f"{fmt}, {what}")

    config = {"workload": workload("{fmt}", f"basis fp{args.basis_bits}, one thick-restart cycle/step"),
              "global_batch": world, "parallelism": f"replicas x{world}",
              "l2": ("inputs larger than L2 (basis >= 2 GB)" if w["kind"] == "anderson" else
                     "working set L2-resident (n = 16384: latency-bound, not an HBM measurement)")}

    if args.impl == "reference":
        # The reference's per-step sample is what this line says it is: the
        # first cpu_sample Lanczos steps of the same solve (a 128-step cycle
        # takes about 40 s on the host cores, too long for --steps K).
        config["workload"] = workload(
            "CSR callback (OpenMP) + OpenBLAS",
            f"basis fp64; sample per step: the first {args.cpu_sample} Lanczos steps of the same solve "
            f"(maxlan=maxmv={args.cpu_sample}, reference trlan)")
        if rank != 0:
            return
        A = build_operator(w, seed)
        from nutrlan_b200 import operators as ops
        x0 = ops.start_vector(A.n)
        times, mvs = [], []
        for s in range(args.warmup + args.steps):
            mv, dt = run_reference_sample(A, w, x0, args.cpu_sample)
            if s >= args.warmup:
                times.append(dt)
                mvs.append(mv)
        val = sum(mvs) / sum(times)
        cores = os.cpu_count()
        line = {"impl": "reference", "metric": metric, "value": val, "unit": "steps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": val, "unit": "steps/s", "cores": cores, "kind": "reference",
                                 "sample": f"reference trlan, first {args.cpu_sample} Lanczos steps "
                                           f"(maxlan=maxmv={args.cpu_sample}) of the same solve, "
                                           "OpenBLAS + OpenMP CSR callback"},
                "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from nutrlan_b200 import load, TrlInfo, TrlxOptions, TrlxStats, DeviceOperator
    from nutrlan_b200 import operators as ops
    lib = load()

    A = build_operator(w, seed)
    n = A.n
    x0 = ops.start_vector(n)
    ned, maxlan, tol = w["ned"], w["maxlan"], w["tol"]
    mev = ned + 1
    steps_per_call = maxlan

    opts = TrlxOptions()
    lib.trlx_default_options(C.byref(opts))
    opts.basis_bits = args.basis_bits
    opts.profile = 1
    stats = TrlxStats()

    # ---- device-resident arm -------------------------------------------------
    op = DeviceOperator(A, fmt=args.format, maxlan=maxlan)
    fmt_used = op.fmt
    tuned_form, tuned_form32 = _forced_forms(
        args, lib, op, (_form_index(op.tune, "project_form"), _form_index(op.tune, "project_form32")), config)
    config["workload"] = config["workload"].replace("{fmt}", fmt_used.upper())
    if op.tune is not None:
        config["format_choice"] = "autotuned (trlx_operator_autotune)"
        config["autotune"] = op.tune
    evec = torch.zeros((mev, n), dtype=torch.float64, device=dev)
    x0_dev = torch.as_tensor(x0, device=dev)
    eval_ = np.zeros(mev)
    wrk = np.zeros(mev)

    def one_call(info):
        lib.trl_init_info(C.byref(info), n, maxlan, -1, ned, tol, 1, steps_per_call, None)
        info.mvparam = op.handle.value
        lib.trl_set_iguess(C.byref(info), 0, 1, 0, None)
        evec[0].copy_(x0_dev)
        lib.trlx_trlan(op.applier, None, C.byref(info), n, mev, eval_.ctypes.data, evec.data_ptr(), n,
                       mev, wrk.ctypes.data, C.byref(opts))
        if info.stat != 0:
            raise RuntimeError(f"trlan stat {info.stat}")

    info = TrlInfo()
    for _ in range(args.warmup):
        one_call(info)
    torch.cuda.synchronize()
    barrier(pg)
    sampler = ClockSampler(local)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ktot = np.zeros(8)
    kbyt = np.zeros(8)
    kcnt = np.zeros(8)
    launches = 0
    matvecs = 0
    torch.cuda.synchronize()
    ev0.record()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one_call(info)
        lib.trlx_get_last_stats(C.byref(stats))
        ktot += np.array(stats.kernel_seconds[:])
        kbyt += np.array(stats.kernel_bytes[:])
        kcnt += np.array(stats.kernel_count[:])
        launches += stats.kernel_launches
        matvecs += info.matvec
    ev1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    dev_s = ev0.elapsed_time(ev1) * 1e-3
    elapsed = reduce_max(pg, dev_s, dev)
    total_steps = reduce_max(pg, matvecs, dev) * world
    value = total_steps / elapsed
    ms_per_step = 1e3 * elapsed / args.steps

    # roofline: dominant kernel class by time
    names = ["spmv", "project", "update", "normalize", "ritz", "dot", "other", "x"]
    dom = int(np.argmax(ktot))
    peak, peak_kind = read_peaks()
    achieved = kbyt[dom] / ktot[dom] / 1e9 if ktot[dom] > 0 else 0.0
    traffic = None
    prof_path = os.path.join(ROOT, "profiles", f"traffic_{names[dom]}_{args.workload}_fp{args.basis_bits}.json")
    if os.path.exists(prof_path):
        try:
            with open(prof_path) as f:
                tr = json.load(f)
            # dram bytes per algorithmic byte, scaled to this run's average launch
            traffic = tr["dram_bytes_per_alg_byte"] * kbyt[dom] / max(kcnt[dom], 1)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": peak_kind,
                "alg_bytes_per_launch": kbyt[dom] / max(kcnt[dom], 1),
                "launches": int(kcnt[dom]),
                "per_kernel": {names[i]: {"seconds": ktot[i], "GB/s": (kbyt[i] / ktot[i] / 1e9) if ktot[i] else 0,
                                          "launches": int(kcnt[i])}
                               for i in range(7) if kcnt[i]},
                "spmv_plus_reorth_GBps": float((kbyt[0] + kbyt[1] + kbyt[2]) /
                                               max(ktot[0] + ktot[1] + ktot[2], 1e-30) / 1e9)}
    op_obj_bytes = A.row_ptr.nbytes + A.col.nbytes + A.val.nbytes

    # ---- end-to-end arm: host buffers through the C ABI ----------------------
    # The headline e2e uses page-locked host buffers (the CSR arrays, the start
    # vector and the evec that receives the results), which the library copies
    # with direct DMA; the same calls with pageable numpy buffers (what an
    # unchanged nuTRLan program passes; staged copies) are reported beside it.
    e2e = None
    if not args.no_e2e:
        handle = C.c_void_p()
        applier = op.applier

        def host_buffers(pinned):
            def like(a):
                if not pinned:
                    return np.ascontiguousarray(a)
                t = torch.empty(a.shape, dtype=torch.from_numpy(np.ascontiguousarray(a[:1])).dtype,
                                pin_memory=True)
                h = t.numpy()
                h[...] = a
                return h
            hev = torch.zeros((mev, n), dtype=torch.float64, pin_memory=pinned).numpy()
            return like(A.row_ptr), like(A.col), like(A.val), hev

        def e2e_call(rp, ci, va, hev):
            handle.value = None
            if fmt_used == "sell":
                rc = lib.trlx_sell_create(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 1, 0,
                                          C.byref(handle))
            else:
                rc = lib.trlx_csr_create(n, rp.ctypes.data, ci.ctypes.data, va.ctypes.data, 0, C.byref(handle))
            if rc != 0:
                raise RuntimeError(f"operator creation from host arrays failed ({rc})")
            lib.trlx_operator_set_project_form(handle, tuned_form)   # the tuning kept above
            lib.trlx_operator_set_project_form32(handle, tuned_form32)
            inf = TrlInfo()
            lib.trl_init_info(C.byref(inf), n, maxlan, -1, ned, tol, 1, steps_per_call, None)
            inf.mvparam = handle.value
            lib.trl_set_iguess(C.byref(inf), 0, 1, 0, None)
            hev[0] = x0
            lib.trlx_trlan(applier, None, C.byref(inf), n, mev, eval_.ctypes.data, hev.ctypes.data, n, mev,
                           wrk.ctypes.data, C.byref(opts))
            lib.trlx_operator_destroy(handle)
            return inf.matvec

        def e2e_rate(pinned, steps):
            bufs = host_buffers(pinned)
            e2e_call(*bufs)
            torch.cuda.synchronize()
            barrier(pg)
            t0 = time.perf_counter()
            mv = 0
            for _ in range(steps):
                mv += e2e_call(*bufs)
            torch.cuda.synchronize()
            e_wall = reduce_max(pg, time.perf_counter() - t0, dev)
            return reduce_max(pg, mv, dev) * world / e_wall

        e2e = {"value": e2e_rate(True, args.steps), "unit": "steps/s",
               "h2d_bytes_per_step": int(op_obj_bytes + 8 * n),
               "d2h_bytes_per_step": int(8 * n * mev + 8 * mev),
               "host_buffers": "page-locked (CSR arrays, start vector, evec)"}
        e2e["pageable"] = {"value": e2e_rate(False, max(3, min(args.steps, 5))), "unit": "steps/s",
                           "host_buffers": "pageable numpy arrays (staged copies)"}
        torch.cuda.empty_cache()

    # ---- secondary timings: the other configured format, 32-bit basis -----
    variants = {}
    if not args.no_variants:
        def time_variant(fmt, bits):
            vop = op
            if fmt != fmt_used:
                # The other format with the same projection forms.
                vop = DeviceOperator(A, fmt=fmt)
                lib.trlx_operator_set_project_form(vop.handle, tuned_form)
                lib.trlx_operator_set_project_form32(vop.handle, tuned_form32)
            vopts = TrlxOptions()
            lib.trlx_default_options(C.byref(vopts))
            vopts.basis_bits = bits
            inf = TrlInfo()

            def call():
                lib.trl_init_info(C.byref(inf), n, maxlan, -1, ned, tol, 1, steps_per_call, None)
                inf.mvparam = vop.handle.value
                lib.trl_set_iguess(C.byref(inf), 0, 1, 0, None)
                evec[0].copy_(x0_dev)
                lib.trlx_trlan(vop.applier, None, C.byref(inf), n, mev, eval_.ctypes.data, evec.data_ptr(), n,
                               mev, wrk.ctypes.data, C.byref(vopts))
                return inf.matvec

            call()
            torch.cuda.synchronize()
            barrier(pg)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            mv = sum(call() for _ in range(args.steps))
            e1.record()
            torch.cuda.synchronize()
            dt = reduce_max(pg, e0.elapsed_time(e1) * 1e-3, dev)
            if vop is not op:
                vop.close()
            return reduce_max(pg, mv, dev) * world / dt

        other = "csr" if fmt_used == "sell" else "sell"
        variants[f"{other}_fp{args.basis_bits}"] = time_variant(other, args.basis_bits)
        alt_bits = 32 if args.basis_bits == 64 else 64
        variants[f"{fmt_used}_fp{alt_bits}"] = time_variant(fmt_used, alt_bits)

    solve_rec = None
    if not args.no_solve and rank == 0 and world == 1:
        from nutrlan_b200 import residual_norms
        solve_rec = {}
        for bits in (64, 32):
            inf = TrlInfo()
            lib.trl_init_info(C.byref(inf), n, maxlan, -1, ned, tol, 1, args.solve_maxmv, None)
            inf.mvparam = op.handle.value
            lib.trl_set_iguess(C.byref(inf), 0, 1, 0, None)
            evec[0].copy_(x0_dev)
            sopts = TrlxOptions()
            lib.trlx_default_options(C.byref(sopts))
            sopts.basis_bits = bits
            torch.cuda.synchronize()
            ts = time.perf_counter()
            lib.trlx_trlan(op.applier, None, C.byref(inf), n, mev, eval_.ctypes.data, evec.data_ptr(), n, mev,
                           wrk.ctypes.data, C.byref(sopts))
            torch.cuda.synchronize()
            ts = time.perf_counter() - ts
            k = max(inf.nec, 1)
            res = residual_norms(op, eval_[:k], evec[:k])
            anrm = inf.anrm
            solve_rec[f"fp{bits}"] = {
                "seconds": ts, "matvecs": inf.matvec, "restarts": inf.nloop, "nec": inf.nec,
                "stat": inf.stat, "restart_scheme": 1,
                "max_residual_estimate": float(np.max(wrk[:k])),
                "max_true_residual": float(res.max()), "anrm": anrm,
                "max_true_residual_rel": float(res.max() / anrm),
                "eval_min": float(eval_[0]), "eval_max_converged": float(eval_[k - 1]),
                "all_residuals_within_tol_anrm": bool(inf.nec >= ned and res.max() <= tol * anrm),
                "evals": [float(v) for v in eval_[:k]]}
        if "fp64" in solve_rec and "fp32" in solve_rec:
            a, b = np.array(solve_rec["fp64"]["evals"]), np.array(solve_rec["fp32"]["evals"])
            kk = min(len(a), len(b))
            solve_rec["fp32_vs_fp64_max_rel_eval_diff"] = float(np.max(np.abs(a[:kk] - b[:kk]) / np.abs(a[:kk])))

    op.close()
    del evec
    torch.cuda.empty_cache()

    # ---- CPU baseline (rank 0, N = 1) ----------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            mv, dt = run_reference_sample(A, w, x0, args.cpu_sample)
            cpu = {"value": mv / dt, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"reference trlan, first {args.cpu_sample} Lanczos steps "
                             f"(maxlan=maxmv={args.cpu_sample}) of the same solve, OpenBLAS + OpenMP CSR callback",
                   "seconds": dt}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            batched = batched_record(WORKLOADS["batched4096"], rank)
        except Exception as e:  # noqa: BLE001
            batched = {"failed": str(e)}
    seed_ab = None
    if rank == 0 and world == 1 and not args.no_learned_seed:
        try:
            seed_ab = learned_seed_ab(8)
        except Exception as e:  # noqa: BLE001
            seed_ab = {"failed": str(e)}
    if rank == 0:
        line = {"metric": metric, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.basis_bits == 64 else "f32 basis / f64",
                "data": "synthetic (seeded Anderson potential and start vector)", "config": config,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clocks, "host_wall_s": wall, "variants": variants, "solve": solve_rec,
                "batched": batched, "learned_seed": seed_ab,
                "matvecs_per_call": int(matvecs // max(args.steps, 1))}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()

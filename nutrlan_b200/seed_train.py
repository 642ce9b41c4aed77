"""Training data, training loop and A/B evaluation of the learned seed on the
Gaussian-well family (-Laplacian + V on an L x L Dirichlet grid, V a sum of
8 wells with centres uniform in the domain, widths uniform[4, 24] cells and
depths uniform[5, 50]).

* ``generate``: potentials for consecutive seeds, their lowest ``ned``
  eigenvectors computed by the batched persistent solver (the plain
  algorithm) and kept on the device (V float32, U bfloat16).
* ``train``: Adam on the subspace loss through the library's own BF16
  forward/backward kernels.
* ``evaluate``: for held-out seeds, the plain solve (seeded uniform start)
  against the learned-seed solves (network forward and the start vector
  built from it timed inside the seeded solve's wall time), same operator,
  same solver options.

Run ``python -m nutrlan_b200.seed_train --help``.
"""
import argparse
import json
import os
import time

import numpy as np

from . import operators as ops
from .batched import Batch
from .seednet import NOUT, SeedNet, seed_start, WEIGHTS_PATH
from .solver import DeviceOperator, solve


def potentials(seeds, L, device="cuda"):
    """Well potentials of ``ops.wells_potential`` for many seeds at once,
    evaluated on the device in FP64 -> (len(seeds), L, L) tensor."""
    import torch
    nw = 8
    prm = np.stack([ops.uniform01(int(s), np.arange(4 * nw, dtype=np.uint64)).reshape(nw, 4) for s in seeds])
    prm = torch.as_tensor(prm, dtype=torch.float64, device=device)
    cx, cy = prm[:, :, 0] * L, prm[:, :, 1] * L
    w = 4.0 + 20.0 * prm[:, :, 2]
    d = 5.0 + 45.0 * prm[:, :, 3]
    g = torch.arange(L, dtype=torch.float64, device=device)
    V = torch.zeros((len(seeds), L, L), dtype=torch.float64, device=device)
    for k in range(nw):
        dx2 = (g[None, :] - cx[:, k, None]) ** 2            # (B, L) over x
        dy2 = (g[None, :] - cy[:, k, None]) ** 2            # (B, L) over y
        r2 = dy2[:, :, None] + dx2[:, None, :]              # (B, y, x)
        V -= d[:, k, None, None] * torch.exp(-r2 / (2.0 * w[:, k, None, None] ** 2))
    return V


def generate(count, L=256, seed0=1, ned=NOUT, maxlan=48, tol=1e-8, chunk=1024, log=print):
    """Returns (V (count, L, L) float32, U (count, L*L, ned) bfloat16, info
    (count, 4) int: stat, nec, matvec, restarts), all but info on the device."""
    import torch
    Vall = torch.empty((count, L, L), dtype=torch.float32, device="cuda")
    Uall = torch.empty((count, L * L, ned), dtype=torch.bfloat16, device="cuda")
    info = np.zeros((count, 4), dtype=np.int64)
    buf = torch.empty((ned, L * L), dtype=torch.float64, device="cuda")
    for c0 in range(0, count, chunk):
        m = min(chunk, count - c0)
        t0 = time.perf_counter()
        V = potentials(range(seed0 + c0, seed0 + c0 + m), L)
        Vh = V.reshape(m, -1).cpu().numpy()
        b = Batch.stencil5([L] * m, [Vh[i] for i in range(m)])
        try:
            r = b.solve(ned=ned, maxlan=maxlan, tol=tol, maxmv=100000)
            info[c0:c0 + m] = r.info
            for i in range(m):
                b.eigenvectors(i, out=buf)
                Uall[c0 + i] = buf.t().to(torch.bfloat16)
        finally:
            b.close()
        Vall[c0:c0 + m] = V.float()
        torch.cuda.synchronize()
        log(f"generate: {c0 + m}/{count} problems, {time.perf_counter() - t0:.1f} s, "
            f"mean matvecs {r.info[:, 2].mean():.0f}, unconverged {(r.info[:, 1] < ned).sum()}")
    return Vall, Uall, info


def train(net, V, U, epochs=30, batch=32, lr=2e-3, lr_min=1e-4, lam=0.1, holdout=256, log=print):
    """Adam with a cosine learning-rate schedule; the last ``holdout``
    samples are kept for validation.  Returns a list of per-epoch records."""
    import torch
    n = V.shape[0] - holdout
    steps = max(1, n // batch)
    total = epochs * steps
    hist = []
    g = torch.Generator(device="cpu").manual_seed(1234)
    it = 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        t0 = time.perf_counter()
        acc = 0.0
        for s in range(steps):
            idx = perm[s * batch:(s + 1) * batch].cuda()
            cur = lr_min + 0.5 * (lr - lr_min) * (1.0 + np.cos(np.pi * it / total))
            loss = net.train_step(V[idx].contiguous(), U[idx].float().contiguous(), lam=lam, lr=cur)
            acc += float(loss.mean())
            it += 1
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        val = validate(net, V[n:], U[n:], batch, lam)
        rec = dict(epoch=ep + 1, train_loss=acc / steps, val_loss=val, seconds=dt,
                   samples_per_s=steps * batch / dt)
        hist.append(rec)
        log(f"train: epoch {ep + 1}/{epochs} loss {acc / steps:.4f} val {val:.4f} "
            f"({dt:.1f} s, {steps * batch / dt:.0f} samples/s)")
    return hist


def validate(net, V, U, batch=32, lam=1.0):
    tot, cnt = 0.0, 0
    for s in range(0, V.shape[0], batch):
        loss, _ = net.gradients(V[s:s + batch].contiguous(), U[s:s + batch].float().contiguous(), lam)
        tot += float(loss.sum())
        cnt += loss.size
    return tot / max(cnt, 1)


def evaluate(net, seeds, L=256, ned=NOUT, maxlan=48, tol=1e-8, restart=1, log=print, subspace=False):
    """Plain vs learned-seed solves on held-out operators.  Per seed: the
    plain solve (seeded uniform start), the seed injected as the sum of its
    Rayleigh-Ritz vectors ("rr", its NOUT projection matvecs counted) and as
    the sum of the normalised network outputs ("sum"); matvecs, wall seconds
    (network forward and projection inside the seeded times), eigenvalue
    agreement with the plain solve and true residuals of the seeded ones.
    With ``subspace`` also the seed as a subspace (seed_subspace.py): dense
    restarted Rayleigh-Ritz ("dense") and one dense cycle followed by trlan
    ("first")."""
    import torch
    from .solver import residual_norms
    out = []
    Y = torch.empty((1, L * L, NOUT), dtype=torch.float32, device="cuda")
    kw = dict(ned=ned, maxlan=maxlan, tol=tol, restart=restart, maxmv=100000, device=True)
    for s in seeds:
        A, V = ops.wells_2d(L, seed=int(s))
        rec = dict(seed=int(s))
        with DeviceOperator(A) as op:
            x0 = torch.as_tensor(ops.start_vector(A.n), device="cuda")
            ev = torch.zeros((ned + 1, A.n), dtype=torch.float64, device="cuda")
            solve(op, start=x0, evec=ev, **kw)          # warm-up, not timed
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rp = solve(op, start=x0, evec=ev, **kw)
            torch.cuda.synchronize()
            rec.update(plain_matvec=int(rp.info.matvec), plain_s=time.perf_counter() - t0, plain_nec=int(rp.nec))
            ep_ = np.sort(rp.eval[:min(rp.nec, ned)])
            Vd = torch.as_tensor(V, dtype=torch.float32, device="cuda")[None]
            for mode, project in (("rr", True), ("sum", False)):
                ev2 = torch.zeros((ned + 1, A.n), dtype=torch.float64, device="cuda")
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                net.forward(Vd, out=Y)
                _, theta, sres = seed_start(op, Y[0], out=ev2[0], project=project)
                rs = solve(op, start=ev2[0], evec=ev2, **kw)
                torch.cuda.synchronize()
                ts = time.perf_counter() - t0
                nec = min(rp.nec, rs.nec, ned)
                true_res = residual_norms(op, rs.eval[:nec], ev2[:nec])
                es_ = np.sort(rs.eval[:nec])
                rel = float(np.max(np.abs(es_ - ep_[:nec]) / np.abs(ep_[:nec]))) if nec else np.inf
                rec.update({f"{mode}_matvec": int(rs.info.matvec) + (NOUT if project else 0),
                            f"{mode}_s": ts, f"{mode}_nec": int(rs.nec), f"{mode}_eval_rel_diff": rel,
                            f"{mode}_max_true_res": float(true_res.max()) if nec else np.inf})
                if project:
                    rec["seed_res_median"] = float(np.median(sres))
            rec["tol_abs"] = tol * float(rp.info.anrm)
            if subspace:
                # The seed as a subspace (evaluation paths, seed_subspace.py).
                from .seed_subspace import dense_cycles, first_cycle_then_trlan
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                net.forward(Vd, out=Y)
                d = dense_cycles(op, Y[0], k=ned, m=maxlan, tol=tol)
                torch.cuda.synchronize()
                rec.update(dense_matvec=int(d["matvec"]), dense_s=time.perf_counter() - t0,
                           dense_cycles=int(d["cycles"]), dense_converged=bool(d["converged"]),
                           dense_eval_rel_diff=float(np.max(np.abs(np.sort(d["theta"]) - ep_[:ned]) /
                                                            np.abs(ep_[:ned]))))
                t0 = time.perf_counter()
                net.forward(Vd, out=Y)
                mv1, r1 = first_cycle_then_trlan(op, Y[0], ned=ned, m=maxlan, tol=tol, maxlan=maxlan)
                torch.cuda.synchronize()
                rec.update(first_matvec=int(mv1), first_s=time.perf_counter() - t0, first_nec=int(r1.nec))
        out.append(rec)
        log(f"eval seed {s}: plain {rec['plain_matvec']} mv {rec['plain_s'] * 1e3:.1f} ms | rr "
            f"{rec['rr_matvec']} mv (incl. {NOUT} projection) {rec['rr_s'] * 1e3:.1f} ms | sum "
            f"{rec['sum_matvec']} mv {rec['sum_s'] * 1e3:.1f} ms | seed residual median "
            f"{rec['seed_res_median']:.2e}")
    return out


def summarize(recs):
    m = lambda k: float(np.mean([r[k] for r in recs]))
    out = dict(problems=len(recs), plain_matvec=m("plain_matvec"), plain_s=m("plain_s"))
    for mode in ("rr", "sum", "dense", "first"):
        if f"{mode}_matvec" not in recs[0]:
            continue
        out[f"{mode}_matvec"] = m(f"{mode}_matvec")
        out[f"{mode}_s"] = m(f"{mode}_s")
        out[f"{mode}_matvec_ratio"] = out["plain_matvec"] / out[f"{mode}_matvec"]
        out[f"{mode}_time_ratio"] = out["plain_s"] / out[f"{mode}_s"]
    return out


def time_steps(batch, steps, L=256, lam=0.1):
    """Wall time of training steps and forward passes on random potentials
    and orthonormal targets (for profiling the network kernels)."""
    import torch
    net = SeedNet(L, L, max_batch=batch)
    g = torch.Generator(device="cuda").manual_seed(0)
    V = -50.0 * torch.rand((batch, L, L), device="cuda", generator=g)
    U = torch.randn((batch, L * L, NOUT), device="cuda", generator=g)
    U = U / torch.linalg.vector_norm(U, dim=1, keepdim=True)
    for _ in range(2):
        net.train_step(V, U, lam=lam, lr=1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        net.train_step(V, U, lam=lam, lr=1e-3)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    Y = torch.empty((batch, L * L, NOUT), device="cuda")
    net.forward(V, out=Y)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        net.forward(V, out=Y)
    torch.cuda.synchronize()
    df = (time.perf_counter() - t0) / steps
    flop_fwd = 2.0 * L * L * 9 * (1 * 32 + 3 * 32 * 32 + 32 * 16)
    net.close()
    return dict(batch=batch, train_ms=dt * 1e3, samples_per_s=batch / dt,
                train_tflops=3 * flop_fwd * batch / dt / 1e12, forward_ms=df * 1e3,
                forward_tflops=flop_fwd * batch / df / 1e12)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--time-steps", type=int, default=0,
                    help="only time this many training steps / forward passes on random data")
    ap.add_argument("--samples", type=int, default=20000)
    ap.add_argument("--L", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lam", type=float, default=0.1)
    ap.add_argument("--maxlan", type=int, default=48)
    ap.add_argument("--eval", type=int, default=16, help="held-out operators for the A/B test")
    ap.add_argument("--weights", default=WEIGHTS_PATH)
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--report", default=None, help="write a JSON report here")
    a = ap.parse_args(argv)
    if a.time_steps:
        print(json.dumps(time_steps(a.batch, a.time_steps, a.L)))
        return
    rep = dict(args=vars(a))
    t0 = time.perf_counter()
    V, U, info = generate(a.samples, a.L, seed0=1, maxlan=a.maxlan)
    rep["generate_seconds"] = time.perf_counter() - t0
    rep["generate_matvec_mean"] = float(info[:, 2].mean())
    rep["generate_unconverged"] = int((info[:, 1] < NOUT).sum())
    net = SeedNet(a.L, a.L, max_batch=a.batch)
    if a.init:
        net.weights = np.load(a.init)
    t0 = time.perf_counter()
    rep["train"] = train(net, V, U, epochs=a.epochs, batch=a.batch, lr=a.lr, lam=a.lam)
    rep["train_seconds"] = time.perf_counter() - t0
    os.makedirs(os.path.dirname(os.path.abspath(a.weights)), exist_ok=True)
    net.save(a.weights)
    del V, U
    ev = evaluate(net, range(10 ** 6, 10 ** 6 + a.eval), a.L, maxlan=a.maxlan)
    rep["eval"] = ev
    rep["summary"] = summarize(ev)
    print(json.dumps(rep["summary"]))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()

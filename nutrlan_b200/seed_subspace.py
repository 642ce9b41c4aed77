"""Subspace injection of the learned seed, measured on the GPU.

The learned seed predicts k = 16 vectors.  Feeding them to thick-restart
Lanczos as a subspace (rather than as one start vector) needs a projected
matrix that is no longer an arrowhead: a thick-restart state must satisfy
A X = X Theta + q b^T with ONE residual direction q (SRC/trlcore.c:961-1017
builds the first step after a restart on exactly that), and the
Rayleigh-Ritz vectors X of a predicted subspace have k independent residual
directions.  The two evaluated ways of carrying the subspace are:

* ``dense``: restarted Rayleigh-Ritz over span(X, K_{m-k}(A, q)), the
  projected matrix kept dense (its X-rows are the X^T A q_j coefficients
  that the Gram-Schmidt projection produces anyway), exact residuals of the
  Ritz pairs from the stored products A V, restart by keeping the k wanted
  Ritz vectors and starting the next Krylov block from the sum of their
  normalised residuals, until all k residuals are <= tol * ||A||;
* ``first_cycle``: one such dense cycle from the seed, then the plain
  thick-restart solver (trlan) started from the sum of the cycle's Ritz
  vectors, which is a valid single-vector start.

Both run on the device: operator applications through the library's
built-in operator (trlx_matvec), projections V^T r through the library's
trlx_g_dot kernel, updates and the small dense eigenproblems with torch.
Matvec counts include the k applications of the seed's Rayleigh-Ritz
projection.  These are evaluation paths beside the solver (the product's
seeded solve is the start-vector channel, guess = 1), kept to measure what
the subspace would buy.
"""
import ctypes as C
import json

from ._lib import load


def _matvec_fn(lib):
    f = lib.trlx_matvec
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    f.restype = None
    return f


class _Ops:
    def __init__(self, op):
        import torch
        self.torch = torch
        self.lib = load()
        self.mv = _matvec_fn(self.lib)
        self.op = op
        self.n = op.n
        self.count = 0

    def apply(self, x, y):
        self.mv(self.n, 1, x.data_ptr(), self.n, y.data_ptr(), self.n, self.op.handle)
        self.count += 1

    def apply_block(self, X):
        Y = self.torch.empty_like(X)
        for j in range(X.shape[1]):
            xj = X[:, j].contiguous()
            yj = self.torch.empty_like(xj)
            self.apply(xj, yj)
            Y[:, j] = yj
        return Y

    def project(self, V, r):
        """V^T r with the library's projection kernel (V column-major: the
        columns of a (m, n) row-major tensor)."""
        m = V.shape[0]
        h = self.torch.empty(m, dtype=self.torch.float64, device=r.device)
        rc = self.lib.trlx_g_dot(self.n, V.data_ptr(), self.n, m, V.data_ptr(), self.n, 0, r.data_ptr(),
                                 h.data_ptr(), None)
        if rc != 0:
            raise RuntimeError(f"trlx_g_dot failed ({rc})")
        return h


def _rayleigh_ritz(o, Y):
    """Orthonormalise the seed (columns of Y, n x k) and project: (Z, AZ,
    theta) with the Ritz vectors as rows."""
    torch = o.torch
    Q, _ = torch.linalg.qr(Y.to(torch.float64))
    AQ = o.apply_block(Q)
    H = Q.t() @ AQ
    th, S = torch.linalg.eigh(0.5 * (H + H.t()))
    return (Q @ S).t().contiguous(), (AQ @ S).t().contiguous(), th


def dense_cycles(op, Y, k=16, m=48, tol=1e-8, maxmv=20000, cycles=None):
    """Restarted dense Rayleigh-Ritz from the seed (columns of Y, an n x k
    device tensor as the network writes it).  Returns dict(matvec, cycles,
    converged, theta (k), Z (k x n), max_res, anrm)."""
    o = _Ops(op)
    torch = o.torch
    Z, AZ, th = _rayleigh_ritz(o, Y)
    Z, AZ, th = Z[:k], AZ[:k], th[:k]
    anrm = float(th.abs().max())
    done = 0
    while o.count < maxmv and (cycles is None or done < cycles):
        done += 1
        R = AZ - th[:, None] * Z
        rn = torch.linalg.vector_norm(R, dim=1)
        q = (R / rn.clamp_min(1e-300)[:, None]).sum(0)
        for _ in range(2):
            q -= o.project(Z, q) @ Z
        q /= torch.linalg.vector_norm(q)
        V = [q]
        AV = []
        y = torch.empty_like(q)
        for j in range(m - k):
            o.apply(V[-1], y)
            AV.append(y.clone())
            if j == m - k - 1:
                break
            B = torch.cat([Z, torch.stack(V)])
            r = y.clone()
            for _ in range(2):
                r -= o.project(B, r) @ B
            V.append(r / torch.linalg.vector_norm(r))
        Vm = torch.cat([Z, torch.stack(V)])
        AVm = torch.cat([AZ, torch.stack(AV)])
        H = Vm @ AVm.t()
        th_all, S = torch.linalg.eigh(0.5 * (H + H.t()))
        anrm = max(anrm, float(th_all.abs().max()))
        S, th = S[:, :k], th_all[:k]
        Z, AZ = (S.t() @ Vm).contiguous(), (S.t() @ AVm).contiguous()
        res = torch.linalg.vector_norm(AZ - th[:, None] * Z, dim=1)
        if bool((res <= tol * anrm).all()):
            break
    res = torch.linalg.vector_norm(AZ - th[:, None] * Z, dim=1)
    return dict(matvec=o.count, cycles=done, converged=bool((res <= tol * anrm).all()),
                theta=th.cpu().numpy(), Z=Z, max_res=float(res.max()), anrm=anrm)


def first_cycle_then_trlan(op, Y, ned=16, m=48, tol=1e-8, maxlan=48):
    """One dense cycle from the seed, then trlan started from the sum of the
    cycle's Ritz vectors.  Returns (total matvecs, SolveResult)."""
    import torch
    from .solver import solve
    d = dense_cycles(op, Y, k=ned, m=m, tol=tol, cycles=1)
    start = d["Z"].sum(0)
    ev = torch.zeros((ned + 1, op.n), dtype=torch.float64, device=start.device)
    ev[0].copy_(start)
    r = solve(op, ned=ned, maxlan=maxlan, tol=tol, restart=1, maxmv=100000, start=ev[0], evec=ev, device=True)
    return d["matvec"] + int(r.info.matvec), r


__all__ = ["dense_cycles", "first_cycle_then_trlan", "seed_quality_study"]


def seed_quality_study(problems=4, eps=(1e-1, 1e-2, 1e-3, 1e-4, 1e-6), L=256, ned=16, maxlan=48, tol=1e-8,
                       seed0=10 ** 6, log=print, weights=None):
    """Matvecs to residual <= tol * ||A|| on held-out well operators for seeds
    of known quality: the exact lowest 16 eigenvectors (from a plain solve of
    the 60 lowest pairs) plus eps times a unit-norm error spread over the
    next 44 eigenvectors and white noise, fed in three ways: as one start
    vector (the sum of the seed's Rayleigh-Ritz vectors, then trlan; the
    product's channel), as a dense restarted subspace (dense_cycles) and as
    one dense cycle followed by trlan (first_cycle_then_trlan).  The trained
    network's own seed is measured the same way.  Returns a list of records
    (one per operator), all on the GPU."""
    import numpy as np
    import torch
    from . import operators as ops
    from .seednet import SeedNet, seed_start
    from .solver import DeviceOperator, solve
    out = []
    net = SeedNet.pretrained(weights) if weights else SeedNet.pretrained()
    try:
        for s in range(seed0, seed0 + problems):
            A, V = ops.wells_2d(L, seed=s)
            rec = {"seed": s}
            with DeviceOperator(A) as op:
                x0 = torch.as_tensor(ops.start_vector(A.n), device="cuda")
                plain = solve(op, ned=ned, maxlan=maxlan, tol=tol, restart=1, maxmv=100000, start=x0, device=True)
                rec["plain"] = int(plain.info.matvec)
                big = solve(op, ned=60, maxlan=160, tol=1e-10, restart=1, maxmv=200000, start=x0, device=True)
                U = big.evec[:60].t().contiguous()                       # (n, 60), ascending
                gen = torch.Generator(device="cuda").manual_seed(s)
                C = torch.randn((44, ned), dtype=torch.float64, device="cuda", generator=gen)
                Wn = torch.randn((A.n, ned), dtype=torch.float64, device="cuda", generator=gen)
                E = U[:, ned:] @ C / np.sqrt(44.0) + 0.1 * Wn / np.sqrt(A.n)
                Y_net = torch.empty((1, A.n, ned), dtype=torch.float32, device="cuda")
                net.forward(torch.as_tensor(V, dtype=torch.float32, device="cuda")[None], out=Y_net)
                seeds = [("net", Y_net[0].double())] + [(f"eps{e:g}", U[:, :ned] + e * E) for e in eps]
                for name, Y in seeds:
                    ev = torch.zeros((ned + 1, A.n), dtype=torch.float64, device="cuda")
                    seed_start(op, Y.float().contiguous(), out=ev[0], project=True)
                    r = solve(op, ned=ned, maxlan=maxlan, tol=tol, restart=1, maxmv=100000, start=ev[0], evec=ev,
                              device=True)
                    d = dense_cycles(op, Y, k=ned, m=maxlan, tol=tol)
                    f, _ = first_cycle_then_trlan(op, Y, ned=ned, m=maxlan, tol=tol, maxlan=maxlan)
                    rec[name] = {"start_vector": int(r.info.matvec) + ned, "dense": int(d["matvec"]),
                                 "dense_converged": bool(d["converged"]), "first_cycle": int(f)}
            out.append(rec)
            log(json.dumps(rec))
    finally:
        net.close()
    return out


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description=seed_quality_study.__doc__)
    ap.add_argument("--problems", type=int, default=4)
    ap.add_argument("--out", default=None, help="write the records as JSON here")
    ap.add_argument("--weights", default=None, help="network weights (default: the packaged ones)")
    ap.add_argument("--eps", type=float, nargs="*", default=[1e-1, 1e-2, 1e-3, 1e-4, 1e-6])
    a = ap.parse_args(argv)
    recs = seed_quality_study(a.problems, eps=tuple(a.eps), weights=a.weights)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(recs, f, indent=1)


if __name__ == "__main__":
    main()

"""Learned seed for the thick-restart solver (trlx_seednet_* and
trlx_seed_start in include/trlx.h).

A 5-layer convolutional network maps the potential V of -Laplacian + V on an
H x W grid to 16 vectors approximating the span of the lowest eigenvectors.
Its forward and backward passes are the library's BF16 tensor-core kernels;
training and inference never leave the GPU.  ``seed_start`` Rayleigh-Ritz
projects the prediction on the operator and returns the sum of the Ritz
vectors, which the solver takes as its ordinary start vector (guess = 1):
the recurrence, restarts and convergence test stay those of a plain solve,
and the seeded random start remains the fallback when no network is given.

    net = SeedNet(256, 256, max_batch=32)
    loss = net.train_step(V_batch, U_batch, lam=1.0, lr=1e-3)
    Y = net.forward(V)                        # (1, H*W, 16) float32
    start, theta, res = seed_start(op, Y[0])  # op: DeviceOperator
    solve(op, ned=16, ..., start=start)
"""
import ctypes as C
import os

import numpy as np

from ._lib import load

NOUT = 16
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                            "seednet_wells256.npy")


def _declare(lib):
    P = C.POINTER
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    lib.trlx_seednet_create.argtypes = [i, i, i, C.c_ulonglong, P(vp)]
    lib.trlx_seednet_destroy.argtypes = [vp]
    lib.trlx_seednet_destroy.restype = None
    lib.trlx_seednet_forward.argtypes = [vp, i, vp, vp]
    lib.trlx_seednet_gradients.argtypes = [vp, i, vp, vp, f, vp, vp]
    lib.trlx_seednet_train_step.argtypes = [vp, i, vp, vp, f, f, vp]
    lib.trlx_seednet_get_weights.argtypes = [vp, vp]
    lib.trlx_seednet_set_weights.argtypes = [vp, vp]
    lib.trlx_seednet_num_params.argtypes = []
    lib.trlx_seed_start.argtypes = [vp, i, i, vp, i, vp, vp, vp]
    return lib


def _ptr(a, dtype, shape=None, output=False):
    """(pointer, keep-alive) of a float32/float64 numpy array or CUDA tensor.
    Inputs are converted when needed; outputs must already match."""
    if hasattr(a, "data_ptr"):
        import torch
        want = torch.float32 if dtype == np.float32 else torch.float64
        if a.dtype != want or not a.is_contiguous():
            if output:
                raise ValueError(f"output must be a contiguous {want} tensor")
            a = a.to(want).contiguous()
        if shape is not None and a.numel() != int(np.prod(shape)):
            raise ValueError(f"expected {shape}, got {tuple(a.shape)}")
        return C.c_void_p(a.data_ptr()), a
    if output and (not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous):
        raise ValueError(f"output must be a contiguous {np.dtype(dtype)} array")
    a = np.ascontiguousarray(a, dtype=dtype)
    if shape is not None and a.size != int(np.prod(shape)):
        raise ValueError(f"expected {shape}, got {a.shape}")
    return C.c_void_p(a.ctypes.data), a


class SeedNet:
    def __init__(self, H=256, W=256, max_batch=32, seed=0x5EED5EED):
        self.lib = _declare(load())
        self.H, self.W, self.max_batch = H, W, max_batch
        self.handle = C.c_void_p()
        rc = self.lib.trlx_seednet_create(H, W, max_batch, seed, C.byref(self.handle))
        if rc:
            raise RuntimeError(f"trlx_seednet_create failed ({rc})")
        self.num_params = self.lib.trlx_seednet_num_params()

    def _check(self, rc, what):
        if rc:
            raise RuntimeError(f"{what} failed ({rc})")

    def _batch(self, V):
        B = V.shape[0] if len(V.shape) == 3 else 1
        if B > self.max_batch:
            raise ValueError(f"batch {B} > max_batch {self.max_batch}")
        return B

    def forward(self, V, out=None):
        """V: (B, H, W) potentials.  Returns (B, H*W, 16) float32 (numpy, or
        `out` when given: a float32 array or CUDA tensor of that size)."""
        B = self._batch(V)
        pv, _keep = _ptr(V, np.float32, (B, self.H, self.W))
        if out is None:
            out = np.zeros((B, self.H * self.W, NOUT), np.float32)
        po, _ = _ptr(out, np.float32, (B, self.H * self.W, NOUT), output=True)
        self._check(self.lib.trlx_seednet_forward(self.handle, B, pv, po), "trlx_seednet_forward")
        return out

    def gradients(self, V, U, lam=1.0):
        B = self._batch(V)
        pv, _k1 = _ptr(V, np.float32, (B, self.H, self.W))
        pu, _k2 = _ptr(U, np.float32, (B, self.H * self.W, NOUT))
        loss = np.zeros(B, np.float32)
        g = np.zeros(self.num_params, np.float32)
        self._check(self.lib.trlx_seednet_gradients(self.handle, B, pv, pu, lam, loss.ctypes.data,
                                                    g.ctypes.data), "trlx_seednet_gradients")
        return loss, g

    def train_step(self, V, U, lam=1.0, lr=1e-3):
        """One Adam step; returns the per-sample losses before the update."""
        B = self._batch(V)
        pv, _k1 = _ptr(V, np.float32, (B, self.H, self.W))
        pu, _k2 = _ptr(U, np.float32, (B, self.H * self.W, NOUT))
        loss = np.zeros(B, np.float32)
        self._check(self.lib.trlx_seednet_train_step(self.handle, B, pv, pu, lam, lr, loss.ctypes.data),
                    "trlx_seednet_train_step")
        return loss

    @property
    def weights(self):
        w = np.zeros(self.num_params, np.float32)
        self._check(self.lib.trlx_seednet_get_weights(self.handle, w.ctypes.data), "get_weights")
        return w

    @weights.setter
    def weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.num_params:
            raise ValueError(f"expected {self.num_params} weights, got {w.size}")
        self._check(self.lib.trlx_seednet_set_weights(self.handle, w.ctypes.data), "set_weights")

    def save(self, path):
        np.save(path, self.weights)

    @classmethod
    def pretrained(cls, path=WEIGHTS_PATH, H=256, W=256, max_batch=1):
        net = cls(H, W, max_batch)
        net.weights = np.load(path)
        return net

    def close(self):
        if self.handle:
            self.lib.trlx_seednet_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def seed_start(op, Y, out=None, project=True):
    """Start vector from a predicted subspace Y ((n, k) float32, numpy or
    CUDA tensor) on the DeviceOperator `op`: the sum of its Rayleigh-Ritz
    vectors (project=True, k operator applications) or of its normalised
    columns (project=False).  Returns (start, theta, res): start is `out`
    (n doubles, numpy or CUDA tensor) or a new numpy array; theta/res are the
    Ritz values and residual norms (zeros / -1 without projection)."""
    lib = _declare(load())
    n = op.n
    k = Y.shape[-1]
    py, _keep = _ptr(Y, np.float32, (n, k))
    if out is None:
        out = np.zeros(n)
    po, _ = _ptr(out, np.float64, (n,), output=True)
    theta = np.zeros(k)
    res = np.zeros(k)
    r = lib.trlx_seed_start(op.handle, n, k, py, 1 if project else 0, po, theta.ctypes.data, res.ctypes.data)
    if r < 1:
        raise RuntimeError(f"trlx_seed_start failed ({r})")
    return out, theta[:r], res[:r]

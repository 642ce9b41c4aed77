"""FP64 numpy restatement of the seed network (test infrastructure only).

The network and its loss have no counterpart in the nuTRLan reference; this
module restates the math that ``nutrlan_b200/csrc/kernels/seednet.cu``
implements so that the GPU forward pass, the loss and every gradient can be
checked on the CPU:

* input (V - min V) / 50 per sample (FP32, then bfloat16);
* 5 layers of 3x3 convolutions, dilations (1, 2, 4, 8, 1), channels
  1 -> 32 -> 32 -> 32 -> 32 -> 16, ReLU after the first four, zero "same"
  padding; out[y, x, co] = sum_{tap, ci} in[y + d*dy, x + d*dx, ci] *
  W[tap, ci, co] + b[co] with tap = 3 * (dy + 1) + (dx + 1);
* loss per sample  sum_k (1 - |U^T y_k|^2 / |y_k|^2)
  + lam * sum_{j != k} (y_j . y_k)^2 / (|y_j|^2 |y_k|^2).

With ``emulate=True`` values are rounded to bfloat16 (round to nearest even)
exactly where the CUDA path stores bfloat16: the scaled input, the weights,
the hidden activations, the output gradient and the back-propagated
activation gradients.  Everything else is FP64, so the remaining difference
to the GPU is its FP32 accumulation.
"""
import numpy as np

DIL = (1, 2, 4, 8, 1)
CIN = (1, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 16)
NC = 32
NOUT = 16
TAPS = 9
LAYER_LEN = TAPS * NC * NC + NC
IN_SCALE = np.float32(1.0 / 50.0)


def bf16(x):
    """Round to bfloat16 (nearest even) and return FP64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    """Flat parameter vector -> [(W (9, 32, 32) [tap, ci, co], b (32,))]."""
    params = np.asarray(params, dtype=np.float64)
    out = []
    for l in range(5):
        p = params[l * LAYER_LEN:(l + 1) * LAYER_LEN]
        out.append((p[:TAPS * NC * NC].reshape(TAPS, NC, NC), p[TAPS * NC * NC:]))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in layers])


def _shift(x, dy, dx):
    """s[b, y, x] = x[b, y + dy, x + dx] (zero outside)."""
    B, H, W = x.shape[:3]
    s = np.zeros_like(x)
    ys, yd = max(0, -dy), min(H, H - dy)
    xs, xd = max(0, -dx), min(W, W - dx)
    if ys < yd and xs < xd:
        s[:, ys:yd, xs:xd] = x[:, ys + dy:yd + dy, xs + dx:xd + dx]
    return s


def conv(x, W, b, dil):
    out = 0.0
    for tap in range(TAPS):
        dy, dx = (tap // 3 - 1) * dil, (tap % 3 - 1) * dil
        out = out + _shift(x, dy, dx) @ W[tap]
    return out + (0.0 if b is None else b)


def forward(params, V, emulate=True):
    """V: (B, H, W) potentials.  Returns (activations, Y) with activations
    [input, hidden1..hidden4] as (B, H, W, 32) and Y (B, H, W, 16)."""
    rnd = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params)
    V = np.asarray(V, dtype=np.float32)
    x = np.zeros(V.shape + (NC,))
    vmin = V.min(axis=(1, 2), keepdims=True)
    x[..., 0] = rnd((V - vmin) * IN_SCALE)
    acts = [x]
    for l, (W, b) in enumerate(layers):
        Wq = rnd(W)
        z = conv(acts[-1], Wq, b, DIL[l])
        if l < 4:
            acts.append(rnd(np.maximum(z, 0.0)))
        else:
            Y = z[..., :NOUT]
    return acts, Y


def loss_terms(Y, U, lam):
    """Per-sample loss and dL/dY (unscaled) for Y, U of shape (B, P, 16)."""
    B = Y.shape[0]
    L = np.zeros(B)
    dY = np.zeros_like(Y)
    for s in range(B):
        y, u = Y[s], U[s]
        C = u.T @ y
        G = y.T @ y
        n2 = np.maximum(np.diag(G).copy(), 1e-30)
        cc = np.sum(C * C, axis=0)
        off = G * G / np.outer(n2, n2)
        np.fill_diagonal(off, 0.0)
        L[s] = np.sum(1.0 - cc / n2) + lam * off.sum()
        A = -2.0 * C / n2[None, :]
        Bm = 4.0 * lam * G / np.outer(n2, n2)
        np.fill_diagonal(Bm, 2.0 * cc / n2 ** 2 - 4.0 * lam * off.sum(axis=0) / n2)
        dY[s] = u @ A + y @ Bm
    return L, dY


def loss_and_grad(params, V, U, lam, emulate=True):
    """V: (B, H, W); U: (B, H*W, 16).  Returns (loss per sample, flat
    gradient of the batch-mean loss)."""
    rnd = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params)
    B, H, W = np.shape(V)
    acts, Y = forward(params, V, emulate)
    U = np.asarray(U, dtype=np.float64).reshape(B, H * W, NOUT)
    L, dY = loss_terms(Y.reshape(B, H * W, NOUT), U, lam)
    g = np.zeros((B, H, W, NC))
    g[..., :NOUT] = rnd(dY.reshape(B, H, W, NOUT) / B)
    grads = [None] * 5
    for l in range(4, -1, -1):
        if l < 4:
            g = np.where(acts[l + 1] > 0.0, g, 0.0)
        x = acts[l]
        gW = np.zeros((TAPS, NC, NC))
        for tap in range(TAPS):
            dy, dx = (tap // 3 - 1) * DIL[l], (tap % 3 - 1) * DIL[l]
            gW[tap] = np.einsum("bhwi,bhwo->io", _shift(x, dy, dx), g)
        gb = g.sum(axis=(0, 1, 2))
        # Only real channels are parameters.
        gW[:, CIN[l]:, :] = 0.0
        gW[:, :, COUT[l]:] = 0.0
        gb[COUT[l]:] = 0.0
        grads[l] = (gW, gb)
        if l > 0:
            Wq = rnd(layers[l][0])
            gin = 0.0
            for tap in range(TAPS):
                dy, dx = (tap // 3 - 1) * DIL[l], (tap % 3 - 1) * DIL[l]
                gin = gin + _shift(g, -dy, -dx) @ Wq[tap].T
            g = rnd(gin)
    return L, pack(grads)


def init_params(seed):
    """Deterministic He-style initial weights (any init works for tests)."""
    rng = np.random.default_rng(seed)
    layers = []
    for l in range(5):
        W = np.zeros((TAPS, NC, NC))
        W[:, :CIN[l], :COUT[l]] = rng.standard_normal((TAPS, CIN[l], COUT[l])) * np.sqrt(2.0 / (TAPS * CIN[l]))
        b = np.zeros(NC)
        b[:COUT[l]] = 0.01 * rng.standard_normal(COUT[l])
        layers.append((W.astype(np.float32).astype(np.float64), b.astype(np.float32).astype(np.float64)))
    return pack(layers)

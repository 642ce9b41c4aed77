"""numpy FP64 restatement of the hot-path vector operations (test
infrastructure only).  Each function states the reference code it follows.
"""
import numpy as np


def g_dot(v1, m1, v2, m2, rr):
    """wrk = [v1(:, :m1) v2(:, :m2)]^H rr.
    Reference: trl_g_dot_ (SRC/trl_comm_none.c:238-329); complex
    ztrl_g_dot_ (SRC/ztrl_comm_none.c:16-130) uses conjugate transposes."""
    parts = []
    if m1 > 0:
        parts.append(np.conj(v1[:, :m1]).T @ rr)
    if m2 > 0:
        parts.append(np.conj(v2[:, :m2]).T @ rr)
    return np.concatenate(parts) if parts else np.zeros(0, dtype=rr.dtype)


def cgs_update(V, h, r):
    """r - V h: the dgemv('N') subtraction of trl_cgs (SRC/trlcore.c:2996-3011)."""
    return r - V @ h


def cgs_pass(V, r):
    """One classical Gram-Schmidt pass: (h, r - V h, ||h||^2, ||r - V h||^2)
    as trl_cgs computes them (SRC/trlcore.c:2993-3036)."""
    h = np.conj(V).T @ r
    rn = r - V @ h
    return h, rn, float(np.vdot(h, h).real), float(np.vdot(rn, rn).real)


def ritz_vectors(V, Y):
    """V * Y: trl_ritz_vectors (SRC/trlcore.c:2761-2910), complex
    ztrl_ritz_vectors with real Y (SRC/ztrlcore.c:1570-1751)."""
    return V @ Y


def lanczos_alpha(q, y):
    """alpha = Re(q^H y) (SRC/trlcore.c:1107; SRC/ztrlcore.c:875-877)."""
    return float(np.vdot(q, y).real)


def csr_matvec(row_ptr, col, val, x):
    """y = A x for CSR (the user operator of the examples)."""
    n = len(row_ptr) - 1
    out = np.zeros(n, dtype=np.result_type(val, x))
    counts = np.diff(row_ptr)
    nz = counts > 0
    if nz.any():
        # reduceat over the starts of non-empty rows only: an empty row would
        # otherwise pick up the element at its start index.
        out[nz] = np.add.reduceat(val * x[col], row_ptr[:-1][nz])
    return out


def ritz_projection(V, matvec, lohi=-1):
    """Rayleigh-Ritz over the rows of V (nev near-orthonormal vectors), the
    five steps trl_ritz_projection documents (SRC/trlan.c:1443-1452):
    G = V V^T = R^T R (Cholesky), H = R^-T (V A V^T) R^-1 = Y D Y^T, Ritz
    vectors (R^-1 Y)^T V, residuals ||A x - d x||.  Returns (d, X, res) in
    ascending order of d, shifted like the reference's output (lohi < 0:
    drop the last pair; lohi > 0: drop the first).

    The reference's own code does not compute this: it fills the lower
    triangle of V^T A V and the transposed copy from column i-1 instead of
    column i (SRC/trlan.c:1589-1593, 1602-1606), which leaves a zero row in
    the projected matrix, so its eigenvalues are wrong; this restatement
    follows the documented steps."""
    V = np.asarray(V, dtype=np.float64)
    G = V @ V.T
    R = np.linalg.cholesky(G).T                    # G = R^T R, R upper
    AV = np.array([matvec(v) for v in V])
    H1 = V @ AV.T
    H1 = 0.5 * (H1 + H1.T)
    Rinv = np.linalg.inv(R)
    H = Rinv.T @ H1 @ Rinv
    d, Y = np.linalg.eigh(H)
    X = (Rinv @ Y).T @ V
    res = np.array([np.linalg.norm(matvec(x) - di * x) for di, x in zip(d, X)])
    if lohi < 0:
        return d[:-1], X[:-1], res[:-1]
    if lohi > 0:
        return d[1:], X[1:], res[1:]
    return d, X, res

"""Synthetic operator families of the benchmark configurations, as CSR.

Every random number comes from ``uniform01(seed, i)``: a counter-based
splitmix64 stream that the CUDA kernels reproduce bit for bit
(``uniform01`` in csrc/kernels/common.cuh), so the GPU runs, the oracle runs
and the CPU baseline see identical operators and start vectors.

Families (sizes from the benchmark configurations):
  * ``laplacian_2d(L)``      5-point Dirichlet Laplacian (4 / -1), n = L^2;
                             eigenvalues 4 - 2cos(i pi/(L+1)) - 2cos(j pi/(L+1)).
  * ``anderson_3d(L, W)``    periodic 7-point hopping -1 plus diagonal
                             potential uniform[-W/2, W/2], n = L^3.
  * ``peierls_2d(L, phi)``   complex Hermitian tight binding on a periodic
                             L x L lattice, Landau-gauge Peierls phases for
                             flux phi per plaquette, diagonal uniform[-1, 1].
  * ``wells_2d(L, ...)``     -Laplacian (Dirichlet) + sum of Gaussian wells.
  * ``batched_laplacians``   L x L Laplacians plus uniform[0, 2] diagonals.
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def uniform01(seed, idx):
    """Counter-based uniform [0,1) numbers: splitmix64 finaliser of
    seed + golden_gamma * (idx + 1), top 53 bits."""
    idx = np.asarray(idx, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * (idx + np.uint64(1))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def start_vector(n, seed=12345):
    """Start vector uniform[-1, 1] (not normalised; the solver normalises)."""
    return 2.0 * uniform01(seed, np.arange(n, dtype=np.uint64)) - 1.0


class CSR:
    """CSR matrix with int64 row pointers, int32 columns, float64/complex128
    values; rows sorted by column."""

    def __init__(self, n, row_ptr, col, val):
        self.n = int(n)
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val)

    @property
    def nnz(self):
        return int(self.row_ptr[-1])

    def matvec(self, x):
        """y = A x (numpy, for the CPU checks)."""
        out = np.zeros(self.n, dtype=np.result_type(self.val, x))
        nz = np.diff(self.row_ptr) > 0
        if nz.any():
            out[nz] = np.add.reduceat(self.val * x[self.col], self.row_ptr[:-1][nz])
        return out

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row_ptr), shape=(self.n, self.n))


def _assemble(n, rows, cols, vals):
    """CSR from coordinate lists (no duplicates), rows sorted by column."""
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    counts = np.bincount(rows, minlength=n)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return CSR(n, row_ptr, cols.astype(np.int32), vals)


def laplacian_2d(L, diag=None):
    """5-point Dirichlet Laplacian on an L x L grid, site (i, j) -> i + L*j.
    ``diag`` (length L^2) is added to the diagonal when given."""
    n = L * L
    idx = np.arange(n, dtype=np.int64)
    i, j = idx % L, idx // L
    rows, cols, vals = [idx], [idx], [np.full(n, 4.0) + (0.0 if diag is None else diag)]
    for di, dj in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        ii, jj = i + di, j + dj
        ok = (ii >= 0) & (ii < L) & (jj >= 0) & (jj < L)
        rows.append(idx[ok])
        cols.append((ii + L * jj)[ok])
        vals.append(np.full(int(ok.sum()), -1.0))
    return _assemble(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def laplacian_2d_eigs(L):
    """All eigenvalues of laplacian_2d(L), ascending."""
    k = np.arange(1, L + 1)
    c = 2.0 - 2.0 * np.cos(k * np.pi / (L + 1))
    return np.sort((c[:, None] + c[None, :]).ravel())


def anderson_3d(L, W=4.0, seed=2024):
    """3D Anderson model: periodic 7-point stencil with hopping -1 and
    diagonal uniform[-W/2, W/2]; site (x, y, z) -> x + L*(y + L*z)."""
    n = L ** 3
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % L, (idx // L) % L, idx // (L * L)
    diag = W * (uniform01(seed, idx.astype(np.uint64)) - 0.5)
    nbrs = []
    for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        xx, yy, zz = (x + d[0]) % L, (y + d[1]) % L, (z + d[2]) % L
        nbrs.append(xx + L * (yy + L * zz))
    cols = np.stack([idx] + nbrs, axis=1)                 # (n, 7)
    vals = np.empty((n, 7))
    vals[:, 0] = diag
    vals[:, 1:] = -1.0
    order = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    vals = np.take_along_axis(vals, order, axis=1)
    row_ptr = np.arange(0, 7 * n + 1, 7, dtype=np.int64)
    return CSR(n, row_ptr, cols.reshape(-1).astype(np.int32), vals.reshape(-1))


def peierls_2d(L, phi=1.0 / 64.0, W=2.0, seed=4242):
    """Complex Hermitian 2D tight binding, periodic L x L, Landau gauge:
    x-bonds -1, y-bonds (x, y) -> (x, y+1) carry -exp(i 2 pi phi x);
    diagonal uniform[-W/2, W/2].  Periodic in x requires L*phi integer."""
    n = L * L
    idx = np.arange(n, dtype=np.int64)
    x, y = idx % L, idx // L
    diag = W * (uniform01(seed, idx.astype(np.uint64)) - 0.5)
    ph = np.exp(2j * np.pi * phi * x)
    xp, xm = (x + 1) % L + L * y, (x - 1) % L + L * y
    yp, ym = x + L * ((y + 1) % L), x + L * ((y - 1) % L)
    # H[(x,y+1),(x,y)] = -e^{i theta_x}; so row r gets -conj(ph) from (x,y+1)
    # and -ph from (x,y-1).
    cols = np.stack([idx, xp, xm, yp, ym], axis=1)
    vals = np.stack([diag.astype(np.complex128), -np.ones(n, np.complex128),
                     -np.ones(n, np.complex128), -np.conj(ph), -ph], axis=1)
    order = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, order, axis=1)
    vals = np.take_along_axis(vals, order, axis=1)
    row_ptr = np.arange(0, 5 * n + 1, 5, dtype=np.int64)
    return CSR(n, row_ptr, cols.reshape(-1).astype(np.int32), vals.reshape(-1))


def wells_potential(L, seed, nwells=8):
    """Sum of Gaussian wells: centres uniform in the domain, widths
    uniform[4, 24] cells, depths uniform[5, 50]; V <= 0."""
    u = uniform01(seed, np.arange(4 * nwells, dtype=np.uint64)).reshape(nwells, 4)
    cx, cy = u[:, 0] * L, u[:, 1] * L
    w = 4.0 + 20.0 * u[:, 2]
    d = 5.0 + 45.0 * u[:, 3]
    gx, gy = np.meshgrid(np.arange(L), np.arange(L), indexing="xy")
    V = np.zeros((L, L))
    for k in range(nwells):
        r2 = (gx - cx[k]) ** 2 + (gy - cy[k]) ** 2
        V -= d[k] * np.exp(-r2 / (2.0 * w[k] ** 2))
    return V            # V[j, i] for site i + L*j


def wells_2d(L=256, seed=0, nwells=8):
    """-Laplacian (5-point Dirichlet) + Gaussian-well potential."""
    V = wells_potential(L, seed, nwells)
    return laplacian_2d(L, diag=V.reshape(-1)), V


def batched_sizes(count=4096, seed=777, lo=48, hi=256):
    """Grid sizes L uniform in [lo, hi]."""
    u = uniform01(seed, np.arange(count, dtype=np.uint64))
    return (lo + np.floor(u * (hi - lo + 1))).astype(np.int64)


def batched_laplacian(L, seed):
    """L x L Laplacian plus a uniform[0, 2] diagonal potential."""
    diag = 2.0 * uniform01(seed, np.arange(L * L, dtype=np.uint64))
    return laplacian_2d(L, diag=diag)

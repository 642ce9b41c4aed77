// Rayleigh-Ritz start vector from a predicted subspace (trlx_seed_start).
//
// Y (n x k, FP32, [site][vector]) -> Q (FP64, column-major) -> G = Q^T Q,
// AQ = A Q (k operator applications), H = Q^T A Q, M = (AQ)^T AQ.  On the
// host: G = W L W^T, B = W_r L_r^{-1/2} over the eigen-directions of G that
// are not numerically zero, B^T H B = Z Theta Z^T.  The Ritz vectors are
// x_i = Q B z_i (orthonormal), their residual norms follow from
// |A x_i - theta_i x_i|^2 = (Bz_i)^T M (Bz_i) - theta_i^2, and the start
// vector is sum_i x_i: every Ritz direction of the predicted subspace with
// equal weight (each x_i signed so that its largest coefficient over the
// columns of Q is positive).  The thick-restart solver takes it through its ordinary
// start-vector channel (trl_set_iguess with guess = 1), so the Lanczos
// recurrence and the convergence test are exactly those of a plain solve.
// With project = 0 the start vector is the sum of the normalised columns of
// Y and the operator is not applied.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../../include/trlx.h"
#include "../host/dense.h"
#include "spmv.h"

namespace {

constexpr int kMaxK = 32;
constexpr int kTileRows = 32;

__global__ void k_gather_cols(const float *__restrict__ Y, long n, int k, double *__restrict__ Q) {
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n * k; i += stride) {
        const long r = i / k;
        const int c = (int)(i % k);
        Q[(long)c * n + r] = (double)Y[i];
    }
}

// part[b][i * k + j] = sum over the rows of block b of X[r, i] * Z[r, j]
// (X, Z column-major with leading dimension n).
__global__ void __launch_bounds__(256) k_xtz(const double *__restrict__ X, const double *__restrict__ Z, long n, int k,
                                              long chunk, double *part) {
    __shared__ double xs[kTileRows][kMaxK + 1], zs[kTileRows][kMaxK + 1];
    const long r0 = (long)blockIdx.x * chunk, r1 = min(n, r0 + chunk);
    const int kk = k * k;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long t0 = r0; t0 < r1; t0 += kTileRows) {
        for (int e = threadIdx.x; e < kTileRows * k; e += blockDim.x) {
            const int c = e / kTileRows, rr = e % kTileRows;
            const long r = t0 + rr;
            xs[rr][c] = r < r1 ? X[(long)c * n + r] : 0.0;
            zs[rr][c] = r < r1 ? Z[(long)c * n + r] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int p = threadIdx.x + 256 * s;
            if (p < kk) {
                const int i = p / k, j = p % k;
                double a = acc[s];
                for (int rr = 0; rr < kTileRows; ++rr) a += xs[rr][i] * zs[rr][j];
                acc[s] = a;
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int p = threadIdx.x + 256 * s;
        if (p < kk) part[(long)blockIdx.x * kk + p] = acc[s];
    }
}

// out[p] = sum_b part[b][p] in block order.
__global__ void k_sum_parts(const double *part, int nb, int len, double *out) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < len; p += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += part[(long)b * len + p];
        out[p] = s;
    }
}

// out[r] = sum_c Q[c * n + r] * coef[c]
__global__ void k_combine(const double *__restrict__ Q, long n, int k, const double *__restrict__ coef, double *out) {
    __shared__ double cs[kMaxK];
    if (threadIdx.x < k) cs[threadIdx.x] = coef[threadIdx.x];
    __syncthreads();
    const long stride = (long)gridDim.x * blockDim.x;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += stride) {
        double s = 0.0;
        for (int c = 0; c < k; ++c) s += Q[(long)c * n + r] * cs[c];
        out[r] = s;
    }
}

struct SeedWork {
    long n = 0;
    int k = 0;
    double *Q = nullptr, *AQ = nullptr, *part = nullptr, *gram = nullptr, *coef = nullptr, *start = nullptr;
    float *Y = nullptr;
    int nb = 0;
    ~SeedWork() { release(); }
    void release() {
        cudaFree(Q);
        cudaFree(AQ);
        cudaFree(part);
        cudaFree(gram);
        cudaFree(coef);
        cudaFree(start);
        cudaFree(Y);
        Q = AQ = part = gram = coef = start = nullptr;
        Y = nullptr;
        n = 0;
        k = 0;
    }
    bool ensure(long n_, int k_) {
        if (n_ == n && k_ <= k) return true;
        release();
        nb = (int)std::max<long>(1, std::min<long>(296, (n_ + 1023) / 1024));
        bool ok = cudaMalloc(&Q, sizeof(double) * n_ * k_) == cudaSuccess &&
                  cudaMalloc(&AQ, sizeof(double) * n_ * k_) == cudaSuccess &&
                  cudaMalloc(&part, sizeof(double) * nb * k_ * k_) == cudaSuccess &&
                  cudaMalloc(&gram, sizeof(double) * 3 * k_ * k_) == cudaSuccess &&
                  cudaMalloc(&coef, sizeof(double) * kMaxK) == cudaSuccess &&
                  cudaMalloc(&start, sizeof(double) * n_) == cudaSuccess &&
                  cudaMalloc(&Y, sizeof(float) * n_ * k_) == cudaSuccess;
        if (!ok) {
            release();
            return false;
        }
        n = n_;
        k = k_;
        return true;
    }
};

thread_local SeedWork g_work;

bool is_device(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// start = sum_i y_i / |y_i| over the columns that are not zero (no
// operator applications).
int normalized_sum(SeedWork &w, long n, int k, const double *gram, double *start, double *theta, double *res) {
    std::vector<double> coef(k, 0.0);
    double gmax = 0.0;
    for (int i = 0; i < k; ++i) gmax = std::max(gmax, gram[i * k + i]);
    if (!(gmax > 0.0)) return -234;
    int r = 0;
    for (int i = 0; i < k; ++i) {
        const double g = gram[i * k + i];
        if (g > 1e-24 * gmax) {
            coef[i] = 1.0 / std::sqrt(g);
            ++r;
        }
        if (theta) theta[i] = 0.0;
        if (res) res[i] = -1.0;
    }
    if (cudaMemcpy(w.coef, coef.data(), sizeof(double) * k, cudaMemcpyHostToDevice) != cudaSuccess) return -1001;
    double *out = is_device(start) ? start : w.start;
    k_combine<<<(int)std::min<long>(148 * 8, (n + 255) / 256), 256>>>(w.Q, n, k, w.coef, out);
    if (out != start && cudaMemcpy(start, out, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1001;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1001;
    return r;
}

}  // namespace

extern "C" int trlx_seed_start(void *op, int nrow, int k, const float *Y, int project, double *start, double *theta,
                               double *res) {
    auto *A = static_cast<trlx_operator *>(op);
    if (!A || !Y || !start || k < 1 || k > kMaxK || nrow < k || A->nrow != nrow || trlb::op_complex(A)) return -1;
    SeedWork &w = g_work;
    if (!w.ensure(nrow, k)) return -5;
    const long n = nrow;
    const float *Yd = Y;
    if (!is_device(Y)) {
        if (cudaMemcpy(w.Y, Y, sizeof(float) * n * k, cudaMemcpyHostToDevice) != cudaSuccess) return -1001;
        Yd = w.Y;
    }
    const int eb = (int)std::min<long>(148 * 8, (n * k + 255) / 256);
    k_gather_cols<<<eb, 256>>>(Yd, n, k, w.Q);
    if (project)
        for (int c = 0; c < k; ++c) trlb::spmv_plain(A, w.Q + (long)c * n, w.AQ + (long)c * n, 0);
    const long chunk = (n + w.nb - 1) / w.nb;
    const int kk = k * k;
    const double *pairs[3][2] = {{w.Q, w.Q}, {w.Q, w.AQ}, {w.AQ, w.AQ}};
    for (int m = 0; m < (project ? 3 : 1); ++m) {
        k_xtz<<<w.nb, 256>>>(pairs[m][0], pairs[m][1], n, k, chunk, w.part);
        k_sum_parts<<<(kk + 255) / 256, 256>>>(w.part, w.nb, kk, w.gram + (long)m * kk);
    }
    std::vector<double> h(3 * kk);
    if (cudaMemcpy(h.data(), w.gram, sizeof(double) * (project ? 3 : 1) * kk, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1001;
    if (!project) return normalized_sum(w, n, k, h.data(), start, theta, res);
    // Row-major part[i*k+j] = X_i . Z_j; the Gram matrices are symmetric in
    // exact arithmetic: symmetrise G and H.
    std::vector<double> G(kk), H(kk), M(kk);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
            G[i + j * k] = 0.5 * (h[i * k + j] + h[j * k + i]);
            H[i + j * k] = 0.5 * (h[kk + i * k + j] + h[kk + j * k + i]);
            M[i + j * k] = 0.5 * (h[2 * kk + i * k + j] + h[2 * kk + j * k + i]);
        }
    std::vector<double> lam(k);
    if (trlb::sym_eig(k, G.data(), k, lam.data())) return -234;
    const double lmax = lam[k - 1];
    if (!(lmax > 0.0)) return -234;
    std::vector<int> keep;
    for (int i = 0; i < k; ++i)
        if (lam[i] > 1e-12 * lmax) keep.push_back(i);
    const int r = (int)keep.size();
    std::vector<double> B((size_t)k * r);  // k x r
    for (int c = 0; c < r; ++c)
        for (int i = 0; i < k; ++i) B[i + c * k] = G[i + keep[c] * k] / std::sqrt(lam[keep[c]]);
    std::vector<double> HB((size_t)k * r), P((size_t)r * r);
    for (int c = 0; c < r; ++c)
        for (int i = 0; i < k; ++i) {
            double s = 0.0;
            for (int j = 0; j < k; ++j) s += H[i + j * k] * B[j + c * k];
            HB[i + c * k] = s;
        }
    for (int a = 0; a < r; ++a)
        for (int c = 0; c < r; ++c) {
            double s = 0.0;
            for (int i = 0; i < k; ++i) s += B[i + a * k] * HB[i + c * k];
            P[a + c * r] = s;
        }
    for (int a = 0; a < r; ++a)
        for (int c = 0; c < a; ++c) P[a + c * r] = P[c + a * r] = 0.5 * (P[a + c * r] + P[c + a * r]);
    std::vector<double> th(r);
    if (trlb::sym_eig(r, P.data(), r, th.data())) return -234;
    // X = Q (B Z): coefficient columns BZ (k x r); start = Q * (BZ * 1).
    // Each Ritz vector's sign is fixed so that its coefficient of largest
    // magnitude is positive (the start vector does not depend on the signs
    // the eigen-solver happens to return).
    std::vector<double> BZ((size_t)k * r), coef(k, 0.0);
    for (int c = 0; c < r; ++c) {
        int imax = 0;
        for (int i = 0; i < k; ++i) {
            double s = 0.0;
            for (int a = 0; a < r; ++a) s += B[i + a * k] * P[a + c * r];
            BZ[i + c * k] = s;
            if (std::fabs(s) > std::fabs(BZ[imax + c * k])) imax = i;
        }
        const double sg = BZ[imax + c * k] < 0.0 ? -1.0 : 1.0;
        for (int i = 0; i < k; ++i) {
            BZ[i + c * k] *= sg;
            coef[i] += BZ[i + c * k];
        }
    }
    for (int c = 0; c < k; ++c) {
        if (theta) theta[c] = c < r ? th[c] : 0.0;
        if (res) {
            if (c < r) {
                double s = 0.0;
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j) s += BZ[i + c * k] * M[i + j * k] * BZ[j + c * k];
                res[c] = std::sqrt(std::max(0.0, s - th[c] * th[c]));
            } else {
                res[c] = -1.0;
            }
        }
    }
    if (cudaMemcpy(w.coef, coef.data(), sizeof(double) * k, cudaMemcpyHostToDevice) != cudaSuccess) return -1001;
    double *out = is_device(start) ? start : w.start;
    k_combine<<<(int)std::min<long>(148 * 8, (n + 255) / 256), 256>>>(w.Q, n, k, w.coef, out);
    if (out != start &&
        cudaMemcpy(start, out, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -1001;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1001;
    return r;
}

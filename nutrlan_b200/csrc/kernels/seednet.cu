// Seed network: a 5-layer convolutional network that maps a potential V
// (H x W, FP32) to 16 vectors spanning an approximation of the lowest
// eigenvectors of -Laplacian + V; used to seed the thick-restart solve.
//
// Layers: 3x3 convolutions with dilations {1, 2, 4, 8, 1}, channels
// 1 -> 32 -> 32 -> 32 -> 32 -> 16, ReLU after the first four; "same" zero
// padding.  Activations are NHWC BF16 with 32 channels (the 1-channel input
// and the 16-channel output are zero-padded to 32), weights BF16, every
// product accumulated in FP32 on the tensor cores (mma.sync m16n8k16
// bf16 -> f32), FP32 master weights updated by Adam.
//
// Kernels (all written for this project):
//   k_conv      forward / backward-data implicit-GEMM convolution
//               (pixels x 288 taps*channels x 32 output channels),
//   k_conv_wgrad weight and bias gradients (288 x 32 per tap, summed over
//               pixels; per-block partials reduced in a fixed order),
//   k_loss_*    subspace loss against the true eigenvectors and its
//               gradient with respect to the network output,
//   k_adam      optimizer step and BF16 weight packing.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../../include/trlx.h"

namespace trlb {
namespace seednet {

constexpr int kC = 32;          // channels of every activation tensor
constexpr int kTaps = 9;
constexpr int kLayers = 5;
constexpr int kOut = 16;        // output vectors
constexpr int kDil[kLayers] = {1, 2, 4, 8, 1};
constexpr int kCin[kLayers] = {1, 32, 32, 32, 32};
constexpr int kCout[kLayers] = {32, 32, 32, 32, 16};

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

// ---------------------------------------------------------------------------
// Shared-memory staging and fragment loads.
constexpr int kTX = 64;      // pixels of one image row per tile
constexpr int kMaxDil = 8;   // largest dilation (halo of a tile)
constexpr int kRowB = 80;    // bytes per staged pixel: 32 channels + 16 B pad (ldmatrix rows hit distinct banks)
constexpr int kRowH = kRowB / 2;

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int sz = valid ? 16 : 0;  // 0: zero-fill, nothing read
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void *p) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}
__device__ __forceinline__ void ldsm_x4_trans(unsigned (&r)[4], const void *p) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// Stages the three input rows y - d, y, y + d of sample b, columns
// x0 - d .. x0 + kTX - 1 + d (zero outside the image), as [row][col][40]
// bf16.  `nth` threads cooperate.
__device__ __forceinline__ void stage_rows(__nv_bfloat16 *xs, const __nv_bfloat16 *in, int b, int y, int x0, int H,
                                           int W, int d, int tid, int nth) {
    const int wid = kTX + 2 * d;
    const int chunks = 3 * wid * 4;
    for (int c = tid; c < chunks; c += nth) {
        const int r = c / (wid * 4), rem = c - r * wid * 4, col = rem >> 2, q = rem & 3;
        const int yy = y + (r - 1) * d, xx = x0 - d + col;
        const bool ok = yy >= 0 && yy < H && xx >= 0 && xx < W;
        const __nv_bfloat16 *src = ok ? in + ((((long)b * H + yy) * W + xx) * kC + q * 8) : in;
        cp_async16(xs + ((size_t)r * wid + col) * kRowH + q * 8, src, ok);
    }
}

// ---------------------------------------------------------------------------
// out[p, co] = act( sum_{tap, ci} in[p + d*off(tap), ci] * w[tap][co][ci] + bias[co] )
// in: NHWC bf16 (32 ch), w: [tap][co][ci] bf16, out: NHWC bf16 (32 ch) or,
// when out_f32 != null, FP32 [pixel][16] (first 16 channels).
// A block computes one tile of kTX pixels of one image row for all 32
// output channels: the three input rows the taps touch (with a halo of d
// pixels) and all weights are staged in shared memory with cp.async, then
// each of the 4 warps runs 9 taps x 2 k16 steps x 4 n8 tiles of
// mma.sync m16n8k16 (bf16 -> f32) on fragments loaded with ldmatrix.
__global__ void __launch_bounds__(128)
    k_conv(const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ w, const float *__restrict__ bias,
           __nv_bfloat16 *out, float *out_f32, int B, int H, int W, int dil, int relu) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __nv_bfloat16 *ws = reinterpret_cast<__nv_bfloat16 *>(smem_raw);  // [9][32 co][40]
    __nv_bfloat16 *xs = ws + kTaps * kC * kRowH;                         // [3][kTX + 2d][40]
    const int tilesx = W / kTX;
    const long tile = blockIdx.x;
    const int xt = (int)(tile % tilesx);
    const long by = tile / tilesx;
    const int y = (int)(by % H), b = (int)(by / H);
    const int x0 = xt * kTX;
    for (int c = threadIdx.x; c < kTaps * kC * 4; c += blockDim.x)
        cp_async16(ws + (size_t)(c >> 2) * kRowH + (c & 3) * 8, w + (size_t)(c >> 2) * kC + (c & 3) * 8, true);
    stage_rows(xs, in, b, y, x0, H, W, dil, threadIdx.x, blockDim.x);
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wid = kTX + 2 * dil;
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    // ldmatrix lane roles: A rows (pixels) lane&7 (+8 for lanes 8-15 / 24-31),
    // k half lane>>4; B rows (output channels) lane&7 of n-tile pair
    // member lane>>4, k half (lane>>3)&1.
    const int a_row = (lane & 7) + ((lane >> 3) & 1) * 8, a_k = (lane >> 4) * 8;
    const int b_row = (lane & 7) + (lane >> 4) * 8, b_k = ((lane >> 3) & 1) * 8;
#pragma unroll 1
    for (int tap = 0; tap < kTaps; ++tap) {
        const int r = tap / 3, dx = (tap % 3 - 1) * dil;
        const __nv_bfloat16 *xrow = xs + ((size_t)r * wid + dil + dx + warp * 16 + a_row) * kRowH + a_k;
        const __nv_bfloat16 *wt = ws + (size_t)tap * kC * kRowH;
#pragma unroll
        for (int k0 = 0; k0 < kC; k0 += 16) {
            unsigned a[4];
            ldsm_x4(a, xrow + k0);
#pragma unroll
            for (int jp = 0; jp < 2; ++jp) {
                unsigned bb[4];
                ldsm_x4(bb, wt + (size_t)(jp * 16 + b_row) * kRowH + k0 + b_k);
                const unsigned b0[2] = {bb[0], bb[1]}, b1[2] = {bb[2], bb[3]};
                mma_bf16(acc[2 * jp], a, b0);
                mma_bf16(acc[2 * jp + 1], a, b1);
            }
        }
    }
    const long pa = (by * W) + x0 + warp * 16 + g, pb = pa + 8;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int co = j * 8 + 2 * t;
        const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
        float v0 = acc[j][0] + b0, v1 = acc[j][1] + b1, v2 = acc[j][2] + b0, v3 = acc[j][3] + b1;
        if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
            v2 = fmaxf(v2, 0.f);
            v3 = fmaxf(v3, 0.f);
        }
        if (out_f32) {
            if (co < kOut) {
                *reinterpret_cast<float2 *>(out_f32 + pa * kOut + co) = make_float2(v0, v1);
                *reinterpret_cast<float2 *>(out_f32 + pb * kOut + co) = make_float2(v2, v3);
            }
        } else {
            reinterpret_cast<unsigned *>(out)[pa * (kC / 2) + co / 2] = pack_bf16(v0, v1);
            reinterpret_cast<unsigned *>(out)[pb * (kC / 2) + co / 2] = pack_bf16(v2, v3);
        }
    }
}

// tcgen05 convolution (kernels/seednet_tc.cu).
bool conv_tc(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias, __nv_bfloat16 *out, float *out_f32,
             int B, int H, int W, int dil, int relu);
int conv_tc_status();
// tcgen05 weight gradient: blocks whose partials it wrote, or 0.
int wgrad_tc(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *part, int max_blocks, int B, int H, int W,
             int dil);

size_t conv_smem_bytes(int dil) {
    return (size_t)kTaps * kC * kRowB + (size_t)3 * (kTX + 2 * dil) * kRowB;
}

// g_pre = g_post * [act > 0] (ReLU backward), NHWC bf16, elementwise.
__global__ void k_relu_mask(__nv_bfloat16 *g, const __nv_bfloat16 *act, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        if (!(__bfloat162float(act[i]) > 0.f)) g[i] = __float2bfloat16(0.f);
}

// ---------------------------------------------------------------------------
// Weight gradient: dW[tap][ci][co] = sum_p in[p + d*off(tap), ci] * g[p, co];
// db[co] = sum_p g[p, co].  A block of 9 warps walks a range of row tiles
// (kTX pixels each); per tile the three input rows and the gradient tile are
// staged with cp.async, and warp w accumulates tap w as a (32 ci) x (32 co)
// product over the tile's pixels: A = staged input rows transposed (ldmatrix
// .trans), B = gradient tile (ldmatrix .trans).  Per-block partials
// part[b][tap][ci][co] (+ part[b][9][0][co] for the bias) are reduced in
// block order by k_reduce_parts.
constexpr int kWgWarps = kTaps;

__global__ void __launch_bounds__(kWgWarps * 32)
    k_conv_wgrad(const __nv_bfloat16 *__restrict__ in, const __nv_bfloat16 *__restrict__ g, float *part, int B, int H,
                 int W, int dil) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __nv_bfloat16 *gs = reinterpret_cast<__nv_bfloat16 *>(smem_raw);  // [kTX][40]
    __nv_bfloat16 *xs = gs + (size_t)kTX * kRowH;                       // [3][kTX + 2d][40]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gi = lane >> 2, t = lane & 3;
    const int tap = warp, r = tap / 3, dx = (tap % 3 - 1) * dil;
    const int wid = kTX + 2 * dil;
    const int tilesx = W / kTX;
    const long ntiles = (long)B * H * tilesx;
    float acc[2][4][4];
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[mi][j][q] = 0.f;
    float bsum = 0.f;
    // A (ci x px) from xs rows (px-major): matrices (px lo, ci lo), (px lo,
    // ci hi), (px hi, ci lo), (px hi, ci hi) -> a0..a3.
    const int a_px = (lane & 7) + (lane >> 4) * 8, a_ci = ((lane >> 3) & 1) * 8;
    // B (px x co) from gs: matrices (px lo, co n), (px hi, co n), (px lo,
    // co n+8), (px hi, co n+8).
    const int b_px = (lane & 7) + ((lane >> 3) & 1) * 8, b_co = (lane >> 4) * 8;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int xt = (int)(tile % tilesx);
        const long by = tile / tilesx;
        const int y = (int)(by % H), b = (int)(by / H);
        const int x0 = xt * kTX;
        const __nv_bfloat16 *gsrc = g + ((by * W) + x0) * kC;
        for (int c = threadIdx.x; c < kTX * 4; c += blockDim.x)
            cp_async16(gs + (size_t)(c >> 2) * kRowH + (c & 3) * 8, gsrc + (size_t)(c >> 2) * kC + (c & 3) * 8, true);
        stage_rows(xs, in, b, y, x0, H, W, dil, threadIdx.x, blockDim.x);
        cp_async_wait_all();
        __syncthreads();
        if (warp == 0) {
            float s = 0.f;
            for (int p = 0; p < kTX; ++p) s += __bfloat162float(gs[(size_t)p * kRowH + lane]);
            bsum += s;
        }
        const __nv_bfloat16 *xrow = xs + ((size_t)r * wid + dil + dx) * kRowH;
#pragma unroll
        for (int k0 = 0; k0 < kTX; k0 += 16) {
            unsigned a[2][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi) ldsm_x4_trans(a[mi], xrow + (size_t)(k0 + a_px) * kRowH + mi * 16 + a_ci);
#pragma unroll
            for (int jp = 0; jp < 2; ++jp) {
                unsigned bb[4];
                ldsm_x4_trans(bb, gs + (size_t)(k0 + b_px) * kRowH + jp * 16 + b_co);
                const unsigned b0[2] = {bb[0], bb[1]}, b1[2] = {bb[2], bb[3]};
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    mma_bf16(acc[mi][2 * jp], a[mi], b0);
                    mma_bf16(acc[mi][2 * jp + 1], a[mi], b1);
                }
            }
        }
        __syncthreads();
    }
    float *pb = part + (size_t)blockIdx.x * (kTaps + 1) * kC * kC;
    float *o = pb + (size_t)tap * kC * kC;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int ci0 = mi * 16 + gi, co = j * 8 + 2 * t;
            o[ci0 * kC + co] = acc[mi][j][0];
            o[ci0 * kC + co + 1] = acc[mi][j][1];
            o[(ci0 + 8) * kC + co] = acc[mi][j][2];
            o[(ci0 + 8) * kC + co + 1] = acc[mi][j][3];
        }
    if (warp == 0) pb[(size_t)kTaps * kC * kC + lane] = bsum;
}

size_t wgrad_smem_bytes(int dil) { return (size_t)kTX * kRowB + (size_t)3 * (kTX + 2 * dil) * kRowB; }

// Sum partials over blocks in order: grad[i] = sum_b part[b][i].
__global__ void k_reduce_parts(const float *part, int nb, int stride, int len, float *grad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nb; ++b) s += part[(size_t)b * stride + i];
        grad[i] = s;
    }
}

// ---------------------------------------------------------------------------
// Loss.  Y: FP32 [pixel][16] network output, U: FP32 [pixel][16] true
// eigenvectors (orthonormal columns per sample).  Per sample b:
//   C = U^T Y, G = Y^T Y (16 x 16), n_k^2 = G_kk,
//   L = sum_k (1 - |C[:,k]|^2 / n_k^2) + lam sum_{j != k} G_jk^2 / (n_j^2 n_k^2)
// (the output columns lie in span(U) and are mutually orthogonal).
// dL/dY = U A + Y Bm with A_jk = -2 C_jk / n_k^2,
//   Bm_jk = 4 lam G_jk / (n_j^2 n_k^2) (j != k),
//   Bm_kk = 2 |C[:,k]|^2 / n_k^4 - 4 lam sum_{j != k} G_jk^2 / (n_j^2 n_k^4).
constexpr int kLossPix = 1024;

__global__ void __launch_bounds__(256) k_loss_stats(const float *Y, const float *U, int HW, float *part) {
    // Block (c, b): pixels [c*kLossPix, ...) of sample b; thread t owns entry
    // (t / 16, t % 16) of C and of G.
    const int b = blockIdx.y;
    const long base = (long)b * HW;
    const int i = threadIdx.x >> 4, k = threadIdx.x & 15;
    float c = 0.f, gsum = 0.f;
    const int p0 = blockIdx.x * kLossPix, p1 = min(HW, p0 + kLossPix);
    for (int p = p0; p < p1; ++p) {
        const float yk = Y[(base + p) * kOut + k];
        c += U[(base + p) * kOut + i] * yk;
        gsum += Y[(base + p) * kOut + i] * yk;
    }
    float *o = part + ((size_t)b * gridDim.x + blockIdx.x) * 512;
    o[threadIdx.x] = c;
    o[256 + threadIdx.x] = gsum;
}

__global__ void k_loss_coeffs(const float *part, int nchunks, float lam, float *coef, float *loss) {
    // One block per sample, 256 threads: reduce C, G; then thread 0 builds
    // A and Bm (coef[b][0..256) = A, [256..512) = Bm) and the loss.
    const int b = blockIdx.x;
    __shared__ float C[256], G[256];
    float c = 0.f, gsum = 0.f;
    for (int ch = 0; ch < nchunks; ++ch) {
        const float *o = part + ((size_t)b * nchunks + ch) * 512;
        c += o[threadIdx.x];
        gsum += o[256 + threadIdx.x];
    }
    C[threadIdx.x] = c;  // C[i*16 + k] = (U^T Y)_ik
    G[threadIdx.x] = gsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float n2[16], cc[16];
        for (int k = 0; k < 16; ++k) {
            n2[k] = fmaxf(G[k * 16 + k], 1e-30f);
            float s = 0.f;
            for (int i = 0; i < 16; ++i) s += C[i * 16 + k] * C[i * 16 + k];
            cc[k] = s;
        }
        float L = 0.f;
        float *A = coef + (size_t)b * 512, *Bm = A + 256;
        for (int k = 0; k < 16; ++k) {
            L += 1.f - cc[k] / n2[k];
            float diag = 2.f * cc[k] / (n2[k] * n2[k]);
            for (int j = 0; j < 16; ++j) {
                A[j * 16 + k] = -2.f * C[j * 16 + k] / n2[k];
                if (j != k) {
                    const float s = G[j * 16 + k] * G[j * 16 + k] / (n2[j] * n2[k]);
                    L += lam * s;
                    Bm[j * 16 + k] = 4.f * lam * G[j * 16 + k] / (n2[j] * n2[k]);
                    diag -= 4.f * lam * s / n2[k];
                }
            }
            Bm[k * 16 + k] = diag;
        }
        loss[b] = L;
    }
}

// dY[p, k] = sum_j U[p, j] A_jk + Y[p, j] Bm_jk, written as NHWC bf16 with
// 32 channels (16..31 zero) for the backward pass of the last layer.
__global__ void k_loss_grad(const float *Y, const float *U, const float *coef, int HW, long P, float scale,
                            __nv_bfloat16 *dY) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long)gridDim.x * blockDim.x) {
        const int b = (int)(p / HW);
        const float *A = coef + (size_t)b * 512, *Bm = A + 256;
        float u[16], y[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            u[j] = U[p * kOut + j];
            y[j] = Y[p * kOut + j];
        }
        for (int k = 0; k < 16; k += 2) {
            float s0 = 0.f, s1 = 0.f;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                s0 += u[j] * A[j * 16 + k] + y[j] * Bm[j * 16 + k];
                s1 += u[j] * A[j * 16 + k + 1] + y[j] * Bm[j * 16 + k + 1];
            }
            reinterpret_cast<unsigned *>(dY)[p * (kC / 2) + k / 2] = pack_bf16(scale * s0, scale * s1);
        }
        for (int k = 16; k < kC; k += 2) reinterpret_cast<unsigned *>(dY)[p * (kC / 2) + k / 2] = 0u;
    }
}

// ---------------------------------------------------------------------------
// Adam on the FP32 master weights (layout [tap][ci][co] per layer, zero
// outside the layer's real channels) and packing of the BF16 copies:
// forward [tap][co][ci] and backward-data [tap'][ci][co] with tap' = 8 - tap.
__global__ void k_adam(float *w, const float *gw, float *m, float *v, int len, float lr, float b1, float b2,
                       float eps, float bc1, float bc2, const unsigned char *mask) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
        if (mask && !mask[i]) continue;
        const float gr = gw[i];
        const float mi = b1 * m[i] + (1.f - b1) * gr;
        const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

__global__ void k_pack(const float *w, __nv_bfloat16 *wf, __nv_bfloat16 *wb) {
    // w: [tap][ci][co] FP32 -> wf[tap][co][ci], wb[8 - tap][ci][co]
    // (backward data: input channels co, output channels ci).
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kTaps * kC * kC; i += gridDim.x * blockDim.x) {
        const int tap = i / (kC * kC), ci = (i / kC) % kC, co = i % kC;
        const __nv_bfloat16 v = __float2bfloat16(w[i]);
        wf[(tap * kC + co) * kC + ci] = v;
        wb[((kTaps - 1 - tap) * kC + ci) * kC + co] = v;
    }
}

// Minimum of each sample's potential (one block per sample).
__global__ void __launch_bounds__(1024) k_sample_min(const float *V, int HW, float *vmin) {
    __shared__ float red[32];
    const float *v = V + (long)blockIdx.x * HW;
    float m = INFINITY;
    for (int i = threadIdx.x; i < HW; i += blockDim.x) m = fminf(m, v[i]);
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : INFINITY;
        for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) vmin[blockIdx.x] = m;
    }
}

// Input packing: (V - min V) * scale (FP32, per sample) into channel 0 of
// NHWC bf16.  Measuring the potential from its global minimum makes "the
// lowest states" a local property the convolutions can see.
__global__ void k_pack_input(const float *V, const float *vmin, int HW, long P, float scale, __nv_bfloat16 *x) {
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long)gridDim.x * blockDim.x) {
        unsigned *o = reinterpret_cast<unsigned *>(x) + p * (kC / 2);
        o[0] = pack_bf16((V[p] - vmin[p / HW]) * scale, 0.f);
        for (int k = 1; k < kC / 2; ++k) o[k] = 0u;
    }
}

}  // namespace seednet
}  // namespace trlb

// ===========================================================================
// Host API
// ===========================================================================
using namespace trlb::seednet;

struct trlx_seednet {
    int H = 0, W = 0, Bmax = 0;
    float in_scale = 1.f / 50.f;
    // per layer: FP32 master [tap][ci][co], Adam moments, BF16 packs, bias
    float *w[kLayers] = {}, *m[kLayers] = {}, *v[kLayers] = {}, *gw[kLayers] = {};
    float *bias[kLayers] = {}, *mb[kLayers] = {}, *vb[kLayers] = {}, *gb[kLayers] = {};
    unsigned char *mask[kLayers] = {};
    __nv_bfloat16 *wf[kLayers] = {}, *wb[kLayers] = {};
    // activations: act[0] = input, act[l+1] = output of layer l (hidden)
    __nv_bfloat16 *act[kLayers] = {};
    __nv_bfloat16 *g0 = nullptr, *g1 = nullptr;  // gradient ping-pong
    float *Y = nullptr;                           // network output [P][16]
    float *part = nullptr;
    size_t part_len = 0;
    float *coef = nullptr, *loss = nullptr, *Vd = nullptr, *Ud = nullptr, *vmin = nullptr;
    int step = 0;
};

namespace {

int blocks_for(long n, int t = 256) { return (int)std::min<long>((n + t - 1) / t, 148L * 16); }

// Weight-gradient grid: about two blocks per SM, each walking several tiles.
int wgrad_blocks(int B, int H, int W) {
    const long tiles = (long)B * H * (W / kTX);
    return (int)std::max<long>(1, std::min<long>(tiles, 148L * 2));
}

void pack_layer(trlx_seednet *net, int l) {
    k_pack<<<36, 256>>>(net->w[l], net->wf[l], net->wb[l]);
}

void pack_input(trlx_seednet *net, int B) {
    const int HW = net->H * net->W;
    k_sample_min<<<B, 1024>>>(net->Vd, HW, net->vmin);
    k_pack_input<<<blocks_for((long)B * HW), 256>>>(net->Vd, net->vmin, HW, (long)B * HW, net->in_scale, net->act[0]);
}

void conv(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias, __nv_bfloat16 *out, float *out_f32,
          int B, int H, int W, int dil, int relu) {
    // The tcgen05 kernel (kernels/seednet_tc.cu) where the shape allows;
    // TRLX_SEEDNET_CONV=mma keeps every layer on k_conv.
    if (conv_tc(in, w, bias, out, out_f32, B, H, W, dil, relu)) return;
    const size_t smem = conv_smem_bytes(dil);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)conv_smem_bytes(kMaxDil));
        cudaFuncSetAttribute(k_conv_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)wgrad_smem_bytes(kMaxDil));
        attr = true;
    }
    const int grid = B * H * (W / kTX);
    k_conv<<<grid, 128, smem>>>(in, w, bias, out, out_f32, B, H, W, dil, relu);
}

// Forward pass for B samples already packed in act[0]; output in net->Y.
void forward(trlx_seednet *net, int B) {
    for (int l = 0; l < kLayers; ++l) {
        const bool last = l == kLayers - 1;
        conv(net->act[l], net->wf[l], net->bias[l], last ? nullptr : net->act[l + 1], last ? net->Y : nullptr, B,
             net->H, net->W, kDil[l], last ? 0 : 1);
    }
}

}  // namespace

extern "C" {

int trlx_seednet_create(int H, int W, int max_batch, unsigned long long seed, trlx_seednet **out) {
    if (!out || H < 8 || W < 64 || W % 64 || max_batch < 1) return -1;
    auto *net = new trlx_seednet();
    net->H = H;
    net->W = W;
    net->Bmax = max_batch;
    const long P = (long)max_batch * H * W;
    const size_t wl = (size_t)kTaps * kC * kC;
    bool ok = true;
    auto alloc = [&](void **p, size_t bytes) {
        if (cudaMalloc(p, bytes) != cudaSuccess) ok = false;
        else cudaMemset(*p, 0, bytes);
    };
    for (int l = 0; l < kLayers; ++l) {
        alloc((void **)&net->w[l], wl * 4);
        alloc((void **)&net->m[l], wl * 4);
        alloc((void **)&net->v[l], wl * 4);
        alloc((void **)&net->gw[l], (wl + kC) * 4);
        alloc((void **)&net->bias[l], kC * 4);
        alloc((void **)&net->mb[l], kC * 4);
        alloc((void **)&net->vb[l], kC * 4);
        alloc((void **)&net->gb[l], kC * 4);
        alloc((void **)&net->mask[l], wl);
        alloc((void **)&net->wf[l], wl * 2);
        alloc((void **)&net->wb[l], wl * 2);
        alloc((void **)&net->act[l], (size_t)P * kC * 2);
        // He-style initialisation of the real channels (host RNG, splitmix).
        std::vector<float> hw(wl, 0.f);
        std::vector<unsigned char> hm(wl, 0);
        const float sd = std::sqrt(2.0f / (kTaps * kCin[l]));
        uint64_t s = seed + 0x9E3779B97F4A7C15ull * (l + 1);
        for (int tap = 0; tap < kTaps; ++tap)
            for (int ci = 0; ci < kCin[l]; ++ci)
                for (int co = 0; co < kCout[l]; ++co) {
                    // Box-Muller from two splitmix draws.
                    auto draw = [&]() {
                        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
                        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                        z ^= z >> 31;
                        return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
                    };
                    const double u1 = draw(), u2 = draw();
                    const size_t i = ((size_t)tap * kC + ci) * kC + co;
                    hw[i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
                    hm[i] = 1;
                }
        if (ok) {
            cudaMemcpy(net->w[l], hw.data(), wl * 4, cudaMemcpyHostToDevice);
            cudaMemcpy(net->mask[l], hm.data(), wl, cudaMemcpyHostToDevice);
        }
    }
    alloc((void **)&net->g0, (size_t)P * kC * 2);
    alloc((void **)&net->g1, (size_t)P * kC * 2);
    alloc((void **)&net->Y, (size_t)P * kOut * 4);
    const long nwg = wgrad_blocks(max_batch, H, W);
    net->part_len = std::max<size_t>((size_t)nwg * (kTaps + 1) * kC * kC, (size_t)max_batch * ((H * W + kLossPix - 1) / kLossPix) * 512);
    alloc((void **)&net->part, net->part_len * 4);
    alloc((void **)&net->coef, (size_t)max_batch * 512 * 4);
    alloc((void **)&net->loss, (size_t)max_batch * 4);
    alloc((void **)&net->Vd, (size_t)P * 4);
    alloc((void **)&net->vmin, (size_t)max_batch * 4);
    alloc((void **)&net->Ud, (size_t)P * kOut * 4);
    if (!ok) {
        trlx_seednet_destroy(net);
        return -5;
    }
    for (int l = 0; l < kLayers; ++l) pack_layer(net, l);
    cudaDeviceSynchronize();
    *out = net;
    return 0;
}

void trlx_seednet_destroy(trlx_seednet *net) {
    if (!net) return;
    for (int l = 0; l < kLayers; ++l) {
        cudaFree(net->w[l]);
        cudaFree(net->m[l]);
        cudaFree(net->v[l]);
        cudaFree(net->gw[l]);
        cudaFree(net->bias[l]);
        cudaFree(net->mb[l]);
        cudaFree(net->vb[l]);
        cudaFree(net->gb[l]);
        cudaFree(net->mask[l]);
        cudaFree(net->wf[l]);
        cudaFree(net->wb[l]);
        cudaFree(net->act[l]);
    }
    cudaFree(net->g0);
    cudaFree(net->g1);
    cudaFree(net->Y);
    cudaFree(net->part);
    cudaFree(net->coef);
    cudaFree(net->loss);
    cudaFree(net->Vd);
    cudaFree(net->vmin);
    cudaFree(net->Ud);
    delete net;
}

// V: B potentials (H*W FP32 each, host or device).  out: B * H*W * 16 FP32
// ([sample][pixel][vector], host or device).
int trlx_seednet_forward(trlx_seednet *net, int B, const float *V, float *out) {
    if (!net || B < 1 || B > net->Bmax || !V) return -1;
    const long P = (long)B * net->H * net->W;
    if (cudaMemcpy(net->Vd, V, P * 4, cudaMemcpyDefault) != cudaSuccess) return -1001;
    pack_input(net, B);
    forward(net, B);
    if (out && cudaMemcpy(out, net->Y, P * kOut * 4, cudaMemcpyDefault) != cudaSuccess) return -1001;
    if (cudaDeviceSynchronize() != cudaSuccess) return -1001;
    return conv_tc_status();
}

// Loss and gradients of a batch (no update); loss_out[b] per sample,
// grads (optional, host or device): per layer [tap][ci][co] then bias (32),
// concatenated: 5 * (9*32*32 + 32) floats.
static int loss_and_grad(trlx_seednet *net, int B, const float *V, const float *U, float lam, float *loss_out) {
    const int H = net->H, W = net->W, HW = H * W;
    const long P = (long)B * HW;
    if (cudaMemcpy(net->Vd, V, P * 4, cudaMemcpyDefault) != cudaSuccess) return -1001;
    if (cudaMemcpy(net->Ud, U, P * kOut * 4, cudaMemcpyDefault) != cudaSuccess) return -1001;
    pack_input(net, B);
    forward(net, B);
    const int nch = (HW + kLossPix - 1) / kLossPix;
    k_loss_stats<<<dim3(nch, B), 256>>>(net->Y, net->Ud, HW, net->part);
    k_loss_coeffs<<<B, 256>>>(net->part, nch, lam, net->coef, net->loss);
    k_loss_grad<<<blocks_for(P), 256>>>(net->Y, net->Ud, net->coef, HW, P, 1.0f / B, net->g0);
    // Backward through the layers.
    const int nwg = wgrad_blocks(B, H, W);
    __nv_bfloat16 *g = net->g0, *gn = net->g1;
    for (int l = kLayers - 1; l >= 0; --l) {
        if (l < kLayers - 1) k_relu_mask<<<blocks_for(P * kC), 256>>>(g, net->act[l + 1], P * kC);
        // tcgen05 kernel where W allows (TRLX_SEEDNET_CONV=mma: mma.sync).
        int nb = wgrad_tc(net->act[l], g, net->part, (int)(net->part_len / ((size_t)(kTaps + 1) * kC * kC)), B, H,
                          W, kDil[l]);
        if (nb == 0) {
            k_conv_wgrad<<<nwg, kWgWarps * 32, wgrad_smem_bytes(kDil[l])>>>(net->act[l], g, net->part, B, H, W,
                                                                              kDil[l]);
            nb = nwg;
        }
        // Partials have stride (kTaps + 1) * kC * kC; only the weight taps and
        // the kC bias entries after them are written and reduced.
        const int len = kTaps * kC * kC + kC;
        k_reduce_parts<<<(len + 255) / 256, 256>>>(net->part, nb, (kTaps + 1) * kC * kC, len, net->gw[l]);
        cudaMemcpyAsync(net->gb[l], net->gw[l] + (size_t)kTaps * kC * kC, kC * 4, cudaMemcpyDeviceToDevice);
        if (l > 0) {
            conv(g, net->wb[l], nullptr, gn, nullptr, B, H, W, kDil[l], 0);
            std::swap(g, gn);
        }
    }
    if (loss_out) cudaMemcpy(loss_out, net->loss, B * 4, cudaMemcpyDeviceToHost);
    if (cudaDeviceSynchronize() != cudaSuccess) return -1001;
    return conv_tc_status();
}

int trlx_seednet_gradients(trlx_seednet *net, int B, const float *V, const float *U, float lam, float *loss_out,
                           float *grads) {
    if (!net || B < 1 || B > net->Bmax || !V || !U) return -1;
    int rc = loss_and_grad(net, B, V, U, lam, loss_out);
    if (rc || !grads) return rc;
    const size_t wl = (size_t)kTaps * kC * kC;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        cudaMemcpy(grads + off, net->gw[l], wl * 4, cudaMemcpyDefault);
        off += wl;
        cudaMemcpy(grads + off, net->gb[l], kC * 4, cudaMemcpyDefault);
        off += kC;
    }
    return 0;
}

int trlx_seednet_train_step(trlx_seednet *net, int B, const float *V, const float *U, float lam, float lr,
                            float *loss_out) {
    if (!net || B < 1 || B > net->Bmax || !V || !U) return -1;
    int rc = loss_and_grad(net, B, V, U, lam, loss_out);
    if (rc) return rc;
    net->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.f - std::pow(b1, (float)net->step), bc2 = 1.f - std::pow(b2, (float)net->step);
    const int wl = kTaps * kC * kC;
    for (int l = 0; l < kLayers; ++l) {
        k_adam<<<(wl + 255) / 256, 256>>>(net->w[l], net->gw[l], net->m[l], net->v[l], wl, lr, b1, b2, eps, bc1, bc2,
                                          net->mask[l]);
        k_adam<<<1, 32>>>(net->bias[l], net->gb[l], net->mb[l], net->vb[l], kCout[l], lr, b1, b2, eps, bc1, bc2,
                          nullptr);
        pack_layer(net, l);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1001;
}

// Weights (FP32) in/out: per layer [tap][ci][co] (9*32*32) then bias (32).
int trlx_seednet_get_weights(trlx_seednet *net, float *out) {
    if (!net || !out) return -1;
    const size_t wl = (size_t)kTaps * kC * kC;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        cudaMemcpy(out + off, net->w[l], wl * 4, cudaMemcpyDefault);
        off += wl;
        cudaMemcpy(out + off, net->bias[l], kC * 4, cudaMemcpyDefault);
        off += kC;
    }
    return 0;
}

int trlx_seednet_set_weights(trlx_seednet *net, const float *in) {
    if (!net || !in) return -1;
    const size_t wl = (size_t)kTaps * kC * kC;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        cudaMemcpy(net->w[l], in + off, wl * 4, cudaMemcpyDefault);
        off += wl;
        cudaMemcpy(net->bias[l], in + off, kC * 4, cudaMemcpyDefault);
        off += kC;
        pack_layer(net, l);
    }
    net->step = 0;
    for (int l = 0; l < kLayers; ++l) {
        cudaMemset(net->m[l], 0, wl * 4);
        cudaMemset(net->v[l], 0, wl * 4);
        cudaMemset(net->mb[l], 0, kC * 4);
        cudaMemset(net->vb[l], 0, kC * 4);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : -1001;
}

int trlx_seednet_num_params(void) { return kLayers * (kTaps * kC * kC + kC); }

}  // extern "C"

// Shared device helpers for the Lanczos kernels: a small complex type,
// per-storage-type vector loads/stores, and deterministic block/grid
// reductions (fixed summation order, so results do not depend on timing).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace trlb {

struct zd {  // complex double, layout-compatible with trl_dcomplex
    double x, y;
};
struct zf {  // complex float (basis storage only)
    float x, y;
};

__host__ __device__ inline zd zmake(double a, double b) { return zd{a, b}; }
__host__ __device__ inline zd operator+(zd a, zd b) { return zd{a.x + b.x, a.y + b.y}; }
__host__ __device__ inline zd operator-(zd a, zd b) { return zd{a.x - b.x, a.y - b.y}; }
__host__ __device__ inline zd operator*(double s, zd a) { return zd{s * a.x, s * a.y}; }
__host__ __device__ inline zd operator*(zd a, double s) { return zd{s * a.x, s * a.y}; }

// ---- compute-type helpers (double or zd) ------------------------------------
__device__ __forceinline__ double czero(double) { return 0.0; }
__device__ __forceinline__ zd czero(zd) { return zd{0.0, 0.0}; }
__device__ __forceinline__ double abs2(double a) { return a * a; }
__device__ __forceinline__ double real_part(double a) { return a; }
__device__ __forceinline__ double real_part(zd a) { return a.x; }
__device__ __forceinline__ double abs2(zd a) { return a.x * a.x + a.y * a.y; }
// acc += conj(v) * r
__device__ __forceinline__ void fma_conj(double &acc, double v, double r) { acc = fma(v, r, acc); }
__device__ __forceinline__ void fma_conj(zd &acc, zd v, zd r) {
    acc.x = fma(v.x, r.x, fma(v.y, r.y, acc.x));
    acc.y = fma(v.x, r.y, fma(-v.y, r.x, acc.y));
}
// acc -= v * h
__device__ __forceinline__ void fms(double &acc, double v, double h) { acc = fma(-v, h, acc); }
__device__ __forceinline__ void fms(zd &acc, zd v, zd h) {
    acc.x = fma(-v.x, h.x, fma(v.y, h.y, acc.x));
    acc.y = fma(-v.x, h.y, fma(-v.y, h.x, acc.y));
}
// acc += v * s (s real)
__device__ __forceinline__ void fma_real(double &acc, double v, double s) { acc = fma(v, s, acc); }
__device__ __forceinline__ void fma_real(zd &acc, zd v, double s) {
    acc.x = fma(v.x, s, acc.x);
    acc.y = fma(v.y, s, acc.y);
}
__device__ __forceinline__ double shfl_down(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
__device__ __forceinline__ zd shfl_down(zd v, int o) {
    return zd{__shfl_down_sync(0xffffffffu, v.x, o), __shfl_down_sync(0xffffffffu, v.y, o)};
}
__device__ __forceinline__ double ldcg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ zd ldcg(const zd *p) {
    double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    return zd{v.x, v.y};
}

// ---- storage traits: R consecutive elements per 16-byte load -----------------
template <class T>
struct Store;
template <>
struct Store<double> {
    using C = double;
    static constexpr int R = 2;
    __device__ __forceinline__ static void load(const double *p, C (&o)[R]) {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        o[0] = v.x;
        o[1] = v.y;
    }
    // The same 16 bytes from shared memory.
    __device__ __forceinline__ static void lds(const double *p, C (&o)[R]) {
        double2 v = *reinterpret_cast<const double2 *>(p);
        o[0] = v.x;
        o[1] = v.y;
    }
    __device__ __forceinline__ static void store(double *p, const C (&o)[R]) {
        *reinterpret_cast<double2 *>(p) = make_double2(o[0], o[1]);
    }
    __device__ __forceinline__ static C to_c(double v) { return v; }
    __device__ __forceinline__ static double from_c(C v) { return v; }
};
template <>
struct Store<float> {
    using C = double;
    static constexpr int R = 4;
    __device__ __forceinline__ static void load(const float *p, C (&o)[R]) {
        float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
    __device__ __forceinline__ static void lds(const float *p, C (&o)[R]) {
        float4 v = *reinterpret_cast<const float4 *>(p);
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    }
    __device__ __forceinline__ static void store(float *p, const C (&o)[R]) {
        *reinterpret_cast<float4 *>(p) =
            make_float4((float)o[0], (float)o[1], (float)o[2], (float)o[3]);
    }
    __device__ __forceinline__ static C to_c(float v) { return v; }
    __device__ __forceinline__ static float from_c(C v) { return (float)v; }
};
template <>
struct Store<zd> {
    using C = zd;
    static constexpr int R = 1;
    __device__ __forceinline__ static void load(const zd *p, C (&o)[R]) {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        o[0] = zd{v.x, v.y};
    }
    __device__ __forceinline__ static void lds(const zd *p, C (&o)[R]) {
        double2 v = *reinterpret_cast<const double2 *>(p);
        o[0] = zd{v.x, v.y};
    }
    __device__ __forceinline__ static void store(zd *p, const C (&o)[R]) {
        *reinterpret_cast<double2 *>(p) = make_double2(o[0].x, o[0].y);
    }
    __device__ __forceinline__ static C to_c(zd v) { return v; }
    __device__ __forceinline__ static zd from_c(C v) { return v; }
};
template <>
struct Store<zf> {
    using C = zd;
    static constexpr int R = 2;
    __device__ __forceinline__ static void load(const zf *p, C (&o)[R]) {
        float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        o[0] = zd{v.x, v.y};
        o[1] = zd{v.z, v.w};
    }
    __device__ __forceinline__ static void lds(const zf *p, C (&o)[R]) {
        float4 v = *reinterpret_cast<const float4 *>(p);
        o[0] = zd{v.x, v.y};
        o[1] = zd{v.z, v.w};
    }
    __device__ __forceinline__ static void store(zf *p, const C (&o)[R]) {
        *reinterpret_cast<float4 *>(p) =
            make_float4((float)o[0].x, (float)o[0].y, (float)o[1].x, (float)o[1].y);
    }
    __device__ __forceinline__ static C to_c(zf v) { return zd{v.x, v.y}; }
    __device__ __forceinline__ static zf from_c(C v) { return zf{(float)v.x, (float)v.y}; }
};

// Loads of the FP64 compute vectors (r, y, x): R elements at p.
template <int R>
__device__ __forceinline__ void load_c(const double *p, double (&o)[R]) {
#pragma unroll
    for (int k = 0; k < R; k += 2) {
        double2 v = *reinterpret_cast<const double2 *>(p + k);
        o[k] = v.x;
        if (k + 1 < R) o[k + 1] = v.y;
    }
}
template <int R>
__device__ __forceinline__ void load_c(const zd *p, zd (&o)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
        double2 v = *reinterpret_cast<const double2 *>(p + k);
        o[k] = zd{v.x, v.y};
    }
}
template <int R>
__device__ __forceinline__ void store_c(double *p, const double (&o)[R]) {
#pragma unroll
    for (int k = 0; k < R; k += 2) *reinterpret_cast<double2 *>(p + k) = make_double2(o[k], o[k + 1]);
}
template <int R>
__device__ __forceinline__ void store_c(zd *p, const zd (&o)[R]) {
#pragma unroll
    for (int k = 0; k < R; ++k) *reinterpret_cast<double2 *>(p + k) = make_double2(o[k].x, o[k].y);
}

// ---- deterministic reductions ------------------------------------------------
// Sum over the block in a fixed tree order; result valid in thread 0.
template <class C>
__device__ __forceinline__ C block_sum(C v, C *smem /* >= 32 entries */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = v + shfl_down(v, o);
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    C s = czero(v);
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 0; w < nw; ++w) s = s + smem[w];
    }
    __syncthreads();
    return s;
}

// Final sum of nb per-block partials, run by every thread of the last block
// in a fixed order: thread t adds part[t], part[t + blockDim.x], ..., then
// the block tree of block_sum.  Returns the total in thread 0.
__device__ __forceinline__ double sum_partials(const double *part, int nb, double *smem /* >= 32 entries */) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += __ldcg(part + b);
    return block_sum(s, smem);
}

// Called by every thread after the block wrote its partials: returns true in
// exactly one block (the last to arrive), which then owns the final sums.
__device__ __forceinline__ bool last_block_arrived(unsigned *ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

// Final step of a grid reduction, run by the last block: out[c] =
// sum_b part[b * m + c] for c < m, in a fixed order.  Each column gets
// tpc = max(1, blockDim / m) threads (power of two); thread j of a column
// sums blocks b = j, j + tpc, ... with 8 independent accumulators (8 loads
// in flight), and the tpc partial sums are then added in thread order.
// Returns, in thread 0, sum_c |out[c]|^2.  smem must hold blockDim.x values.
template <class C>
__device__ inline double reduce_columns(const C *part, int nb, int m, C *out, C *smem) {
    int tpc = 1;
    while (tpc * 2 * m <= (int)blockDim.x) tpc *= 2;
    const int groups = blockDim.x / tpc;  // columns handled per round
    double norm2 = 0.0;
    for (int c0 = 0; c0 < m; c0 += groups) {
        const int c = c0 + (int)threadIdx.x / tpc;
        const int j = threadIdx.x % tpc;
        C acc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[u] = czero(C());
        if (c < m) {
            int b = j;
            for (; b + 7 * tpc < nb; b += 8 * tpc) {
#pragma unroll
                for (int u = 0; u < 8; ++u) acc[u] = acc[u] + ldcg(part + (long)(b + u * tpc) * m + c);
            }
            for (; b < nb; b += tpc) acc[0] = acc[0] + ldcg(part + (long)b * m + c);
        }
        smem[threadIdx.x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
        __syncthreads();
        if (j == 0 && c < m) {
            C s = smem[threadIdx.x];
            for (int q = 1; q < tpc; ++q) s = s + smem[threadIdx.x + q];
            out[c] = s;
            smem[threadIdx.x] = s;  // keep for the norm below
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int g = 0; g < groups && c0 + g < m; ++g) norm2 += abs2(smem[g * tpc]);
        }
        __syncthreads();
    }
    return norm2;
}

// Counter-based uniform [0,1) generator (splitmix64 finaliser).
__host__ __device__ inline double uniform01(uint64_t seed, uint64_t i) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace trlb

// Seed-network convolution on the 5th-generation tensor cores (tcgen05).
//
// The same implicit GEMM as k_conv (pixels x 288 taps*channels x 32 output
// channels, BF16 in, FP32 accumulate, bias + optional ReLU), Blackwell-style:
//   * one persistent CTA of 4 warps per SM walks tiles of 128 pixels
//     (TW x TH pixels of one sample: a full 128-pixel row segment, or 2 rows
//     of 64, ...);
//   * the 3x3 taps of a tile are 9 TMA loads of 128 pixels x 32 channels
//     (64 B per pixel, 64-byte swizzle) from the NHWC activations, at
//     coordinates shifted by the dilated tap offset: the "same" zero padding
//     is the TMA's out-of-bounds fill.  Tiles are double-buffered;
//   * the weights ([tap][co][ci], 9 x 32 x 64 B, same swizzle) are one TMA
//     load per CTA;
//   * one thread issues 18 tcgen05.mma (M = 128, N = 32, K = 16, kind::f16
//     with BF16 operands) from shared-memory descriptors into a TMEM
//     accumulator of 32 columns and commits to an mbarrier;
//   * the 4 warps read the accumulator with tcgen05.ld (warp w: TMEM lanes =
//     pixels 32w .. 32w+31, 32 channels each), add the bias, apply the ReLU
//     and store BF16 NHWC (or the first 16 channels as FP32 for the last
//     layer).
// That is k_conv_tc, used for images narrower than 128 pixels (and under
// TRLX_SEEDNET_CONV=tap).  Wider images (W a multiple of 128) use
// k_conv_rows: the three input rows of a tile loaded once, a producer warp
// for the loads, several MMA-issuing lanes, and the BF16 output staged in
// shared memory and written with TMA stores.  The weight gradients are
// k_wgrad_rows (staged rows) and k_wgrad_tc (nine tap tiles).
// Every mbarrier wait is bounded; a wait that runs out sets a device flag
// (read by the seed-network entry points) and the kernel still runs to its
// end, so the TMEM allocation is always released.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

namespace trlb {
namespace seednet {
namespace {

constexpr int kTM = 128;                      // pixels per tile (MMA M)
constexpr int kCh = 32;                       // channels (MMA N and K per tap)
constexpr int kTapsTC = 9;
constexpr int kRow = kCh * 2;                 // bytes per pixel / weight row
constexpr int kTapA = kTM * kRow;             // 8 KB per tap tile
constexpr int kStageA = kTapsTC * kTapA;      // 72 KB per pixel tile
constexpr int kTapW = kCh * kRow;             // 2 KB per tap of weights
constexpr int kWBytes = kTapsTC * kTapW;      // 18 KB
constexpr int kOffA = kWBytes;                // 1 KB aligned
constexpr int kOffBar = kOffA + 2 * kStageA;  // mbarriers after the buffers
constexpr size_t kSmemTC = kOffBar + 128 + 1024;  // 9 mbarriers + TMEM slot + alignment slack
constexpr long kWaitLimit = 1L << 24;

__device__ int g_tc_error = 0;

__device__ __forceinline__ unsigned saddr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t *b, unsigned n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect(uint64_t *b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t *b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(saddr(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; on timeout records the failure and returns.
__device__ __forceinline__ void bar_wait(uint64_t *b, unsigned parity) {
    for (long i = 0; !bar_try(b, parity); ++i) {
        if (i > kWaitLimit) {
            atomicExch(&g_tc_error, 1);
            return;
        }
    }
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];" ::"r"(saddr(dst)),
        "l"(map), "r"(saddr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(saddr(dst)),
        "l"(map), "r"(saddr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Shared-memory matrix descriptor: K-major operand, rows of 64 B in 8-row
// groups 512 B apart, 64-byte swizzle (layout type 4), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(unsigned addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)1 << 16;                        // leading byte offset (unused with swizzle)
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;    // stride byte offset: 8 rows x 64 B
    d |= (uint64_t)1 << 46;                        // version
    d |= (uint64_t)4 << 61;                        // SWIZZLE_64B
    return d;
}
// Instruction descriptor: D FP32, A and B BF16, both K-major, N = 32, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCh >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
        "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<unsigned *>(&v);
}

// Warp roles: warps 0-3 read the accumulator (warp w owns TMEM lanes = tile
// pixels 32w .. 32w+31), one lane of warp 4 issues the TMA loads and the
// MMAs.  Two accumulators of 32 TMEM columns alternate between tiles, so the
// MMAs of tile i+1 run while tile i's epilogue reads its accumulator.
// Barriers: full[s] (tile loaded into stage s), done[a] (MMAs into
// accumulator a finished: the epilogue may read it and stage s may be
// refilled), empty[a] (the 4 epilogue warps finished reading accumulator
// a), weights.  Serves images narrower than 128 pixels (tiles of TW x TH
// pixels), dilations above 8 and TRLX_SEEDNET_CONV=tap, as 9 shifted tap
// tiles.
__global__ void __launch_bounds__(160, 1)
    k_conv_tc(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap twt,
              const float *__restrict__ bias, __nv_bfloat16 *out, float *out_f32, int H, int W, int TW, int TH,
              int dil, int relu, int ntiles) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *ws = sm;
    unsigned char *as = sm + kOffA;
    constexpr int NS = 2;  // stages of 72 KB (9 tap tiles)
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kOffBar);
    uint64_t *full = bars, *done = bars + 4, *empty = bars + 6, *wbar = bars + 8;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 9);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = W / TW, tiles_y = H / TH;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < 6; ++k) bar_init(bars + k, 1);  // full[4], done[2]
        bar_init(empty, 4);
        bar_init(empty + 1, 4);
        bar_init(wbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 4) {
        if (lane == 0) {
            auto issue = [&](int it) {
                const int tile = blockIdx.x + it * gridDim.x;
                const int tx = tile % tiles_x, rest = tile / tiles_x;
                const int ty = rest % tiles_y, b = rest / tiles_y;
                const int x0 = tx * TW, y0 = ty * TH, st = it % NS;
                bar_expect(full + st, kStageA);
                for (int tap = 0; tap < kTapsTC; ++tap) {
                    const int dy = (tap / 3 - 1) * dil, dx = (tap % 3 - 1) * dil;
                    tma_load_4d(as + st * kStageA + tap * kTapA, &tin, full + st, 0, x0 + dx, y0 + dy, b);
                }
            };
            // Every load issued here is waited for below (no copy is in
            // flight when the CTA exits).
            if (my_tiles > 0) {
                bar_expect(wbar, kWBytes);
                tma_load_3d(ws, &twt, wbar, 0, 0, 0);
            }
            for (int it = 0; it < NS && it < my_tiles; ++it) issue(it);
            if (my_tiles > 0) bar_wait(wbar, 0);
            const unsigned w0 = saddr(ws);
            for (int it = 0; it < my_tiles; ++it) {
                const int st = it % NS, acc = it & 1;
                bar_wait(full + st, (unsigned)((it / NS) & 1));
                if (it >= 2) bar_wait(empty + acc, (unsigned)(((it >> 1) - 1) & 1));
                tc_fence_after();
                const unsigned a0 = saddr(as + st * kStageA);
                const uint32_t d = tmem + (uint32_t)(acc * kCh);
#pragma unroll 1
                for (int tap = 0; tap < kTapsTC; ++tap)
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        mma_f16(d, smem_desc(a0 + tap * kTapA + k * 32), smem_desc(w0 + tap * kTapW + k * 32),
                                (tap | k) != 0);
                mma_commit(done + acc);
                if (it + NS < my_tiles) {
                    // The MMAs have read stage st once they complete.
                    bar_wait(done + acc, (unsigned)((it >> 1) & 1));
                    issue(it + NS);
                }
            }
        }
    } else {
        float bv[kCh];
#pragma unroll
        for (int c = 0; c < kCh; ++c) bv[c] = bias ? bias[c] : 0.f;
        for (int it = 0; it < my_tiles; ++it) {
            const int acc = it & 1;
            const int tile = blockIdx.x + it * gridDim.x;
            bar_wait(done + acc, (unsigned)((it >> 1) & 1));
            tc_fence_after();
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * kCh), r);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(empty + acc)) : "memory");
            const int tx = tile % tiles_x, rest = tile / tiles_x;
            const int ty = rest % tiles_y, b = rest / tiles_y;
            const int i = warp * 32 + lane;
            const long p = ((long)b * H + ty * TH + i / TW) * W + tx * TW + i % TW;
            float v[kCh];
#pragma unroll
            for (int c = 0; c < kCh; ++c) {
                v[c] = __uint_as_float(r[c]) + bv[c];
                if (relu) v[c] = fmaxf(v[c], 0.f);
            }
            if (out_f32) {
                float4 *o = reinterpret_cast<float4 *>(out_f32 + p * 16);
#pragma unroll
                for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
                uint4 *o = reinterpret_cast<uint4 *>(out + p * kCh);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    o[q] = make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                      pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
}

// Row tiles (W a multiple of 128, dilation <= 8): one tile = 128 pixels of
// one image row.  Instead of 9 tap tiles, the three input rows y - d, y,
// y + d are loaded once with a halo of d pixels on each side (box of
// 128 + 2d pixels), and each tap's A operand is a view starting kx*d rows
// into its row buffer (the swizzle follows the absolute shared-memory
// address, as the TMA wrote it; results are bitwise those of the 9-tap
// form).  Warp roles (kEpi epilogue warpgroups, kLanes MMA lanes):
//   * warps 0 .. 4*kEpi-1 run the epilogue, warpgroup g taking the tiles
//     it = g (mod kEpi): read accumulator it % kAcc, add the bias, apply
//     the ReLU, and for BF16 output write their 32 pixels x 64 B into a
//     shared-memory buffer in the output tensor map's 64-byte swizzle
//     (conflict-free 16-byte stores), which one lane sends out with a TMA
//     tensor store (two buffers per warp; a buffer is rewritten once the
//     store from two tiles back has read it).  FP32 output (the last
//     layer) is stored directly;
//   * warp 4*kEpi (one lane) is the producer: weights once, then the three
//     rows of each tile into kStages stages, refilling stage s once the
//     MMAs that read it have completed (free[s]);
//   * the next kLanes warps (one lane each) issue the MMAs, lane m taking
//     the tiles it = m (mod kLanes): 18 tcgen05.mma from descriptors
//     precomputed per tile (the taps are compile-time offsets), committed
//     to free[s] and done[a].
// Measured (256 x 256, 32 -> 32 channels, batch 8, clock stamps per tile):
// one lane spends about 71 cycles per M = 128, N = 32, K = 16 MMA issue, 18
// per tile, while the tensor pipe is mostly idle, so several lanes issue
// for different tiles.
constexpr int kRowBuf = 9 * 1024;  // one staged input row, (128 + 2*8) x 64 B, 1 KB aligned

template <int kLanes, int kEpi, int kStages>
struct RowCfg {
    static constexpr int kAcc = 2 * kLanes;  // TMEM accumulators of 32 columns
    static_assert(kAcc % kEpi == 0, "an accumulator belongs to one epilogue warpgroup");
    static constexpr int kThreads = 32 * (4 * kEpi + 1 + kLanes);
    static constexpr int kCols = kAcc * kCh;
    static_assert(kCols >= 32 && kCols <= 512 && (kCols & (kCols - 1)) == 0, "TMEM allocations are powers of two");
    static constexpr int kOffA = kWBytes;
    static constexpr int kOffO = kOffA + kStages * 3 * kRowBuf;  // 4*kEpi warps x 2 buffers of 2 KB
    static constexpr int kOffBar = kOffO + 4 * kEpi * 2 * 2048;
    static constexpr int kBars = 2 * kStages + 2 * kAcc + 1;
    static_assert(kBars * 8 + 4 <= 256, "mbarriers and the TMEM slot fit in 256 bytes");
    static constexpr size_t kSmem = kOffBar + 256 + 1024;  // + alignment slack
};

__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(map),
                 "r"(saddr(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

template <int kLanes, int kEpi, int kStages>
__global__ void __launch_bounds__(RowCfg<kLanes, kEpi, kStages>::kThreads, 1)
    k_conv_rows(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap twt,
                const __grid_constant__ CUtensorMap tout, const float *__restrict__ bias, float *out_f32, int H,
                int W, int dil, int relu, int ntiles) {
    using Cfg = RowCfg<kLanes, kEpi, kStages>;
    constexpr int NS = kStages, NA = Cfg::kAcc;
    constexpr int SB = 3 * kRowBuf;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char *ws = sm;
    unsigned char *as = sm + Cfg::kOffA;
    unsigned char *os = sm + Cfg::kOffO;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + Cfg::kOffBar);
    uint64_t *full = bars, *freeb = bars + NS, *done = bars + 2 * NS, *empty = bars + 2 * NS + NA;
    uint64_t *wbar = bars + 2 * NS + 2 * NA;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + Cfg::kBars);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = W / kTM;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                     "r"(Cfg::kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < 2 * NS + NA; ++k) bar_init(bars + k, 1);  // full, free, done
        for (int k = 0; k < NA; ++k) bar_init(empty + k, 4);          // the 4 warps of a warpgroup
        bar_init(wbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 4 * kEpi) {
        // Every load issued here is waited for by an MMA lane (full[s]), so
        // no copy is in flight when the CTA exits.
        if (lane == 0 && my_tiles > 0) {
            bar_expect(wbar, kWBytes);
            tma_load_3d(ws, &twt, wbar, 0, 0, 0);
            int tile = blockIdx.x;
            for (int it = 0; it < my_tiles; ++it, tile += gridDim.x) {
                const int st = it % NS;
                const int tx = tile % tiles_x, rest = tile / tiles_x;
                const int y = rest % H, b = rest / H;
                if (it >= NS) bar_wait(freeb + st, (unsigned)(((it / NS) - 1) & 1));
                bar_expect(full + st, 3u * (unsigned)(kTM + 2 * dil) * kRow);
                for (int ky = 0; ky < 3; ++ky)
                    tma_load_4d(as + st * SB + ky * kRowBuf, &tin, full + st, 0, tx * kTM - dil, y + (ky - 1) * dil,
                                b);
            }
        }
    } else if (warp > 4 * kEpi) {
        const int m = warp - 4 * kEpi - 1;  // MMA lane
        if (lane == 0 && m < my_tiles) {
            bar_wait(wbar, 0);
            const uint64_t dB = smem_desc(saddr(ws));
            const uint32_t d4 = (uint32_t)dil * (kRow >> 4);  // one pixel shift in 16-byte units
            for (int it = m; it < my_tiles; it += kLanes) {
                const int st = it % NS, acc = it % NA;
                bar_wait(full + st, (unsigned)((it / NS) & 1));
                if (it >= NA) bar_wait(empty + acc, (unsigned)(((it / NA) - 1) & 1));
                tc_fence_after();
                // Descriptor start addresses stay below 2^14 x 16 B (shared
                // memory), so adding offsets never carries out of the field.
                const uint64_t dA = smem_desc(saddr(as + st * SB));
                const uint32_t d = tmem + (uint32_t)(acc * kCh);
#pragma unroll
                for (int tap = 0; tap < kTapsTC; ++tap)
#pragma unroll
                    for (int k = 0; k < 2; ++k)
                        mma_f16(d, dA + (uint64_t)((tap / 3) * (kRowBuf >> 4) + (tap % 3) * d4 + k * 2),
                                dB + (uint64_t)((tap * kTapW + k * 32) >> 4), (tap | k) != 0);
                mma_commit(freeb + st);
                mma_commit(done + acc);
            }
        }
    } else {
        const int g = warp >> 2, quarter = warp & 3;  // epilogue warpgroup, TMEM lane quarter
        float bv[kCh];
#pragma unroll
        for (int c = 0; c < kCh; ++c) bv[c] = bias ? bias[c] : 0.f;
        int nb = 0;  // this warp's tiles so far (output buffer parity)
        for (int it = g; it < my_tiles; it += kEpi, ++nb) {
            const int acc = it % NA;
            const int tile = blockIdx.x + it * gridDim.x;
            bar_wait(done + acc, (unsigned)((it / NA) & 1));
            tc_fence_after();
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kCh), r);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(saddr(empty + acc)) : "memory");
            const int tx = tile % tiles_x, rest = tile / tiles_x;
            const int y = rest % H, b = rest / H;
            float v[kCh];
#pragma unroll
            for (int c = 0; c < kCh; ++c) {
                v[c] = __uint_as_float(r[c]) + bv[c];
                if (relu) v[c] = fmaxf(v[c], 0.f);
            }
            if (out_f32) {
                const long p = ((long)b * H + y) * W + tx * kTM + quarter * 32 + lane;
                float4 *o = reinterpret_cast<float4 *>(out_f32 + p * 16);
#pragma unroll
                for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            } else {
                unsigned char *ob = os + (warp * 2 + (nb & 1)) * 2048;
                if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                __syncwarp();
                // 16-byte chunk q of pixel l at l*64 + 16*(q ^ ((l >> 1) & 3)):
                // the 64-byte swizzle of the output tensor map.
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    *reinterpret_cast<uint4 *>(ob + lane * 64 + ((q ^ ((lane >> 1) & 3)) << 4)) =
                        make_uint4(pack2(v[8 * q], v[8 * q + 1]), pack2(v[8 * q + 2], v[8 * q + 3]),
                                   pack2(v[8 * q + 4], v[8 * q + 5]), pack2(v[8 * q + 6], v[8 * q + 7]));
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    tma_store_4d(&tout, ob, 0, tx * kTM + quarter * 32, y, b);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                }
            }
        }
        // The stores have finished before the CTA exits.
        if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
        __syncwarp();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kCols) : "memory");
}

// The configuration the library launches: four MMA lanes, two epilogue
// warpgroups, six stages (213 KB of shared memory, 416 threads).  Measured
// per 32 -> 32 layer at 256 x 256, batch 16: 1 lane 66 us, 2 lanes 41 us,
// 4 lanes with one epilogue warpgroup 41 us (the epilogue bound), 4 lanes
// with two 37 us; every configuration bitwise equal to the 9-tap kernel.
using RowsCfg = RowCfg<4, 2, 6>;
constexpr auto *kRowsKernel = &k_conv_rows<4, 2, 6>;

// ---------------------------------------------------------------------------
// Weight gradient on tcgen05: dW[tap][ci][co] = sum_p in[p + off(tap)][ci] *
// g[p][co] and db[co] = sum_p g[p][co], as a GEMM over pixels (K) with the
// taps stacked along M: accumulator group j (M = 128 rows = 4 slots x 32
// ci) covers taps 4j .. 4j+3; the third group holds tap 8, a slot of ones
// (its rows give db) and two zero slots.  Both operands are MN-major (ci or
// co contiguous, 64 B per pixel, 64-byte swizzle): a stage is one 64-pixel
// row segment, i.e. 9 TMA loads of the shifted input (zero fill outside the
// image) and one of g, 4 KB each, into slots 4 KB apart (the descriptors'
// leading byte offset between M atoms; 8-pixel K atoms are 512 B apart).
// One CTA per SM accumulates its segments in TMEM (3 x 32 columns), then
// writes the per-block partials part[block][tap][ci][co] (+ [9][0][co] =
// db) that k_reduce_parts sums in block order.
constexpr int kWSeg = 64;                                   // pixels per stage (K)
constexpr int kWSlot = kWSeg * kRow;                        // 4 KB
constexpr int kWSlots = 12;                                 // 9 taps, ones, 2 zero
constexpr int kWStage = (kWSlots + 1) * kWSlot;             // + g tile: 52 KB
constexpr int kWStages = 3;
constexpr int kWOffBar = kWStages * kWStage;
constexpr size_t kSmemWG = kWOffBar + 128 + 1024;
constexpr uint32_t kIdescMN = kIdesc | (1u << 15) | (1u << 16);  // A and B MN-major

__device__ __forceinline__ uint64_t smem_desc_mn(unsigned addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);               // start address
    d |= (uint64_t)((kWSlot >> 4) & 0x3FFF) << 16;       // leading byte offset: next 32-wide M atom
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;          // stride byte offset: next 8 pixels of K
    d |= (uint64_t)1 << 46;                              // version
    d |= (uint64_t)4 << 61;                              // SWIZZLE_64B
    return d;
}
__device__ __forceinline__ void mma_f16_mn(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdescMN), "r"(accumulate)
        : "memory");
}

__global__ void __launch_bounds__(160, 1)
    k_wgrad_tc(const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tg, float *part, int H,
               int W, int dil, int nseg) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kWOffBar);
    uint64_t *full = bars, *done = bars + kWStages, *fin = bars + 2 * kWStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * kWStages + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int segs_x = W / kWSeg;
    const int my = (int)blockIdx.x < nseg ? (nseg - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    // Constant slots of every stage: ones (slot 9), zeros (10, 11).
    for (int st = 0; st < kWStages; ++st) {
        uint4 *o = reinterpret_cast<uint4 *>(sm + st * kWStage + 9 * kWSlot);
        const unsigned one2 = 0x3F803F80u;  // two bf16 1.0
        for (int i = tid; i < 3 * kWSlot / 16; i += blockDim.x)
            o[i] = i < kWSlot / 16 ? make_uint4(one2, one2, one2, one2) : make_uint4(0u, 0u, 0u, 0u);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                     "r"(128)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < 2 * kWStages + 1; ++k) bar_init(bars + k, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        if (lane == 0) {
            auto issue = [&](int it) {
                const int seg = blockIdx.x + it * gridDim.x;
                const int sx = seg % segs_x, rest = seg / segs_x;
                const int y = rest % H, b = rest / H, x0 = sx * kWSeg;
                const int st = it % kWStages;
                unsigned char *base = sm + st * kWStage;
                bar_expect(full + st, 10 * kWSlot);
                for (int tap = 0; tap < 9; ++tap) {
                    const int dy = (tap / 3 - 1) * dil, dx = (tap % 3 - 1) * dil;
                    tma_load_4d(base + tap * kWSlot, &tin, full + st, 0, x0 + dx, y + dy, b);
                }
                tma_load_4d(base + kWSlots * kWSlot, &tg, full + st, 0, x0, y, b);
            };
            for (int it = 0; it < my && it < kWStages; ++it) issue(it);
            for (int it = 0; it < my; ++it) {
                const int st = it % kWStages;
                const unsigned ph = (unsigned)((it / kWStages) & 1);
                bar_wait(full + st, ph);
                tc_fence_after();
                const unsigned a0 = saddr(sm + st * kWStage), b0 = a0 + kWSlots * kWSlot;
#pragma unroll 1
                for (int grp = 0; grp < 3; ++grp)
#pragma unroll
                    for (int k = 0; k < kWSeg / 16; ++k)
                        mma_f16_mn(tmem + (uint32_t)(grp * kCh), smem_desc_mn(a0 + grp * 4 * kWSlot + k * 1024),
                                   smem_desc_mn(b0 + k * 1024), (it | k) != 0);
                mma_commit(done + st);
                if (it + kWStages < my) {
                    bar_wait(done + st, ph);  // the MMAs have read this stage
                    issue(it + kWStages);
                }
            }
            mma_commit(fin);
        }
    } else if (my > 0) {
        bar_wait(fin, 0);
        tc_fence_after();
        float *pb = part + (size_t)blockIdx.x * (kTapsTC + 1) * kCh * kCh;
#pragma unroll 1
        for (int grp = 0; grp < 3; ++grp) {
            uint32_t r[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(grp * kCh), r);
            const int slot = grp * 4 + warp;  // row block: tap, or ones (9), or zeros
            if (slot < 9) {
                float4 *o = reinterpret_cast<float4 *>(pb + ((size_t)slot * kCh + lane) * kCh);
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    o[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                       __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
            } else if (slot == 9 && lane == 0) {
                float4 *o = reinterpret_cast<float4 *>(pb + (size_t)kTapsTC * kCh * kCh);
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    o[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                       __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
}

// Weight gradient with the input rows staged once per segment: a stage holds
// the three input rows y - d, y, y + d of a 64-pixel segment with a halo of
// d pixels (64 + 2d pixels each, zero fill outside the image), a row of
// ones and the g tile.  Accumulator group kx (M = 128 = 4 atoms of 32 ci)
// is one descriptor whose M atoms are the three rows at pixel shift kx*d
// (taps (0, kx), (1, kx), (2, kx)) and the ones row (the leading byte
// offset is the row-buffer stride), so the K shift runs along the pixels of
// an MN-major operand, read at the absolute swizzled addresses the TMA
// wrote.  Group 0's ones atom gives db; the ones atoms of groups 1 and 2
// compute the same sums and are not written.  Loads per segment: 3 rows of
// at most 5 KB and a 4 KB g tile, against 9 + 1 tiles of 4 KB.
// Warps 0-3 read the accumulators, warp 4 (one lane) is the producer, and
// kLanes warps (one lane each) issue the MMAs for alternate segments into
// private accumulators (3 x 32 columns each), which the epilogue adds in
// lane order.
constexpr int kWRowBuf = 5 * 1024;                       // (64 + 2*8) px x 64 B, 1 KB aligned
constexpr int kWRowStage = 4 * kWRowBuf + kWSlot;        // 3 rows, ones, g: 24 KB
constexpr int kWRowStages = 6;
constexpr int kWRowLanes = 2;
constexpr int kWRowOffBar = kWRowStages * kWRowStage;
constexpr int kWRowThreads = 32 * (5 + kWRowLanes);
constexpr size_t kSmemWR = kWRowOffBar + 128 + 1024;

__device__ __forceinline__ uint64_t smem_desc_mn_rows(unsigned addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);               // start address
    d |= (uint64_t)((kWRowBuf >> 4) & 0x3FFF) << 16;     // leading byte offset: next row buffer (M atom)
    d |= (uint64_t)((512 >> 4) & 0x3FFF) << 32;          // stride byte offset: next 8 pixels of K
    d |= (uint64_t)1 << 46;                              // version
    d |= (uint64_t)4 << 61;                              // SWIZZLE_64B
    return d;
}

__global__ void __launch_bounds__(kWRowThreads, 1)
    k_wgrad_rows(const __grid_constant__ CUtensorMap trow, const __grid_constant__ CUtensorMap tg, float *part,
                 int H, int W, int dil, int nseg) {
    constexpr int NS = kWRowStages;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kWRowOffBar);
    uint64_t *full = bars, *freeb = bars + NS, *fin = bars + 2 * NS;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2 * NS + kWRowLanes);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int segs_x = W / kWSeg;
    const int my = (int)blockIdx.x < nseg ? (nseg - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    // The ones row of every stage (bf16 1.0 pairs).
    for (int st = 0; st < NS; ++st) {
        uint4 *o = reinterpret_cast<uint4 *>(sm + st * kWRowStage + 3 * kWRowBuf);
        for (int i = tid; i < kWRowBuf / 16; i += blockDim.x)
            o[i] = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(tslot)),
                     "r"(256)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int k = 0; k < 2 * NS + kWRowLanes; ++k) bar_init(bars + k, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        // Every load issued here is waited for by an MMA lane (full[s]).
        if (lane == 0) {
            int seg = blockIdx.x;
            for (int it = 0; it < my; ++it, seg += gridDim.x) {
                const int st = it % NS;
                const int sx = seg % segs_x, rest = seg / segs_x;
                const int y = rest % H, b = rest / H, x0 = sx * kWSeg;
                unsigned char *base = sm + st * kWRowStage;
                if (it >= NS) bar_wait(freeb + st, (unsigned)(((it / NS) - 1) & 1));
                bar_expect(full + st, 3u * (unsigned)(kWSeg + 2 * dil) * kRow + kWSlot);
                for (int ky = 0; ky < 3; ++ky)
                    tma_load_4d(base + ky * kWRowBuf, &trow, full + st, 0, x0 - dil, y + (ky - 1) * dil, b);
                tma_load_4d(base + 4 * kWRowBuf, &tg, full + st, 0, x0, y, b);
            }
        }
    } else if (warp >= 5) {
        const int m = warp - 5;  // MMA lane
        if (lane == 0 && m < my) {
            const uint32_t d0 = tmem + (uint32_t)(m * 128);
            const unsigned shift = (unsigned)dil * kRow;  // bytes per pixel shift
            for (int it = m; it < my; it += kWRowLanes) {
                const int st = it % NS;
                bar_wait(full + st, (unsigned)((it / NS) & 1));
                tc_fence_after();
                const unsigned a0 = saddr(sm + st * kWRowStage), b0 = a0 + 4 * kWRowBuf;
#pragma unroll
                for (int kx = 0; kx < 3; ++kx)
#pragma unroll
                    for (int k = 0; k < kWSeg / 16; ++k)
                        mma_f16_mn(d0 + (uint32_t)(kx * kCh), smem_desc_mn_rows(a0 + kx * shift + k * 1024),
                                   smem_desc_mn(b0 + k * 1024), (it != m || k != 0) ? 1u : 0u);
                mma_commit(freeb + st);
            }
            mma_commit(fin + m);
        }
    } else if (my > 0) {
        const int lanes = my < kWRowLanes ? my : kWRowLanes;  // lanes that accumulated
        for (int m = 0; m < lanes; ++m) bar_wait(fin + m, 0);
        tc_fence_after();
        float *pb = part + (size_t)blockIdx.x * (kTapsTC + 1) * kCh * kCh;
#pragma unroll 1
        for (int kx = 0; kx < 3; ++kx) {
            if (warp == 3 && kx > 0) continue;  // ones atoms of groups 1, 2: not used
            float v[32];
            {
                uint32_t r[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kx * kCh), r);
#pragma unroll
                for (int c = 0; c < 32; ++c) v[c] = __uint_as_float(r[c]);
            }
            for (int m = 1; m < lanes; ++m) {
                uint32_t r[32];
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * 128 + kx * kCh), r);
#pragma unroll
                for (int c = 0; c < 32; ++c) v[c] += __uint_as_float(r[c]);
            }
            float *row = nullptr;
            if (warp < 3) row = pb + ((size_t)(warp * 3 + kx) * kCh + lane) * kCh;  // tap (ky = warp, kx), ci = lane
            else if (lane == 0) row = pb + (size_t)kTapsTC * kCh * kCh;             // db
            if (row) {
                float4 *o = reinterpret_cast<float4 *>(row);
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
    static EncodeTiled fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiled) nullptr;
        }
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

// Reports once why the tcgen05 kernel is not used (the mma.sync kernel runs).
void tc_note(const char *why) {
    static bool said = false;
    if (!said) std::fprintf(stderr, "TRLAN-B200: seed network on the mma.sync convolution: %s\n", why);
    said = true;
}

// Input rows staged once per tile (the default for 128-pixel row tiles;
// TRLX_SEEDNET_CONV=tap keeps the 9 tap loads).
bool rows_mode() {
    static const bool on = [] {
        const char *e = std::getenv("TRLX_SEEDNET_CONV");
        return !(e && e[0] == 't');
    }();
    return on;
}

// Per device (the shared-memory attribute is set on the current device):
// 0 not tried, 1 usable, -1 not usable.
constexpr int kMaxDev = 64;
int g_dev_state[kMaxDev] = {};

bool tc_enabled() {
    static const bool allowed = [] {
        const char *e = std::getenv("TRLX_SEEDNET_CONV");
        if (e && e[0] == 'm') return false;  // "mma": the mma.sync kernel
        if (!encoder()) {
            tc_note("cuTensorMapEncodeTiled not available");
            return false;
        }
        return true;
    }();
    if (!allowed) return false;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) return false;
    if (g_dev_state[dev] == 0) {
        cudaError_t err =
            cudaFuncSetAttribute(k_conv_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTC);
        if (err == cudaSuccess)
            err = cudaFuncSetAttribute(kRowsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)RowsCfg::kSmem);
        if (err != cudaSuccess) {
            tc_note(cudaGetErrorString(err));
            cudaGetLastError();
        }
        g_dev_state[dev] = err == cudaSuccess ? 1 : -1;
    }
    return g_dev_state[dev] == 1;
}

}  // namespace

// Runs the convolution on the tcgen05 kernel when the shape allows (tiles of
// 128 pixels: W a multiple of min(W, 128) and H of 128 / min(W, 128)) and
// returns true; false leaves it to the caller's kernel.
bool conv_tc(const __nv_bfloat16 *in, const __nv_bfloat16 *w, const float *bias, __nv_bfloat16 *out, float *out_f32,
             int B, int H, int W, int dil, int relu) {
    if (!tc_enabled()) return false;
    const int TW = W < kTM ? W : kTM;
    if (TW < 8 || kTM % TW != 0 || W % TW != 0) return false;
    const int TH = kTM / TW;
    if (H % TH != 0) return false;
    if (((uintptr_t)in & 15) || ((uintptr_t)w & 15)) {
        tc_note("operands not 16-byte aligned");
        return false;
    }
    CUtensorMap tin, twt;
    const cuuint64_t din[4] = {(cuuint64_t)kCh, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t sin[3] = {(cuuint64_t)kRow, (cuuint64_t)W * kRow, (cuuint64_t)H * W * kRow};
    const cuuint32_t bin[4] = {(cuuint32_t)kCh, (cuuint32_t)TW, (cuuint32_t)TH, 1};
    const cuuint32_t ones[4] = {1, 1, 1, 1};
    if (encoder()(&tin, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(in), din, sin, bin, ones,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        tc_note("activation tensor map rejected");
        return false;
    }
    const cuuint64_t dw[3] = {(cuuint64_t)kCh, (cuuint64_t)kCh, (cuuint64_t)kTapsTC};
    const cuuint64_t sw[2] = {(cuuint64_t)kRow, (cuuint64_t)kTapW};
    const cuuint32_t bw[3] = {(cuuint32_t)kCh, (cuuint32_t)kCh, (cuuint32_t)kTapsTC};
    if (encoder()(&twt, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16 *>(w), dw, sw, bw, ones,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        tc_note("weight tensor map rejected");
        return false;
    }
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int ntiles = B * (H / TH) * (W / TW);
    const int grid = ntiles < sms ? ntiles : sms;
    if (rows_mode() && TW == kTM && dil >= 1 && dil <= 8 && (out_f32 || !((uintptr_t)out & 15))) {
        CUtensorMap trow, tout;
        const cuuint32_t brow[4] = {(cuuint32_t)kCh, (cuuint32_t)(TW + 2 * dil), 1, 1};
        const cuuint32_t bout[4] = {(cuuint32_t)kCh, 32, 1, 1};  // one warp's 32 pixels
        // The output map is only used for BF16 output (same NHWC shape as the
        // input); for FP32 output it is encoded over the input and not used.
        void *obase = out_f32 ? const_cast<__nv_bfloat16 *>(in) : static_cast<void *>(out);
        if (encoder()(&trow, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(in), din, sin, brow, ones,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
            encoder()(&tout, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, obase, din, sin, bout, ones,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS) {
            kRowsKernel<<<grid, RowsCfg::kThreads, RowsCfg::kSmem>>>(trow, twt, tout, bias, out_f32, H, W, dil,
                                                                          relu, ntiles);
            const cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) return true;
            tc_note(cudaGetErrorString(e));
            return false;
        }
    }
    k_conv_tc<<<grid, 160, kSmemTC>>>(tin, twt, bias, out, out_f32, H, W, TW, TH, dil, relu, ntiles);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {  // not launched: the caller's kernel runs instead
        tc_note(cudaGetErrorString(err));
        return false;
    }
    return true;
}

// Weight gradient on the tcgen05 kernel when W is a multiple of 64: returns
// the number of blocks whose partials it wrote (at most max_blocks), or 0 to
// leave it to the caller's kernel.
int wgrad_tc(const __nv_bfloat16 *in, const __nv_bfloat16 *g, float *part, int max_blocks, int B, int H, int W,
             int dil) {
    if (!tc_enabled() || W % kWSeg != 0) return 0;
    static int wg_ok[kMaxDev] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) return 0;
    if (wg_ok[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemWG);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_wgrad_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemWR);
        if (e != cudaSuccess) {
            tc_note(cudaGetErrorString(e));
            cudaGetLastError();
        }
        wg_ok[dev] = e == cudaSuccess ? 1 : -1;
    }
    if (wg_ok[dev] != 1) return 0;
    if (((uintptr_t)in & 15) || ((uintptr_t)g & 15)) return 0;
    CUtensorMap tin, tgm;
    const cuuint64_t dims[4] = {(cuuint64_t)kCh, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[3] = {(cuuint64_t)kRow, (cuuint64_t)W * kRow, (cuuint64_t)H * W * kRow};
    const cuuint32_t box[4] = {(cuuint32_t)kCh, (cuuint32_t)kWSeg, 1, 1};
    const cuuint32_t ones[4] = {1, 1, 1, 1};
    if (encoder()(&tin, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(in), dims, strides, box,
                  ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        encoder()(&tgm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(g), dims, strides, box,
                  ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        tc_note("weight-gradient tensor map rejected");
        return 0;
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
    const int nseg = B * H * (W / kWSeg);
    int grid = nseg < sms ? nseg : sms;
    if (grid > max_blocks) grid = max_blocks;
    if (grid < 1) return 0;
    if (rows_mode() && dil >= 1 && dil <= 8) {
        // Three staged rows per segment (box of 64 + 2d pixels).
        CUtensorMap trow;
        const cuuint32_t brow[4] = {(cuuint32_t)kCh, (cuuint32_t)(kWSeg + 2 * dil), 1, 1};
        if (encoder()(&trow, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(in), dims, strides,
                      brow, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS) {
            k_wgrad_rows<<<grid, kWRowThreads, kSmemWR>>>(trow, tgm, part, H, W, dil, nseg);
            const cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) return grid;
            tc_note(cudaGetErrorString(e));
            return 0;
        }
    }
    k_wgrad_tc<<<grid, 160, kSmemWG>>>(tin, tgm, part, H, W, dil, nseg);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        tc_note(cudaGetErrorString(err));
        return 0;
    }
    return grid;
}

// Reads and clears the flag of a timed-out wait in k_conv_tc (a sync point).
int conv_tc_status() {
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)) != cudaSuccess) return -1001;
    if (v) cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
    return v ? -1012 : 0;
}

}  // namespace seednet
}  // namespace trlb

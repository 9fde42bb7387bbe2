// wgrad_tc.cuh -- the weight gradient of a 3x3x3 convolution with 16 input
// and 16 output channels on the 5th-generation tensor cores.
//
//   dW[t][ci][co] = sum over cells c of G[c][co] * X[c + off(t)][ci]
//
// with X the layer's input activations and G the gradient with respect to its
// pre-activation, both channels-last BF16 (16 channels = 32 bytes per cell),
// and off(t) = dx + dy*nx + dz*nx*ny.  As a GEMM the cells are the reduction
// (K) dimension: D[m][n] = sum_k A[m][k] B[n][k] with m = (tap, ci), n = co,
// k = cell, FP32 in tensor memory.
//
// Operands.  The 3-D TMA view of an activation array used by conv_tc.cuh --
// (8 channels, rows at 32 bytes, 2 channel groups at 16 bytes) -- with box
// {8, 128, 2} lands 128 cells as [group][cell][8 channels]: 8 cells x 16 bytes
// form one 128-byte core matrix with the CHANNELS contiguous, which is the
// no-swizzle MN-major operand layout (channels on M or N, cells on K; K groups
// of 8 cells 128 bytes apart = LBO, channel groups 2048 bytes apart = SBO).
// Operand A of one MMA (M = 128) is 8 taps x 16 channels: the windows
// X[c0 + off(t) + 0..127] of 8 taps loaded as 8 such boxes back to back, so
// the 16 channel groups (tap, group) follow each other 2048 bytes apart.
// Operand B (N = 16) is the box G[c0 + 0..127].  One MMA covers K = 16 cells
// (descriptor start + 256 bytes per step), 8 MMAs a tile of 128 cells, and
// the 27 taps take 4 tap groups (the last one pads with tap 26 again; its
// extra rows are never read).  Each tap group accumulates into its own 16
// TMEM columns over every tile the CTA takes; at the end the four
// accumulators are the CTA's partial dW.
//
// Windows that start before the array or run past it read zeros (TMA fill).
// Batched grids are consecutive in the array; a window crossing into the next
// member meets only G = 0 there (G vanishes off the interior, and an interior
// cell's 27 neighbours lie inside its own member).
//
// Warp roles (192 threads): warp 4 lane 0 issues the TMA loads, warp 5 lane 0
// the MMAs, warps 0-3 read the accumulators out at the end (TMEM lanes
// 32w..32w+31).  mbarriers: full[s] (a stage's 9 boxes landed), empty[s] (the
// MMAs reading the stage completed), done (every MMA completed).  Every wait
// is bounded; a role that gives up raises *err, and the producer and the MMA
// issuer still wait for their own copies and MMAs before the CTA leaves.
#pragma once

#include "conv_tc.cuh"

namespace piro {
namespace tc {

constexpr int kWgRows = 128;                   // cells per tile (8 MMAs of K = 16)
constexpr int kWgBox = kWgRows * 32;           // one {8, 128, 2} box: 4096 bytes
constexpr int kWgTaps = 8;                     // taps per MMA (M = 8 x 16)
constexpr int kWgGroups = 4;                   // tap groups covering the 27 taps
constexpr int kWgStageBytes = (kWgTaps + 1) * kWgBox;  // 8 X windows + the G tile: 36 KB
constexpr int kWgStages = 4;
constexpr int kWgThreads = 192;
constexpr int kWgBarOff = kWgStages * kWgStageBytes;
constexpr int kWgSmemBytes = kWgBarOff + (2 * kWgStages + 2) * 8 + 16 + 128;

// Instruction descriptor of kind::f16 with both operands MN-major (bits 15
// and 16): FP32 accumulator, BF16 A and B, N = 16, M = 128.
constexpr uint32_t kIdescMN = kIdesc | (1u << 15) | (1u << 16);

struct WgArgs {
    int nx;
    int64_t nxy;
    int64_t ntiles;   // tiles of kWgRows cells over all rows of the arrays
    int ci_n, co_n;   // channels kept in the partial layout (the layer's CI and CO)
    float *partials;  // [gridDim.x][27 * ci_n * co_n], per CTA: (t * ci_n + ci) * co_n + co
    int *err;
};

__device__ __forceinline__ int64_t wg_tap_off(int t, int nx, int64_t nxy)
{
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    return (int64_t)dx + (int64_t)dy * nx + (int64_t)dz * nxy;
}

__global__ void __launch_bounds__(kWgThreads, 1) k_wgrad_tc(const __grid_constant__ CUtensorMap xmap,
                                                             const __grid_constant__ CUtensorMap gmap, WgArgs a)
{
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    const uint32_t stage_s = smem_u32(sm);
    const uint32_t bar_s = stage_s + kWgBarOff;  // full[S], empty[S], done, drain
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + kWgBarOff + (2 * kWgStages + 2) * 8);
    auto full = [&](int i) { return bar_s + 8u * i; };
    auto empty = [&](int i) { return bar_s + 8u * (kWgStages + i); };
    const uint32_t done_s = bar_s + 8u * (2 * kWgStages);
    const uint32_t drain_s = bar_s + 8u * (2 * kWgStages + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t my_tiles = (int64_t)blockIdx.x < a.ntiles ? (a.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t items = my_tiles * kWgGroups;  // (tile, tap group) pairs, tile-major

    if (threadIdx.x == 0) {
        for (int i = 0; i < kWgStages; ++i) {
            mbar_init(full(i), 1);
            mbar_init(empty(i), 1);
        }
        mbar_init(done_s, 1);
        mbar_init(drain_s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(64)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(tmem_slot);
    bool mma_ok = items > 0;

    if (warp == 4) {
        if (lane == 0 && items > 0) {
            int64_t i = 0;
            for (; i < items; ++i) {
                const int s = (int)(i % kWgStages);
                if (i >= kWgStages && !mbar_wait(empty(s), (uint32_t)(((i / kWgStages) - 1) & 1), a.err)) break;
                const int64_t tile = blockIdx.x + (i / kWgGroups) * gridDim.x;
                const int tg = (int)(i % kWgGroups);
                const int64_t c0 = tile * kWgRows;
                const uint32_t st = stage_s + (uint32_t)s * kWgStageBytes;
                mbar_expect_tx(full(s), kWgStageBytes);
                for (int tl = 0; tl < kWgTaps; ++tl) {
                    const int t = tg * kWgTaps + tl < 27 ? tg * kWgTaps + tl : 26;
                    tma_load_3d(st + tl * kWgBox, &xmap, full(s), 0, (int)(c0 + wg_tap_off(t, a.nx, a.nxy)), 0);
                }
                tma_load_3d(st + kWgTaps * kWgBox, &gmap, full(s), 0, (int)c0, 0);
            }
            // each stage's latest load is the only one that can still be in flight
            for (int64_t q = i - kWgStages < 0 ? 0 : i - kWgStages; q < i; ++q)
                mbar_drain(full((int)(q % kWgStages)), (uint32_t)((q / kWgStages) & 1));
        }
    } else if (warp == 5) {
        if (lane == 0 && items > 0) {
            for (int64_t i = 0; i < items && mma_ok; ++i) {
                const int s = (int)(i % kWgStages);
                if (!(mma_ok = mbar_wait(full(s), (uint32_t)((i / kWgStages) & 1), a.err))) break;
                fence_after();
                const int tg = (int)(i % kWgGroups);
                const uint32_t st = stage_s + (uint32_t)s * kWgStageBytes;
                const uint32_t d_tmem = tmem + (uint32_t)(tg * 16);
#pragma unroll
                for (int ks = 0; ks < kWgRows / 16; ++ks) {
                    const uint64_t ad = desc_nosw(st + ks * 256, 128, kWgBox / 2);
                    const uint64_t bd = desc_nosw(st + kWgTaps * kWgBox + ks * 256, 128, kWgBox / 2);
                    const uint32_t acc = (i >= kWgGroups || ks > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                        "l"(ad), "l"(bd), "r"(kIdescMN), "r"(acc)
                        : "memory");
                }
                mma_commit(empty(s));
            }
            mma_commit(done_s);
            // every MMA issued here has completed before TMEM is read or released
            mma_commit(drain_s);
            mbar_drain(drain_s, 0);
        }
    } else {
        // read-out: warp w holds accumulator rows m = 32w .. 32w+31, m = tl * 16 + ci
        const int m = warp * 32 + lane;
        const int tl = m / 16, ci = m % 16;
        float *pb = a.partials + (int64_t)blockIdx.x * 27 * a.ci_n * a.co_n;
        bool got = items > 0 && mbar_wait(done_s, 0, a.err);
        got = __all_sync(0xffffffffu, got);  // tcgen05.ld is warp-wide: the warp reads together or not at all
        if (got) fence_after();
        for (int tg = 0; tg < kWgGroups; ++tg) {
            uint32_t v[16];
            if (got) {
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(tg * 16), v);
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) v[k] = 0u;  // a CTA without tiles contributes zeros
            }
            const int t = tg * kWgTaps + tl;
            if (t < 27 && ci < a.ci_n) {
#pragma unroll
                for (int co = 0; co < 16; ++co)
                    if (co < a.co_n) pb[((int64_t)t * a.ci_n + ci) * a.co_n + co] = __uint_as_float(v[co]);
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64) : "memory");
    }
}

}  // namespace tc
}  // namespace piro

// conv_tc.cuh -- the 3x3x3 convolution with 16 input and 16 output channels
// (the two middle layers of the learned preconditioner) as an implicit GEMM on
// the 5th-generation tensor cores: tcgen05.mma (kind::f16, BF16 operands,
// FP32 accumulation in tensor memory), operands staged by TMA.
//
// Activations are channels-last BF16, 16 channels = 32 bytes per cell, on the
// ghost-inclusive grid; boundary cells hold zeros.  An output tile is 128
// consecutive cells (MMA M = 128), N = 16 output channels, and the K loop is
// the 27 taps x 16 input channels: 27 MMAs of K = 16.
//
// Operand A of tap (dx, dy, dz) is the input at rows c0 + dx + dy*nx + dz*nx*ny
// + [0, 128).  For each (dy, dz) one "line block" of 130 rows (the tile and one
// row each side) is loaded once; the three dx taps read it at row offsets 0, 1,
// 2.  The line block sits in shared memory in the no-swizzle K-major layout of
// the MMA -- [channel group 2][130 rows][8 channels], so an 8-row x 16-byte core
// matrix is 128 contiguous bytes, consecutive rows are 16 bytes apart (SBO =
// 128 bytes per 8 rows) and the two channel groups LBO = 130*16 bytes apart --
// and a row offset is a 16-byte move of the descriptor's start address.  TMA
// writes exactly that layout from a 3-D view of the activations:
// (8 channels, rows with a 32-byte stride, 2 groups with a 16-byte stride),
// box {8, 130, 2}.  Rows outside the array read as zeros (TMA fill).
//
// A CTA owns one 128-cell column and marches it along z: the 9 line blocks of
// tile z are the 3 of each of the planes z-1, z, z+1, so each new tile loads 3
// line blocks (one plane) while the others stay resident: a ring of 4 planes
// (3 in use, 1 loading).  L2 -> SM traffic is about 3 * 130/128 * 32 bytes
// per output cell, against 27 * 32 for a load per tap.
//
// Batched grids (blockIdx.y = member b) are consecutive in the array: rows
// b*N .. b*N + N - 1.
//
// Warp roles (192 threads): warps 0-3 read the accumulator (TMEM lanes
// 32w..32w+31), apply GELU and store; warp 4 lane 0 issues the TMA loads;
// warp 5 lane 0 issues the MMAs.  Two TMEM accumulators (2 x 16 columns)
// overlap a tile's epilogue with the next tile's MMAs (four measured slower).  mbarriers: full[slot]
// (TMA bytes landed), empty[slot] (the MMAs reading a plane completed),
// acc_full[b] (a tile's MMAs completed), acc_empty[b] (its epilogue read it).
// Every wait is bounded: on timeout the kernel raises *err and every role
// leaves its loop.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace piro {
namespace tc {

typedef __nv_bfloat16 bf16;

constexpr int kRows = 128;                    // output cells per tile (MMA M)
constexpr int kLineRows = kRows + 2;          // rows of a line block
constexpr int kLineBytes = kLineRows * 32;    // 4160
constexpr int kLineStride = 4224;             // 128-byte aligned slot of a line block
constexpr int kSlots = 4;                     // planes resident (3 read by a tile, 1 loading)
constexpr int kPlaneBytes = 3 * kLineStride;  // the 3 line blocks (dy = -1, 0, 1) of a plane
constexpr int kWBytes = 27 * 512;             // one layer's weights: per tap [group][co 16][8 ci] BF16
constexpr int kThreads = 192;
constexpr int kBarOff = kSlots * kPlaneBytes + kWBytes;
constexpr int kAcc = 2;                       // TMEM accumulators (16 columns each) per CTA
constexpr int kBarSlots = 2 * kSlots + 2 * kAcc + 1;  // full, empty, acc_full, acc_empty, drain
constexpr int kSmemBytes = kBarOff + kBarSlots * 8 + 16 + 128;  // + barriers, TMEM address, alignment slack
constexpr long long kSpin = 1ll << 24;        // polls before a wait gives up

struct Args {
    GridDiv g;
    int64_t N, nxy;
    int ncol, zchunk;
    const bf16 *wpk;   // packed weights of this layer
    bf16 *out;         // output activations (epilogues 0, 2) or gradient (epilogue 3)
    float *zout;       // FP32 output channel 0 (epilogue 1)
    const double *rr;  // epilogue 1: output scale sqrt(rr[b] / n_int) (NULL: 1)
    double n_int;
    const int *skip;   // launch returns at once when set (may be NULL)
    int *err;          // raised on a timed-out wait
    bf16 *yout;        // epilogue 2: the pre-activation bf16(acc)
    const bf16 *yprev; // epilogue 3: the previous layer's pre-activation
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity; false on timeout or when
// another role already gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err)
{
    for (long long i = 0; i < kSpin; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 1023) == 1023 && *((volatile int *)err)) return false;
    }
    atomicExch(err, 1);
    return false;
}

// Wait for a phase that is certain to complete (copies or MMAs this CTA
// issued itself), with its own bound so that a role which gave up on a
// partner still leaves nothing in flight behind it.
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kSpin; ++i)
        if (mbar_try_wait(bar, parity)) return;
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address, LBO
// (between the two 8-element K groups), SBO (between 8-row groups), all in
// 16-byte units; bits 46-47 = 1 (the tcgen05 descriptor version).
__device__ __forceinline__ uint64_t desc_nosw(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A
// and B (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at
// bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// GELU in its tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh(sqrt(2/pi)
// (x + 0.044715 x^3))), with the hardware tanh.approx (one instruction; the
// erf form costs several special-function operations per element and made
// this epilogue the kernel's bottleneck).
__device__ __forceinline__ float gelu_tc(float x)
{
    float t;
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return 0.5f * x * (1.0f + t);
}

// GELU'(x) of the tanh form above: 0.5 (1 + t) + 0.5 x (1 - t^2) c (1 + 3 a x^2).
__device__ __forceinline__ float gelu_d_tc(float x)
{
    float t;
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}

// kEpi 0: GELU, 16 BF16 channels out (hidden layers); 1: output channel 0 in
// FP32 times the batch member's scale (the last layer, N padded to 16);
// 2 (training forward): the pre-activation y = bf16(acc) to yout and GELU(y)
// to out; 3 (data gradient, run with the transposed, tap-reversed weights):
// out = bf16(acc * GELU'(yprev)), the gradient with respect to the previous
// layer's pre-activation.  Every epilogue writes zeros on non-interior cells.
template <int kEpi>
__global__ void __launch_bounds__(kThreads, 3) k_conv16_tc(const __grid_constant__ CUtensorMap xmap, Args a)
{
    if (a.skip && *((volatile const int *)a.skip)) return;
    extern __shared__ unsigned char smem_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    const uint32_t planes_s = smem_u32(sm);
    const uint32_t w_s = planes_s + kSlots * kPlaneBytes;
    const uint32_t bar_s = planes_s + kBarOff;  // full[kSlots], empty[kSlots], acc_full[kAcc], acc_empty[kAcc], drain
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + kBarOff + kBarSlots * 8);
    auto full = [&](int i) { return bar_s + 8u * i; };
    auto empty = [&](int i) { return bar_s + 8u * (kSlots + i); };
    auto accf = [&](int b) { return bar_s + 8u * (2 * kSlots + b); };
    auto acce = [&](int b) { return bar_s + 8u * (2 * kSlots + kAcc + b); };
    const uint32_t drain_s = bar_s + 8u * (2 * kSlots + 2 * kAcc);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t boff = (int64_t)blockIdx.y * a.N;  // batch member: rows b*N ..
    const int col = blockIdx.x % a.ncol;
    const int zb = 1 + (blockIdx.x / a.ncol) * a.zchunk;
    const int ze = min(zb + a.zchunk, a.g.nz - 1);
    const int P = ze - zb;  // tiles (output planes) of this CTA

    // weights -> shared memory (generic proxy), then made visible to the tensor cores
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.wpk);
        uint4 *dst = reinterpret_cast<uint4 *>(sm + kSlots * kPlaneBytes);
        for (int i = threadIdx.x; i < kWBytes / 16; i += kThreads) dst[i] = src[i];
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kSlots; ++i) {
            mbar_init(full(i), 1);
            mbar_init(empty(i), 1);
        }
        for (int b = 0; b < kAcc; ++b) {
            mbar_init(accf(b), 1);
            mbar_init(acce(b), 4);
        }
        mbar_init(drain_s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kAcc * 16)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(tmem_slot);

    if (P > 0) {
        if (warp == 4) {
            if (lane == 0) {
                // producer: planes zb-1 .. ze, three line blocks each
                int p = 0;
                for (; p < P + 2; ++p) {
                    const int slot = p % kSlots;
                    if (p >= kSlots && !mbar_wait(empty(slot), ((p / kSlots) - 1) & 1, a.err)) break;
                    const int64_t L = zb - 1 + p;
                    mbar_expect_tx(full(slot), 3 * kLineBytes);
                    for (int dy = 0; dy < 3; ++dy) {
                        const int64_t r = boff + L * a.nxy + (int64_t)col * kRows - 1 + (int64_t)(dy - 1) * a.g.nx;
                        tma_load_3d(planes_s + slot * kPlaneBytes + dy * kLineStride, &xmap, full(slot), 0, (int)r,
                                    0);
                    }
                }
                // no copy may land after the CTA has left, whatever the other
                // roles did: wait for each slot's latest load
                for (int q = p - kSlots < 0 ? 0 : p - kSlots; q < p; ++q) mbar_drain(full(q % kSlots), (q / kSlots) & 1);
            }
        } else if (warp == 5) {
            if (lane == 0) {
                int waited = 0;
                bool ok = true;
                for (int j = 0; j < P && ok; ++j) {
                    while (ok && waited < j + 3) {
                        ok = mbar_wait(full(waited % kSlots), (waited / kSlots) & 1, a.err);
                        ++waited;
                    }
                    const int buf = j % kAcc;
                    if (ok && j >= kAcc) ok = mbar_wait(acce(buf), ((j / kAcc) - 1) & 1, a.err);
                    if (!ok) break;
                    fence_after();
                    const uint32_t d_tmem = tmem + (uint32_t)(buf * 16);
#pragma unroll 1
                    for (int dz = 0; dz < 3; ++dz) {
                        const uint32_t pbase = planes_s + ((j + dz) % kSlots) * kPlaneBytes;
#pragma unroll
                        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                            for (int dx = 0; dx < 3; ++dx) {
                                const int tap = dz * 9 + dy * 3 + dx;
                                const uint64_t ad =
                                    desc_nosw(pbase + dy * kLineStride + dx * 16, kLineRows * 16, 128);
                                const uint64_t bd = desc_nosw(w_s + tap * 512, 256, 128);
                                mma_bf16(d_tmem, ad, bd, tap > 0 ? 1u : 0u);
                            }
                    }
                    mma_commit(accf(buf));
                    mma_commit(empty(j % kSlots));  // plane z-1 is read by no later tile
                }
                // every MMA issued here has completed before TMEM is released
                mma_commit(drain_s);
                mbar_drain(drain_s, 0);
            }
        } else {
            // the boundary planes z = 0 and nz - 1 of this column hold zeros
            // in every output (no tile computes them; a buffer reused for
            // another grid must not keep values there)
            for (int e = 0; e < 2; ++e) {
                if ((e == 0 && zb != 1) || (e == 1 && ze != a.g.nz - 1)) continue;
                const int64_t inplane = (int64_t)col * kRows + warp * 32 + lane;
                if (inplane >= a.nxy) continue;
                const int64_t c = (e == 0 ? 0 : (int64_t)(a.g.nz - 1) * a.nxy) + inplane;
                if (kEpi == 1) {
                    a.zout[boff + c] = 0.0f;
                } else {
                    uint4 *o = reinterpret_cast<uint4 *>(a.out + (boff + c) * 16);
                    o[0] = make_uint4(0, 0, 0, 0);
                    o[1] = make_uint4(0, 0, 0, 0);
                    if (kEpi == 2) {
                        uint4 *oy = reinterpret_cast<uint4 *>(a.yout + (boff + c) * 16);
                        oy[0] = make_uint4(0, 0, 0, 0);
                        oy[1] = make_uint4(0, 0, 0, 0);
                    }
                }
            }
            // epilogue: warp w holds tile rows 32w .. 32w+31
            for (int j = 0; j < P; ++j) {
                const int buf = j % kAcc;
                if (!mbar_wait(accf(buf), (j / kAcc) & 1, a.err)) break;
                fence_after();
                uint32_t v[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * 16), v);
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acce(buf));
                const int64_t c = (int64_t)(zb + j) * a.nxy + (int64_t)col * kRows + warp * 32 + lane;
                if (kEpi == 1) {
                    if (c < a.N) {
                        float sc = 1.0f;
                        if (a.rr) sc = (float)sqrt(a.rr[blockIdx.y] / a.n_int);
                        a.zout[boff + c] = a.g.interior(c) ? __uint_as_float(v[0]) * sc : 0.0f;
                    }
                } else if (kEpi == 3) {
                    if (c < a.N) {
                        uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                        if (a.g.interior(c)) {
                            const uint4 *yp = reinterpret_cast<const uint4 *>(a.yprev + (boff + c) * 16);
                            const uint4 u0 = yp[0], u1 = yp[1];
                            const uint32_t yw[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
                            for (int k = 0; k < 8; ++k) {
                                const float2 y = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&yw[k]));
                                const __nv_bfloat162 h = __floats2bfloat162_rn(__uint_as_float(v[2 * k]) * gelu_d_tc(y.x),
                                                                               __uint_as_float(v[2 * k + 1]) * gelu_d_tc(y.y));
                                w[k] = *reinterpret_cast<const uint32_t *>(&h);
                            }
                        }
                        uint4 *o = reinterpret_cast<uint4 *>(a.out + (boff + c) * 16);
                        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
                        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
                    }
                } else if (c < a.N) {
                    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0}, yw[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    if (a.g.interior(c)) {
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const float y0 = __bfloat162float(__float2bfloat16_rn(__uint_as_float(v[2 * k])));
                            const float y1 = __bfloat162float(__float2bfloat16_rn(__uint_as_float(v[2 * k + 1])));
                            const __nv_bfloat162 h = __floats2bfloat162_rn(gelu_tc(y0), gelu_tc(y1));
                            w[k] = *reinterpret_cast<const uint32_t *>(&h);
                            if (kEpi == 2) {
                                const __nv_bfloat162 hy = __floats2bfloat162_rn(y0, y1);
                                yw[k] = *reinterpret_cast<const uint32_t *>(&hy);
                            }
                        }
                    }
                    uint4 *o = reinterpret_cast<uint4 *>(a.out + (boff + c) * 16);
                    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
                    if (kEpi == 2) {
                        uint4 *oy = reinterpret_cast<uint4 *>(a.yout + (boff + c) * 16);
                        oy[0] = make_uint4(yw[0], yw[1], yw[2], yw[3]);
                        oy[1] = make_uint4(yw[4], yw[5], yw[6], yw[7]);
                    }
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kAcc * 16) : "memory");
    }
}

}  // namespace tc
}  // namespace piro

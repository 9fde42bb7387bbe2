// common.cuh -- shared helpers of the piro_b200 CUDA library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <atomic>
#include <mutex>
#include <string>

#include "piro.h"

namespace piro {

// Per-thread message for piro_last_error().
void set_error(const char *fmt, ...);

inline cudaStream_t as_stream(piro_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// B200: 148 SMs; launch grids are sized against the device's SM count.
int sm_count();

// The poll count of the bounded device waits that piro_set_wait_limit sets,
// or `builtin` when none is set.
long long wait_limit(long long builtin);

__host__ __device__ inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Grid size for a grid-stride loop over n items with `per_block` items per block.
inline unsigned grid_for(int64_t n, int64_t per_block, int blocks_per_sm = 8)
{
    int64_t want = cdiv(n, per_block);
    int64_t cap = (int64_t)sm_count() * blocks_per_sm * 16;
    if (want < 1) want = 1;
    return (unsigned)(want < cap ? want : cap);
}

// One-time setup per (call site, device): kernel attributes, occupancy
// figures, small device buffers.  Safe when several host threads drive the
// library; a setup that fails is tried again on the next call.
constexpr int kMaxDevices = 64;
struct DeviceOnce {
    std::mutex mu;
    std::atomic<bool> done[kMaxDevices] = {};
};

template <typename F>
int device_once(DeviceOnce &once, int dev, F &&init)
{
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index %d out of range", dev);
        return PIRO_ERR_CUDA;
    }
    if (once.done[dev].load(std::memory_order_acquire)) return PIRO_OK;
    std::lock_guard<std::mutex> lock(once.mu);
    if (once.done[dev].load(std::memory_order_relaxed)) return PIRO_OK;
    const int rc = init();
    if (rc == PIRO_OK) once.done[dev].store(true, std::memory_order_release);
    return rc;
}

}  // namespace piro

#define PIRO_CHECK_LAUNCH(what)                                                              \
    do {                                                                                     \
        cudaError_t e_ = cudaGetLastError();                                                 \
        if (e_ != cudaSuccess) {                                                             \
            piro::set_error("%s: %s", what, cudaGetErrorString(e_));                        \
            return PIRO_ERR_CUDA;                                                            \
        }                                                                                    \
    } while (0)

#define PIRO_CUDA(call)                                                                      \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            piro::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                            __LINE__);                                                       \
            return PIRO_ERR_CUDA;                                                            \
        }                                                                                    \
    } while (0)

#define PIRO_ARG(cond, msg)                         \
    do {                                            \
        if (!(cond)) {                              \
            piro::set_error("%s", msg);             \
            return PIRO_ERR_ARG;                    \
        }                                           \
    } while (0)

// Device-side helpers --------------------------------------------------------
namespace piro {

// Reference arithmetic without contraction: (a*b) rounded, then +.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }

// Division by a runtime constant for numerators below 2^31: with
// l = ceil(log2 d) and m = ceil(2^(31+l) / d) (< 2^32), n / d =
// (n * m) >> (31 + l) exactly, since n*(m - 2^(31+l)/d) / 2^(31+l) < 1/d
// (round-up reciprocal method, Granlund & Montgomery 1994).
struct FastDiv {
    uint32_t d, m, sh;  // sh = l - 1 applied after the high-word multiply; d == 1 handled apart
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t div) : d(div), m(0), sh(0)
    {
        uint32_t l = 0;
        while ((1ull << l) < div) ++l;
        if (div > 1) {
            m = (uint32_t)(((1ull << (31 + l)) + div - 1) / div);
            sh = l - 1;
        }
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const { return d == 1 ? n : __umulhi(n, m) >> sh; }
};

// x mod d for 64-bit x and d >= 1 by a multiply-high with floor((2^64-1)/d)
// (Barrett reduction): the estimated quotient is at most 2 below the true one,
// so two conditional subtractions give the exact remainder.
struct ModU64 {
    uint64_t d, m;
    ModU64() = default;
    __host__ explicit ModU64(uint64_t div) : d(div), m(div > 1 ? ~0ull / div : 0) {}
    __device__ __forceinline__ uint64_t mod(uint64_t x) const
    {
        if (d == 1) return 0;
        uint64_t r = x - __umul64hi(x, m) * d;
        r = r >= d ? r - d : r;
        return r >= d ? r - d : r;
    }
};

// Grid with fast coordinate decomposition of a linear index i < 2^31.
struct GridDiv {
    int nx, ny, nz;
    FastDiv fx, fxy;
    GridDiv() = default;
    __host__ GridDiv(int x, int y, int z) : nx(x), ny(y), nz(z), fx((uint32_t)x), fxy((uint32_t)x * (uint32_t)y) {}
    __device__ __forceinline__ void coords(uint32_t i, int &x, int &y, int &z) const
    {
        const uint32_t zz = fxy.div(i);
        const uint32_t rem = i - zz * fxy.d;
        const uint32_t yy = fx.div(rem);
        z = (int)zz;
        y = (int)yy;
        x = (int)(rem - yy * fx.d);
    }
    // interior test of SpMVCSR.cl:29-32 (ghost-inclusive sizes)
    __device__ __forceinline__ bool interior(int64_t i) const
    {
        int x, y, z;
        coords((uint32_t)i, x, y, z);
        return x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1;
    }
};

// Interior test of SpMVCSR.cl:29-32 with general 64-bit division (one-off use).
__device__ __forceinline__ bool interior(int64_t i, int nx, int ny, int nz)
{
    int64_t sxy = (int64_t)nx * ny;
    int z = (int)(i / sxy);
    int64_t rem = i - (int64_t)z * sxy;
    int y = (int)(rem / nx);
    int x = (int)(rem - (int64_t)y * nx);
    return x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1;
}

// 1/a by PTX rcp.approx (max error about 1 ulp): for the weights 1/alpha of
// CG dot products, which need no correct rounding.
__device__ __forceinline__ float rcp_approx(float a)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_sum_i(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace piro

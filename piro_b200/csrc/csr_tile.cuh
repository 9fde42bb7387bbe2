// csr_tile.cuh -- staging of a CSR row tile's col/val range in shared memory.
#pragma once
#include "common.cuh"

namespace piro {

constexpr int kTileRows = 256;
constexpr int kTileCap = 2048;  // staged nonzeros per tile (7-point rows: <= 1792)

// Stage [s, e) of col/val into shared memory; 16-byte loads for the aligned
// middle, scalar loads for the ragged ends.
__device__ __forceinline__ void stage_tile(const int32_t *__restrict__ col, const float *__restrict__ val, int64_t s,
                                           int64_t e, int32_t *s_col, float *s_val)
{
    const int64_t a0 = (s + 3) & ~(int64_t)3;
    const int64_t a1 = e & ~(int64_t)3;
    if (a0 >= a1) {
        for (int64_t k = s + threadIdx.x; k < e; k += blockDim.x) {
            s_col[k - s] = __ldcs(col + k);
            s_val[k - s] = __ldcs(val + k);
        }
        return;
    }
    for (int64_t k = s + threadIdx.x; k < a0; k += blockDim.x) {
        s_col[k - s] = __ldcs(col + k);
        s_val[k - s] = __ldcs(val + k);
    }
    const int64_t nv = (a1 - a0) >> 2;
    const int4 *c4 = reinterpret_cast<const int4 *>(col + a0);
    const float4 *v4 = reinterpret_cast<const float4 *>(val + a0);
    const int o = (int)(a0 - s);
    for (int64_t t = threadIdx.x; t < nv; t += blockDim.x) {
        int4 c = __ldcs(c4 + t);
        float4 v = __ldcs(v4 + t);
        int b = o + (int)(t << 2);
        s_col[b] = c.x; s_col[b + 1] = c.y; s_col[b + 2] = c.z; s_col[b + 3] = c.w;
        s_val[b] = v.x; s_val[b + 1] = v.y; s_val[b + 2] = v.z; s_val[b + 3] = v.w;
    }
    for (int64_t k = a1 + threadIdx.x; k < e; k += blockDim.x) {
        s_col[k - s] = __ldcs(col + k);
        s_val[k - s] = __ldcs(val + k);
    }
}

}  // namespace piro

// csr_tile.cuh -- pipelined streaming of CSR row tiles through shared memory.
//
// A persistent block walks tiles of kTileRows consecutive rows.  While the
// threads reduce tile t (one row per thread, storage order, so results keep
// the reference's summation order), the tile's successor streams in:
// cp.async (16-byte, L2-only, zero-filled past the array end) copies tile
// t+1's col/val range and tile t+2's rowptr slice into the next of three
// shared-memory stages.  HBM therefore always has the next tile's bytes in
// flight instead of idling during the gathers of the current one.
//
// Shared memory per block: 3 stages x (rowptr 1040 B + col/val 2 x 8224 B)
// = 52.5 KB; four blocks fill an SM.  Tiles whose nonzeros exceed kTileCap
// (rows much longer than a 7-point stencil's) fall back to direct loads.
#pragma once
#include "common.cuh"

namespace piro {

constexpr int kTileRows = 256;
constexpr int kTileCap = 2048;           // staged nonzeros per tile (7-point rows: <= 1792)
constexpr int kStages = 3;
constexpr int kRpWords = kTileRows + 4;  // rowptr slice rounded to 16 B
constexpr int kCvWords = kTileCap + 8;   // col/val slice + alignment slack

struct CsrStages {
    int32_t rp[kStages][kRpWords];
    int32_t col[kStages][kCvWords];
    float val[kStages][kCvWords];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Copy words [g0, g0 + 4*nchunks) of src (length len words) into dst, 16 B at
// a time; bytes at or past len are zero-filled and never read.
__device__ __forceinline__ void copy_words(int32_t *dst, const int32_t *src, int64_t g0, int nchunks, int64_t len)
{
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x) {
        const int64_t g = g0 + 4 * (int64_t)c;
        int64_t rem = len - g;
        const int bytes = rem >= 4 ? 16 : rem > 0 ? (int)rem * 4 : 0;
        cp_async16(dst + 4 * c, bytes ? (const void *)(src + g) : (const void *)src, bytes);
    }
}

// Issue the rowptr slice of tile `tile` into stage `st`.
__device__ __forceinline__ void issue_rp(CsrStages &sm, int st, int64_t tile, int64_t ntiles, int64_t N,
                                         const int32_t *__restrict__ rowptr)
{
    if (tile >= ntiles) return;
    const int64_t r0 = tile * kTileRows;
    copy_words(sm.rp[st], rowptr, r0, kRpWords / 4, N + 1);
}

// Issue the col/val slice of tile `tile` (its rowptr slice is in stage `st`).
__device__ __forceinline__ void issue_cv(CsrStages &sm, int st, int64_t tile, int64_t ntiles, int64_t N, int64_t nnz,
                                         const int32_t *__restrict__ col, const float *__restrict__ val)
{
    if (tile >= ntiles) return;
    const int64_t r0 = tile * kTileRows;
    const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
    const int64_t s = sm.rp[st][0], e = sm.rp[st][nrows];
    if (e - s > kTileCap) return;  // long rows: computed from global memory
    const int64_t a0 = s & ~(int64_t)3;
    const int nch = (int)((e - a0 + 3) >> 2);
    copy_words(sm.col[st], col, a0, nch, nnz);
    copy_words(reinterpret_cast<int32_t *>(sm.val[st]), reinterpret_cast<const int32_t *>(val), a0, nch, nnz);
}

// Walk this block's tiles.  For each row the functor receives
//   op(row, c, v, n): the row's n column indices / values (shared memory when
//   staged, global memory otherwise), in storage order.
// Threads beyond a short last tile do not call op.  Every thread of the block
// must call this function.
template <class RowOp>
__device__ __forceinline__ void csr_for_rows(CsrStages &sm, int64_t N, const int32_t *__restrict__ rowptr,
                                             const int32_t *__restrict__ col, const float *__restrict__ val,
                                             RowOp &op)
{
    const int64_t ntiles = cdiv(N, kTileRows);
    const int64_t nnz = rowptr[N];
    const int64_t t0 = blockIdx.x, dt = gridDim.x;
    // prologue: rowptr of tiles t0 and t0+dt, then col/val of t0
    issue_rp(sm, 0, t0, ntiles, N, rowptr);
    issue_rp(sm, 1, t0 + dt, ntiles, N, rowptr);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue_cv(sm, 0, t0, ntiles, N, nnz, col, val);
    cp_async_commit();
    int k = 0;  // stage of the current tile
    for (int64_t t = t0; t < ntiles; t += dt, k = k == kStages - 1 ? 0 : k + 1) {
        cp_async_wait_all();
        __syncthreads();
        const int k1 = k == kStages - 1 ? 0 : k + 1;
        const int k2 = k1 == kStages - 1 ? 0 : k1 + 1;
        issue_rp(sm, k2, t + 2 * dt, ntiles, N, rowptr);
        issue_cv(sm, k1, t + dt, ntiles, N, nnz, col, val);
        cp_async_commit();
        const int64_t r0 = t * kTileRows;
        const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
        const int64_t s = sm.rp[k][0], e = sm.rp[k][nrows];
        if (threadIdx.x < nrows) {
            const int32_t k0 = sm.rp[k][threadIdx.x], kend = sm.rp[k][threadIdx.x + 1];
            if (e - s <= kTileCap) {
                const int o = (int)(k0 - (s & ~(int64_t)3));
                op(r0 + threadIdx.x, &sm.col[k][o], &sm.val[k][o], (int)(kend - k0));
            } else {
                op(r0 + threadIdx.x, col + k0, val + k0, (int)(kend - k0));
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

}  // namespace piro

// csr_tile.cuh -- pipelined streaming of CSR row tiles through shared memory.
//
// A persistent block walks tiles of kTileRows consecutive rows.  While the
// threads reduce tile t (one row per thread, storage order, so results keep
// the reference's summation order), the tile's successor streams in:
// cp.async (16-byte, L2-only, zero-filled past the array end) copies the
// col/val range of the tile kAhead steps ahead and the rowptr slice 2*kAhead
// steps ahead into circular shared-memory stages.  HBM therefore always has the next tile's bytes in
// flight instead of idling during the gathers of the current one.
//
// Shared memory per block: 5 rowptr stages x 1040 B + 3 col/val stages x
// 2 x 8224 B = 54.5 KB; four blocks fill an SM, each with two tiles in flight.  Tiles whose nonzeros exceed kTileCap
// (rows much longer than a 7-point stencil's) fall back to direct loads.
#pragma once
#include "common.cuh"

namespace piro {

constexpr int kTileRows = 256;
constexpr int kTileCap = 2048;           // staged nonzeros per tile (7-point rows: <= 1792)
constexpr int kAhead = 2;                // col/val tiles in flight ahead of the one being reduced
constexpr int kCvStages = kAhead + 1;    // col/val stages
constexpr int kRpStages = 2 * kAhead + 1;  // rowptr slices run kAhead further ahead
constexpr int kRpWords = kTileRows + 4;  // rowptr slice rounded to 16 B
constexpr int kCvWords = kTileCap + 8;   // col/val slice + alignment slack

struct CsrStages {
    int32_t rp[kRpStages][kRpWords];
    int32_t col[kCvStages][kCvWords];
    float val[kCvStages][kCvWords];
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int kPending>
__device__ __forceinline__ void cp_async_wait_pending()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kPending) : "memory");
}

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

// Issue the col/val slice of tile `tile` into col/val stage `st` (its rowptr
// slice is in rowptr stage `rst`).
__device__ __forceinline__ void issue_cv(CsrStages &sm, int st, int rst, int64_t tile, int64_t ntiles, int64_t N,
                                         int64_t nnz, const int32_t *__restrict__ col, const float *__restrict__ val)
{
    if (tile >= ntiles) return;
    const int64_t r0 = tile * kTileRows;
    const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
    const int64_t s = sm.rp[rst][0], e = sm.rp[rst][nrows];
    if (e - s > kTileCap) return;  // long rows: computed from global memory
    const int64_t a0 = s & ~(int64_t)3;
    const int nch = (int)((e - a0 + 3) >> 2);
    copy_words(sm.col[st], col, a0, nch, nnz);
    copy_words(reinterpret_cast<int32_t *>(sm.val[st]), reinterpret_cast<const int32_t *>(val), a0, nch, nnz);
}

// Walk this block's tiles.  The functor sees each row as
//   op.begin(row), op.add(col, val) for every entry in storage order,
//   op.end(row);
// staged entries are read from shared memory by index (LDS), so the row loop
// carries no generic-address overhead.  Threads beyond a short last tile skip
// their row.  Every thread of the block must call this function.
template <class RowOp>
__device__ __forceinline__ void csr_for_rows(CsrStages &sm, int64_t N, const int32_t *__restrict__ rowptr,
                                             const int32_t *__restrict__ col, const float *__restrict__ val,
                                             RowOp &op)
{
    const int64_t ntiles = cdiv(N, kTileRows);
    const int64_t nnz = rowptr[N];
    const int64_t t0 = blockIdx.x, dt = gridDim.x;
    // Tile j of this block (tile t0 + j*dt) uses rowptr stage j % kRpStages
    // and col/val stage j % kCvStages.  Iteration j commits one group holding
    // rowptr(j + 2*kAhead) and col/val(j + kAhead); col/val(j) and rowptr(j +
    // kAhead) were committed kAhead iterations earlier, so waiting until at
    // most kAhead - 1 groups are pending makes both visible.
    for (int a = 0; a < 2 * kAhead; ++a) issue_rp(sm, a % kRpStages, t0 + a * dt, ntiles, N, rowptr);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    for (int a = 0; a < kAhead; ++a) {
        issue_cv(sm, a % kCvStages, a % kRpStages, t0 + a * dt, ntiles, N, nnz, col, val);
        cp_async_commit();
    }
    int j = 0;
    for (int64_t t = t0; t < ntiles; t += dt, ++j) {
        cp_async_wait_pending<kAhead - 1>();
        __syncthreads();
        {
            const int jr = j + 2 * kAhead, jc = j + kAhead;
            issue_rp(sm, jr % kRpStages, t0 + (int64_t)jr * dt, ntiles, N, rowptr);
            issue_cv(sm, jc % kCvStages, jc % kRpStages, t0 + (int64_t)jc * dt, ntiles, N, nnz, col, val);
            cp_async_commit();
        }
        const int kr = j % kRpStages, kc = j % kCvStages;
        const int64_t r0 = t * kTileRows;
        const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
        if (threadIdx.x < nrows) {
            const int32_t s = sm.rp[kr][0];
            const int32_t k0 = sm.rp[kr][threadIdx.x], kend = sm.rp[kr][threadIdx.x + 1];
            const int64_t row = r0 + threadIdx.x;
            op.begin(row);
            if (sm.rp[kr][nrows] - s <= kTileCap) {
                const int base = s & ~3;
                const int32_t *scol = sm.col[kc];
                const float *sval = sm.val[kc];
                for (int q = k0 - base; q < kend - base; ++q) op.add(scol[q], sval[q]);
            } else {
                for (int32_t q = k0; q < kend; ++q) op.add(col[q], val[q]);
            }
            op.end(row);
        }
    }
    cp_async_wait_all();
    __syncthreads();
}

}  // namespace piro

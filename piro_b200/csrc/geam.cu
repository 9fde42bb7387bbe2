// geam.cu -- csrgeam (the v.grad merge of operator&), A + beta*B for the
// backward-Euler matrix, and the device row-pointer scan they share.
//
// The reference computes row counts, then runs prefixsum.cl N times from the
// host with a clFinish after each (src/kernelcsrgeam.cpp:55-62).  Here the
// counts are written straight into rowptr[1..N] and scanned in place by a
// three-pass block scan (block sums -> scan of block sums -> block-local scan
// plus offset), two launches plus one small single-block launch regardless of
// N.  The block sums live in caller-provided workspace.
#include <algorithm>

#include "common.cuh"

namespace piro {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_inclusive_scan(int64_t v, int64_t *s_warp)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) s_warp[w] = v;
    __syncthreads();
    if (w == 0) {
        int64_t t = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t q = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += q;
        }
        s_warp[lane] = t;
    }
    __syncthreads();
    if (w > 0) v += s_warp[w - 1];
    __syncthreads();
    return v;
}

// Pass 1: per-chunk sums of a[0..n).
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int64_t n, const int32_t *__restrict__ a,
                                                            int64_t *__restrict__ sums)
{
    __shared__ int64_t s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    int64_t v = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        const int64_t i = base + (int64_t)threadIdx.x * kScanItems + t;
        if (i < n) v += a[i];
    }
    v = block_inclusive_scan(v, s_warp);
    if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = v;
}

// Pass 2: exclusive scan of the chunk sums, one block, carried across rounds.
__global__ void __launch_bounds__(kScanThreads) k_scan_offsets(int64_t nb, int64_t *__restrict__ sums)
{
    __shared__ int64_t s_warp[32];
    __shared__ int64_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t b0 = 0; b0 < nb; b0 += kScanThreads) {
        const int64_t i = b0 + threadIdx.x;
        const int64_t v = i < nb ? sums[i] : 0;
        const int64_t inc = block_inclusive_scan(v, s_warp);
        const int64_t carry = s_carry;
        if (i < nb) sums[i] = carry + inc - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = carry + inc;
        __syncthreads();
    }
}

// Pass 3: in-place inclusive scan of a[0..n) plus the chunk offset.
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(int64_t n, int32_t *__restrict__ a,
                                                             const int64_t *__restrict__ offs)
{
    __shared__ int64_t s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * kScanChunk;
    int64_t loc[kScanItems];
    int64_t v = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        const int64_t i = base + (int64_t)threadIdx.x * kScanItems + t;
        loc[t] = i < n ? a[i] : 0;
        v += loc[t];
    }
    int64_t run = block_inclusive_scan(v, s_warp) - v + offs[blockIdx.x];
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        const int64_t i = base + (int64_t)threadIdx.x * kScanItems + t;
        run += loc[t];
        if (i < n) a[i] = (int32_t)run;
    }
}

// Counts for csrgeam_1.cl: lenA + lenB + lenC (no dedup, csrgeam_1.cl:27-67).
__global__ void k_geam3_count(int64_t N, const int32_t *__restrict__ rpA, const int32_t *__restrict__ rpB,
                              const int32_t *__restrict__ rpC, int32_t *__restrict__ rpD)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        rpD[r + 1] = (rpA[r + 1] - rpA[r]) + (rpB[r + 1] - rpB[r]) + (rpC[r + 1] - rpC[r]);
        if (r == 0) rpD[0] = 0;
    }
}

// csrgeam_3.cl:21-88: three-way merge per row, ties A before B before C,
// tails appended A, B, C; values scaled by v[row + comp*N].  A warp takes 32
// consecutive rows.  Their entries in each input are one contiguous segment,
// and so are their outputs: the warp loads the three input segments into
// shared memory with consecutive lanes on consecutive entries, each lane
// merges its row there, and the warp stores the output segment the same
// coalesced way.  A chunk whose segments exceed the staging capacity (or
// whose row pointers are not monotone) runs the same merge per lane on
// global memory instead.
constexpr int kGeamWarps = 8;
constexpr int kGeamCap = 64;  // staged entries per input and warp (2 per row: a gradient matrix)
// 5 blocks per SM (48 registers): with the next chunk's row pointers held in
// registers, 6 blocks (40 registers) spilled and took 1.09 ms for the 256^3
// merge, 4 blocks 0.61 ms, 5 blocks 0.56 ms (0.64 ms before the prefetch).
constexpr int kGeamBlocksPerSM = 5;

__global__ void __launch_bounds__(kGeamWarps * 32, kGeamBlocksPerSM) k_geam3_fill_warp(
    int64_t N, const int32_t *__restrict__ rpA, const int32_t *__restrict__ cA, const float *__restrict__ vA,
    const int32_t *__restrict__ rpB, const int32_t *__restrict__ cB, const float *__restrict__ vB,
    const int32_t *__restrict__ rpC, const int32_t *__restrict__ cC, const float *__restrict__ vC,
    const float *__restrict__ v, const int32_t *__restrict__ rpD, int32_t *__restrict__ cD, float *__restrict__ vD)
{
    __shared__ int32_t s_c[kGeamWarps][6 * kGeamCap];  // A, B, C inputs, then the 3 * kGeamCap outputs
    __shared__ float s_v[kGeamWarps][6 * kGeamCap];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t *sc = s_c[w];
    float *sv = s_v[w];
    const int64_t nchunk = (N + 31) >> 5;
    const int64_t stride = (int64_t)gridDim.x * kGeamWarps;
    // Each lane's row pointers and scale factors for its row of a chunk; the
    // next chunk's are loaded while the current one is staged and merged, so
    // that a warp waits on one dependent round trip per chunk, not two.
    struct Rows {
        int32_t i, ie, j, je, k, ke, dd, dn;
        float sa, sb, sc;
    };
    auto fetch = [&](int64_t ch, Rows &R) {
        const int64_t row = (ch << 5) + lane;
        if (ch < nchunk && row < N) {
            R.i = rpA[row]; R.ie = rpA[row + 1];
            R.j = rpB[row]; R.je = rpB[row + 1];
            R.k = rpC[row]; R.ke = rpC[row + 1];
            R.dd = rpD[row]; R.dn = rpD[row + 1];
            R.sa = v[row]; R.sb = v[N + row]; R.sc = v[2 * N + row];
        } else {
            R.i = R.ie = R.j = R.je = R.k = R.ke = R.dd = R.dn = 0;
            R.sa = R.sb = R.sc = 0.0f;
        }
    };
    Rows nxt;
    fetch((int64_t)blockIdx.x * kGeamWarps + w, nxt);
    for (int64_t ch = (int64_t)blockIdx.x * kGeamWarps + w; ch < nchunk; ch += stride) {
        const Rows R = nxt;
        fetch(ch + stride, nxt);
        const int64_t r0 = ch << 5, r1 = r0 + 32 < N ? r0 + 32 : N;
        const int64_t row = r0 + lane;
        const bool live = row < r1;
        const int lastl = (int)(r1 - r0) - 1;  // the chunk's last row: its end pointers close the segments
        const int32_t a0 = __shfl_sync(0xffffffffu, R.i, 0), a1 = __shfl_sync(0xffffffffu, R.ie, lastl);
        const int32_t b0 = __shfl_sync(0xffffffffu, R.j, 0), b1 = __shfl_sync(0xffffffffu, R.je, lastl);
        const int32_t c0 = __shfl_sync(0xffffffffu, R.k, 0), c1 = __shfl_sync(0xffffffffu, R.ke, lastl);
        const int32_t d0 = __shfl_sync(0xffffffffu, R.dd, 0), d1 = __shfl_sync(0xffffffffu, R.dn, lastl);
        int32_t i = R.i, ie = R.ie, j = R.j, je = R.je, k = R.k, ke = R.ke;
        const float sa = R.sa, sb = R.sb, sc_ = R.sc;
        const int32_t rowD = R.dd;
        // stage only when every lane's ranges lie inside the chunk's segments (a
        // monotone row pointer) and the segments fit; else the global loop
        const bool inside = !live || (a0 <= i && i <= ie && ie <= a1 && b0 <= j && j <= je && je <= b1 &&
                                      c0 <= k && k <= ke && ke <= c1 && d0 <= rowD && d1 <= d0 + 3 * kGeamCap);
        const bool fits = (uint32_t)(a1 - a0) <= (uint32_t)kGeamCap && (uint32_t)(b1 - b0) <= (uint32_t)kGeamCap &&
                          (uint32_t)(c1 - c0) <= (uint32_t)kGeamCap;
        if (!__all_sync(0xffffffffu, inside && fits)) {
            if (live) {
                int64_t d = rowD;
                while (i < ie && j < je && k < ke) {
                    const int32_t a = cA[i], b = cB[j], c = cC[k];
                    const int32_t m = min(a, min(c, b));
                    if (a == m) { cD[d] = a; vD[d] = __fmul_rn(vA[i], sa); ++i; }
                    else if (b == m) { cD[d] = b; vD[d] = __fmul_rn(vB[j], sb); ++j; }
                    else { cD[d] = c; vD[d] = __fmul_rn(vC[k], sc_); ++k; }
                    ++d;
                }
                for (; i < ie; ++i, ++d) { cD[d] = cA[i]; vD[d] = __fmul_rn(vA[i], sa); }
                for (; j < je; ++j, ++d) { cD[d] = cB[j]; vD[d] = __fmul_rn(vB[j], sb); }
                for (; k < ke; ++k, ++d) { cD[d] = cC[k]; vD[d] = __fmul_rn(vC[k], sc_); }
            }
            continue;
        }
        for (int t = lane; t < a1 - a0; t += 32) { sc[t] = cA[a0 + t]; sv[t] = vA[a0 + t]; }
        for (int t = lane; t < b1 - b0; t += 32) { sc[kGeamCap + t] = cB[b0 + t]; sv[kGeamCap + t] = vB[b0 + t]; }
        for (int t = lane; t < c1 - c0; t += 32) {
            sc[2 * kGeamCap + t] = cC[c0 + t];
            sv[2 * kGeamCap + t] = vC[c0 + t];
        }
        __syncwarp();
        if (live) {
            int32_t *oc = sc + 3 * kGeamCap;
            float *ov = sv + 3 * kGeamCap;
            int d = rowD - d0;
            i -= a0; ie -= a0;
            j -= b0; je -= b0;
            k -= c0; ke -= c0;
            const int32_t *lc_a = sc, *lc_b = sc + kGeamCap, *lc_c = sc + 2 * kGeamCap;
            const float *lv_a = sv, *lv_b = sv + kGeamCap, *lv_c = sv + 2 * kGeamCap;
            while (i < ie && j < je && k < ke) {
                const int32_t a = lc_a[i], b = lc_b[j], c = lc_c[k];
                const int32_t m = min(a, min(c, b));
                if (a == m) { oc[d] = a; ov[d] = __fmul_rn(lv_a[i], sa); ++i; }
                else if (b == m) { oc[d] = b; ov[d] = __fmul_rn(lv_b[j], sb); ++j; }
                else { oc[d] = c; ov[d] = __fmul_rn(lv_c[k], sc_); ++k; }
                ++d;
            }
            for (; i < ie; ++i, ++d) { oc[d] = lc_a[i]; ov[d] = __fmul_rn(lv_a[i], sa); }
            for (; j < je; ++j, ++d) { oc[d] = lc_b[j]; ov[d] = __fmul_rn(lv_b[j], sb); }
            for (; k < ke; ++k, ++d) { oc[d] = lc_c[k]; ov[d] = __fmul_rn(lv_c[k], sc_); }
        }
        __syncwarp();
        for (int t = lane; t < d1 - d0; t += 32) {
            cD[d0 + t] = sc[3 * kGeamCap + t];
            vD[d0 + t] = sv[3 * kGeamCap + t];
        }
        __syncwarp();
    }
}

constexpr int kUnionMax = 64;

// Sorted unique union of two rows' columns in a local array; -1 on overflow.
__device__ __forceinline__ int row_union(const int32_t *__restrict__ ca, int na, const int32_t *__restrict__ cb, int nb,
                                         int32_t *u)
{
    if (na + nb > kUnionMax) return -1;
    int n = 0;
    for (int t = 0; t < na + nb; ++t) {
        const int32_t c = t < na ? ca[t] : cb[t - na];
        int p = n;
        bool dup = false;
        for (int q = 0; q < n; ++q)
            if (u[q] == c) { dup = true; break; }
        if (dup) continue;
        while (p > 0 && u[p - 1] > c) { u[p] = u[p - 1]; --p; }
        u[p] = c;
        ++n;
    }
    return n;
}

__global__ void k_geam2_count(int64_t N, const int32_t *__restrict__ rpA, const int32_t *__restrict__ cA,
                              const int32_t *__restrict__ rpB, const int32_t *__restrict__ cB,
                              int32_t *__restrict__ rpD, int *__restrict__ err)
{
    int32_t u[kUnionMax];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        const int n = row_union(cA + rpA[r], rpA[r + 1] - rpA[r], cB + rpB[r], rpB[r + 1] - rpB[r], u);
        if (n < 0) { atomicExch(err, 1); rpD[r + 1] = 0; }
        else rpD[r + 1] = n;
        if (r == 0) rpD[0] = 0;
    }
}

__global__ void k_geam2_fill(int64_t N, const int32_t *__restrict__ rpA, const int32_t *__restrict__ cA,
                             const float *__restrict__ vA, float beta, const int32_t *__restrict__ rpB,
                             const int32_t *__restrict__ cB, const float *__restrict__ vB,
                             const int32_t *__restrict__ rpD, int32_t *__restrict__ cD, float *__restrict__ vD)
{
    int32_t u[kUnionMax];
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a0 = rpA[r], a1 = rpA[r + 1], b0 = rpB[r], b1 = rpB[r + 1];
        const int n = row_union(cA + a0, a1 - a0, cB + b0, b1 - b0, u);
        if (n < 0) continue;
        const int64_t d0 = rpD[r];
        for (int t = 0; t < n; ++t) {
            const int32_t c = u[t];
            float acc = 0.0f;
            bool have = false;
            for (int32_t a = a0; a < a1; ++a)
                if (cA[a] == c) { acc = have ? __fadd_rn(acc, vA[a]) : vA[a]; have = true; }
            for (int32_t b = b0; b < b1; ++b)
                if (cB[b] == c) {
                    const float t2 = __fmul_rn(beta, vB[b]);
                    acc = have ? __fadd_rn(acc, t2) : t2;
                    have = true;
                }
            cD[d0 + t] = c;
            vD[d0 + t] = acc;
        }
    }
}

}  // namespace

// In-place scan of rowptr[1..N] (counts -> inclusive sums); rowptr[0] = 0
// must already be set.  Exposed to the other translation units.
int scan_rowptr_inplace(int64_t N, int32_t *rowptr, void *work, size_t work_bytes, cudaStream_t s)
{
    const int64_t nb = cdiv(N, kScanChunk);
    PIRO_ARG(work && work_bytes >= sizeof(int64_t) * (size_t)nb, "scan: workspace too small");
    int64_t *sums = static_cast<int64_t *>(work);
    k_scan_sums<<<(unsigned)nb, kScanThreads, 0, s>>>(N, rowptr + 1, sums);
    PIRO_CHECK_LAUNCH("k_scan_sums");
    k_scan_offsets<<<1, kScanThreads, 0, s>>>(nb, sums);
    PIRO_CHECK_LAUNCH("k_scan_offsets");
    k_scan_apply<<<(unsigned)nb, kScanThreads, 0, s>>>(N, rowptr + 1, sums);
    PIRO_CHECK_LAUNCH("k_scan_apply");
    return PIRO_OK;
}

size_t scan_workspace_bytes(int64_t N) { return sizeof(int64_t) * (size_t)(cdiv(N, kScanChunk) + 1) + 256; }

}  // namespace piro

using namespace piro;

extern "C" int piro_scan_workspace(int64_t nrows, size_t *bytes)
{
    PIRO_ARG(bytes && nrows >= 0, "piro_scan_workspace: bad arguments");
    *bytes = scan_workspace_bytes(nrows);
    return PIRO_OK;
}

extern "C" int piro_csrgeam3(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, const int32_t *rpB,
                             const int32_t *cB, const float *vB, const int32_t *rpC, const int32_t *cC,
                             const float *vC, const float *v, int32_t *rpD, int32_t *cD, float *vD, void *work,
                             size_t work_bytes, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rpA && cA && vA && rpB && cB && vB && rpC && cC && vC && v && rpD && cD && vD,
             "piro_csrgeam3: null argument");
    PIRO_ARG(N < INT32_MAX, "piro_csrgeam3: too many rows");
    cudaStream_t s = as_stream(stream);
    k_geam3_count<<<grid_for(N, 256, 8), 256, 0, s>>>(N, rpA, rpB, rpC, rpD);
    PIRO_CHECK_LAUNCH("k_geam3_count");
    int rc = scan_rowptr_inplace(N, rpD, work, work_bytes, s);
    if (rc) return rc;
    // one resident wave: every warp walks many chunks, so that the next
    // chunk's row pointers are in flight behind the current one
    const unsigned fill_grid =
        (unsigned)std::min<int64_t>(cdiv(cdiv(N, 32), kGeamWarps), (int64_t)sm_count() * kGeamBlocksPerSM);
    k_geam3_fill_warp<<<fill_grid, kGeamWarps * 32, 0, s>>>(
        N, rpA, cA, vA, rpB, cB, vB, rpC, cC, vC, v, rpD, cD, vD);
    PIRO_CHECK_LAUNCH("k_geam3_fill_warp");
    return PIRO_OK;
}

extern "C" int piro_csrgeam2_count(int64_t N, const int32_t *rpA, const int32_t *cA, const int32_t *rpB,
                                   const int32_t *cB, int32_t *rpD, void *work, size_t work_bytes,
                                   piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rpA && cA && rpB && cB && rpD, "piro_csrgeam2_count: null argument");
    cudaStream_t s = as_stream(stream);
    // the last 256 bytes of the workspace hold the overflow flag
    PIRO_ARG(work && work_bytes >= scan_workspace_bytes(N), "piro_csrgeam2_count: workspace too small");
    int *err = reinterpret_cast<int *>(static_cast<char *>(work) + work_bytes - sizeof(int));
    PIRO_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    k_geam2_count<<<grid_for(N, 256, 8), 256, 0, s>>>(N, rpA, cA, rpB, cB, rpD, err);
    PIRO_CHECK_LAUNCH("k_geam2_count");
    int rc = scan_rowptr_inplace(N, rpD, work, work_bytes - 256, s);
    if (rc) return rc;
    int h_err = 0;
    PIRO_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    PIRO_CUDA(cudaStreamSynchronize(s));
    if (h_err) {
        piro::set_error("piro_csrgeam2_count: a row has more than %d combined entries", kUnionMax);
        return PIRO_ERR_ARG;
    }
    return PIRO_OK;
}

extern "C" int piro_csrgeam2_fill(int64_t N, const int32_t *rpA, const int32_t *cA, const float *vA, float beta,
                                  const int32_t *rpB, const int32_t *cB, const float *vB, const int32_t *rpD,
                                  int32_t *cD, float *vD, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rpA && cA && vA && rpB && cB && vB && rpD && cD && vD, "piro_csrgeam2_fill: null argument");
    k_geam2_fill<<<grid_for(N, 128, 8), 128, 0, as_stream(stream)>>>(N, rpA, cA, vA, beta, rpB, cB, vB, rpD, cD, vD);
    PIRO_CHECK_LAUNCH("k_geam2_fill");
    return PIRO_OK;
}

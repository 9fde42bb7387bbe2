// hashtable_lu.cu -- scheme 27 (TIMESCHEME 12 + solver 27): Gaussian
// elimination on a matrix stored in the open-addressing hash table (key
// row*N + col, home slot key % ts, linear probing; -1 empty, -2 deleted).
//
// PIRO's factorization (src/matrixoperations.cpp:10-104 with
// lu_decompHT.cl) runs, for each pivot row ro:
//   1. the columns co >= ro with |a(ro, co)| > 1e-6, in order;
//   2. on the host, for each row r > ro with a(r, ro) != 0, each of those
//      columns inserted as an explicit zero (methods::lookupandset: no change
//      if the key exists; else into the first deleted slot met on the probe, or
//      the empty slot that ends it) -- the fill-in;
//   3. a kernel over (r, c), r > ro, c >= ro: a(r, c) -= (a(r, ro)/a(ro, ro)) *
//      a(ro, c) when both factors are nonzero, and the key is deleted (-2)
//      when |a(r, c)| < 1e-6.  Item (r, ro) rewrites the factor that the other
//      items of row r read; here the pivot row and the factor column are
//      gathered before the round, so every item sees the pre-round values (the
//      reference leaves this to scheduling).  An item whose own key is absent
//      writes to slot -1 in the reference; here it writes nothing.
// The multipliers end as deleted keys, and the reference never substitutes:
// each scheme-27 step returns a zero field.  piro_ht_lu_reference reproduces
// that factorization on the device with no per-round table round trips (the
// reference uploads and downloads the whole table each round).  The fill-in
// is one device thread, because slot placement depends on the insertion order.
// The elimination is a gather kernel and an item kernel per round.
//
// piro_ht_lu_factor / piro_ht_lu_solve make scheme 27 return a solution.
// Rows couple only within the bandwidth bw (nx*ny for the 7-point grid in
// natural order), and elimination without pivoting fills in nothing outside
// the band.  So the whole band is inserted once, in parallel (atomicCAS
// linear probing; placement is free here), and each round is the same gather
// and item kernels over the (bw+1)^2 block below and right of the pivot, with
// exact zero tests, nothing deleted, and the multiplier a(r, ro)/a(ro, ro)
// stored in place of a(r, ro): an in-place LU, L unit lower.  The solve is
// forward then backward substitution in one block, by blocks of 32 rows: the
// warps form the rows' sums over the solved part of the band, then one warp
// finishes the 32x32 triangle from shared memory.
#include "common.cuh"

namespace piro {
namespace {

constexpr int64_t kEmpty = -1, kDeleted = -2;
constexpr int kTri = 32;  // rows per substitution block

// methods::lookup / lu_decompHT.cl lookup: value and slot of key, or 0 and -1.
__device__ __forceinline__ float ht_find(int64_t key, const int64_t *__restrict__ keys, const float *__restrict__ vals,
                                         int64_t ts, int64_t *slot)
{
    int64_t h = key % ts;
    for (int64_t a = 0; a < ts; ++a) {
        const int64_t k = keys[h];
        if (k == kEmpty) break;
        if (k == key) {
            *slot = h;
            return vals[h];
        }
        h = h + 1 == ts ? 0 : h + 1;
    }
    *slot = -1;
    return 0.0f;
}

__device__ __forceinline__ float ht_value(int64_t key, const int64_t *__restrict__ keys,
                                          const float *__restrict__ vals, int64_t ts)
{
    int64_t s;
    return ht_find(key, keys, vals, ts, &s);
}

// methods::lookupandset with value 0: insert the key if absent.  false if the
// table has no room.
__device__ __forceinline__ bool ht_ensure(int64_t key, int64_t *keys, float *vals, int64_t ts)
{
    int64_t h = key % ts, first_deleted = -1;
    for (int64_t a = 0; a <= ts; ++a) {
        const int64_t k = keys[h];
        if (k == key) return true;
        if (k == kEmpty) {
            const int64_t at = first_deleted != -1 ? first_deleted : h;
            keys[at] = key;
            vals[at] = 0.0f;
            return true;
        }
        if (k == kDeleted && first_deleted == -1) first_deleted = h;
        h = h + 1 == ts ? 0 : h + 1;
    }
    if (first_deleted != -1) {
        keys[first_deleted] = key;
        vals[first_deleted] = 0.0f;
        return true;
    }
    return false;
}

// Pre-round values: prow[j] = a(ro, ro+j), j < ncol; fac[i] = a(ro+1+i, ro), i < nrow.
__global__ void k_lu_gather(int64_t N, int64_t ro, int64_t ncol, int64_t nrow, const int64_t *__restrict__ keys,
                            const float *__restrict__ vals, int64_t ts, float *__restrict__ prow,
                            float *__restrict__ fac)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncol + nrow;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (t < ncol)
            prow[t] = ht_value(ro * N + ro + t, keys, vals, ts);
        else
            fac[t - ncol] = ht_value((ro + 1 + t - ncol) * N + ro, keys, vals, ts);
    }
}

// The reference's fill-in for pivot row ro (one thread, its insertion order).
__global__ void k_lu_fill(int64_t N, int64_t ro, int64_t *keys, float *vals, int64_t ts,
                          const float *__restrict__ prow, const float *__restrict__ fac, int32_t *__restrict__ cols,
                          int *err)
{
    if (blockIdx.x != 0 || threadIdx.x != 0 || *err) return;
    int ncols = 0;
    for (int64_t co = ro; co < N; ++co)
        if ((double)fabsf(prow[co - ro]) > 1e-6) cols[ncols++] = (int32_t)co;
    for (int64_t r = ro + 1; r < N; ++r) {
        if (fac[r - ro - 1] == 0.0f) continue;
        for (int k = 0; k < ncols; ++k)
            if (!ht_ensure(r * N + cols[k], keys, vals, ts)) {
                atomicExch(err, 1);
                return;
            }
    }
}

// Elimination round ro over rows ro+1 .. ro+nrow and columns ro .. ro+ncol-1.
// reference: PIRO's update and deletion rule; else the in-place LU (column
// ro stores the multiplier; a zero pivot-row entry changes nothing).
__global__ void k_lu_round(int64_t N, int64_t ro, int64_t nrow, int64_t ncol, int64_t *keys, float *vals,
                           int64_t ts, const float *__restrict__ prow, const float *__restrict__ fac, int reference,
                           int *err)
{
    const float piv = prow[0];
    if (piv == 0.0f) {
        // the reference skips the round; the in-place LU cannot go on
        if (!reference && blockIdx.x == 0 && threadIdx.x == 0 && atomicCAS(err, 0, 3) == 0) err[1] = (int)ro;
        return;
    }
    const int64_t items = nrow * ncol;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < items; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ncol, j = t % ncol;
        const float factor = fac[i], val0 = prow[j];
        if (factor == 0.0f || (!reference && j > 0 && val0 == 0.0f)) continue;
        int64_t hk;
        float val = ht_find((ro + 1 + i) * N + ro + j, keys, vals, ts, &hk);
        if (hk < 0) continue;
        if (reference) {
            val = __fsub_rn(val, __fmul_rn(__fdiv_rn(factor, piv), val0));
            vals[hk] = val;
            if ((double)fabsf(val) < 1e-6) keys[hk] = kDeleted;
        } else if (j == 0) {
            vals[hk] = __fdiv_rn(factor, piv);  // the multiplier l(r, ro)
        } else {
            vals[hk] = __fsub_rn(val, __fmul_rn(__fdiv_rn(factor, piv), val0));
        }
    }
}

// Every (r, c) with |r - c| <= bw present (value 0 when inserted here).
__global__ void k_lu_band_insert(int64_t N, int64_t bw, int64_t *keys, float *vals, int64_t ts, int *err)
{
    const int64_t w = 2 * bw + 1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < N * w; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / w, c = r - bw + t % w;
        if (c < 0 || c >= N) continue;
        const int64_t key = r * N + c;
        int64_t h = key % ts;
        int64_t a = 0;
        for (; a < ts; ++a) {
            const int64_t k = *((volatile int64_t *)keys + h);
            if (k == key) break;
            if (k == kEmpty) {
                const unsigned long long old =
                    atomicCAS((unsigned long long *)keys + h, (unsigned long long)kEmpty, (unsigned long long)key);
                if (old == (unsigned long long)kEmpty) {
                    vals[h] = 0.0f;
                    break;
                }
                if ((int64_t)old == key) break;
            }
            h = h + 1 == ts ? 0 : h + 1;
        }
        if (a == ts) atomicCAS(err, 0, 1);
    }
}

// Flags a stored key outside the band (the factor would ignore it).
__global__ void k_lu_band_check(int64_t N, int64_t bw, const int64_t *__restrict__ keys, int64_t ts, int *err)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ts; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = keys[s];
        if (k < 0) continue;
        const int64_t d = k / N - k % N;
        if (d > bw || d < -bw) atomicCAS(err, 0, 2);
    }
}

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// L U x = b.  Row blocks of kTri: the sums over the already-solved part of each
// row's band (one warp per row), then the kTri x kTri triangle (loaded by all
// threads into shared memory) solved by warp 0, lane i owning row R+i.
__global__ void __launch_bounds__(1024) k_lu_solve(int64_t N, int64_t bw, const int64_t *__restrict__ keys,
                                                   const float *__restrict__ vals, int64_t ts,
                                                   const float *__restrict__ b, float *__restrict__ x)
{
    __shared__ float s_tri[kTri][kTri + 1];
    __shared__ float s_sum[kTri];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    // forward: unit L, y kept in x
    for (int64_t R = 0; R < N; R += kTri) {
        const int nb = (int)(N - R < kTri ? N - R : kTri);
        for (int i = warp; i < nb; i += nwarp) {
            const int64_t r = R + i, c0 = r - bw > 0 ? r - bw : 0;
            float s = 0.0f;
            for (int64_t c = c0 + lane; c < R; c += 32) s += ht_value(r * N + c, keys, vals, ts) * x[c];
            s = warp_sum(s);
            if (lane == 0) s_sum[i] = s;
        }
        for (int t = threadIdx.x; t < kTri * kTri; t += blockDim.x) {
            const int i = t / kTri, j = t % kTri;
            s_tri[i][j] = (i < nb && j < i && i - j <= bw) ? ht_value((R + i) * N + R + j, keys, vals, ts) : 0.0f;
        }
        __syncthreads();
        if (warp == 0) {
            float v = lane < nb ? b[R + lane] - s_sum[lane] : 0.0f;
            for (int j = 0; j < nb; ++j) {
                const float xj = __shfl_sync(0xffffffffu, v, j);
                if (lane > j) v -= s_tri[lane][j] * xj;
            }
            if (lane < nb) x[R + lane] = v;
        }
        __syncthreads();
    }
    // backward: U
    for (int64_t R = ((N - 1) / kTri) * kTri; R >= 0; R -= kTri) {
        const int nb = (int)(N - R < kTri ? N - R : kTri);
        for (int i = warp; i < nb; i += nwarp) {
            const int64_t r = R + i, c1 = r + bw + 1 < N ? r + bw + 1 : N;
            float s = 0.0f;
            for (int64_t c = R + nb + lane; c < c1; c += 32) s += ht_value(r * N + c, keys, vals, ts) * x[c];
            s = warp_sum(s);
            if (lane == 0) s_sum[i] = s;
        }
        for (int t = threadIdx.x; t < kTri * kTri; t += blockDim.x) {
            const int i = t / kTri, j = t % kTri;
            s_tri[i][j] = (i < nb && j < nb && j >= i && j - i <= bw) ? ht_value((R + i) * N + R + j, keys, vals, ts)
                                                                      : 0.0f;
        }
        __syncthreads();
        if (warp == 0) {
            float v = lane < nb ? x[R + lane] - s_sum[lane] : 0.0f;
            for (int j = nb - 1; j >= 0; --j) {
                if (lane == j) v = v / s_tri[j][j];
                const float xj = __shfl_sync(0xffffffffu, v, j);
                if (lane < j) v -= s_tri[lane][j] * xj;
            }
            if (lane < nb) x[R + lane] = v;
        }
        __syncthreads();
    }
}

int lu_run(int64_t N, int64_t bw, int64_t *keys, float *vals, int64_t ts, bool reference, cudaStream_t st)
{
    const int64_t span = reference ? N : bw + 1;  // pivot-row columns gathered per round
    float *prow = nullptr, *fac = nullptr;
    int32_t *cols = nullptr;
    int *err = nullptr;
    cudaError_t e = cudaMalloc(&prow, sizeof(float) * (size_t)(2 * span));
    if (e == cudaSuccess) {
        fac = prow + span;
        e = cudaMalloc(&err, 2 * sizeof(int));  // flag, zero-pivot row
    }
    if (e == cudaSuccess && reference) e = cudaMalloc(&cols, sizeof(int32_t) * (size_t)N);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, 2 * sizeof(int), st);
    if (e == cudaSuccess && !reference) {
        k_lu_band_check<<<grid_for(ts, 256, 8), 256, 0, st>>>(N, bw, keys, ts, err);
        k_lu_band_insert<<<grid_for(N * (2 * bw + 1), 256, 8), 256, 0, st>>>(N, bw, keys, vals, ts, err);
        e = cudaGetLastError();
    }
    int herr[2] = {0, 0};
    if (e == cudaSuccess && !reference) {  // a table that fails here is not factorized
        e = cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    // the in-place LU also checks the last pivot (a round with no items)
    const int64_t rounds = reference ? N - 1 : N;
    for (int64_t ro = 0; ro < rounds && e == cudaSuccess && herr[0] == 0; ++ro) {
        const int64_t ncol = reference ? N - ro : (N - ro < bw + 1 ? N - ro : bw + 1);
        const int64_t nrow = ncol - 1;
        k_lu_gather<<<grid_for(ncol + nrow, 256, 4), 256, 0, st>>>(N, ro, ncol, nrow, keys, vals, ts, prow, fac);
        if (reference) k_lu_fill<<<1, 1, 0, st>>>(N, ro, keys, vals, ts, prow, fac, cols, err);
        k_lu_round<<<grid_for(nrow * ncol, 256, 4), 256, 0, st>>>(N, ro, nrow, ncol, keys, vals, ts, prow, fac,
                                                                  reference ? 1 : 0, err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(prow);
    cudaFree(cols);
    cudaFree(err);
    if (e != cudaSuccess) {
        set_error("ht lu: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    if (herr[0] == 3) {
        set_error("ht lu: zero pivot at row %d (elimination without pivoting)", herr[1]);
        return PIRO_ERR_ZERO_PIVOT;
    }
    if (herr[0] == 2) {
        set_error("ht lu: the table holds an entry outside the bandwidth %lld", (long long)bw);
        return PIRO_ERR_ARG;
    }
    if (herr[0]) {
        set_error("ht lu: the hash table has no room for the fill-in (raise its size)");
        return PIRO_ERR_TABLE_FULL;
    }
    return PIRO_OK;
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_ht_lu_reference(int64_t N, int64_t *keys, float *vals, int64_t ts, piro_stream_t stream)
{
    PIRO_ARG(N >= 1 && keys && vals && ts > 0 && N <= 46340, "piro_ht_lu_reference: bad arguments");
    return lu_run(N, N, keys, vals, ts, true, as_stream(stream));
}

extern "C" int piro_ht_lu_table_size(int64_t N, int64_t bw, float lf, int64_t *entries, int64_t *ts)
{
    PIRO_ARG(N >= 1 && bw >= 0 && lf > 0.0f && lf <= 1.0f && entries && ts, "piro_ht_lu_table_size: bad arguments");
    if (bw > N - 1) bw = N - 1;
    // rows r: min(N-1, r+bw) - max(0, r-bw) + 1 entries
    const int64_t n = N * (2 * bw + 1) - bw * (bw + 1);
    *entries = n;
    return piro_ht_table_size(n, N, 1, 0.0f, 0.0f, 0.0f, lf, ts);
}

extern "C" int piro_ht_lu_factor(int64_t N, int64_t bw, int64_t *keys, float *vals, int64_t ts, piro_stream_t stream)
{
    PIRO_ARG(N >= 1 && bw >= 1 && keys && vals && ts > 0 && N < ((int64_t)1 << 31), "piro_ht_lu_factor: bad arguments");
    return lu_run(N, bw < N ? bw : N, keys, vals, ts, false, as_stream(stream));
}

extern "C" int piro_ht_lu_solve(int64_t N, int64_t bw, const int64_t *keys, const float *vals, int64_t ts,
                                const float *b, float *x, piro_stream_t stream)
{
    PIRO_ARG(N >= 1 && bw >= 1 && keys && vals && ts > 0 && b && x && b != x, "piro_ht_lu_solve: bad arguments");
    k_lu_solve<<<1, 1024, 0, as_stream(stream)>>>(N, bw < N ? bw : N, keys, vals, ts, b, x);
    PIRO_CHECK_LAUNCH("k_lu_solve");
    return PIRO_OK;
}

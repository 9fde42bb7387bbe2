// hashtable_lu.cu -- scheme 27 (TIMESCHEME 12 + solver 27): Gaussian
// elimination of a matrix stored in PIRO's open-addressing hash table (key
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
// When the table fits in shared memory (up to ~18 K slots, which covers the
// grids the reference runs this scheme on), the whole factorization is one
// block with the table in shared memory; otherwise it is a gather, fill-in and
// elimination launch per round on the table in HBM.
//
// piro_ht_lu_factor / piro_ht_lu_solve make scheme 27 return a solution.  The
// table is the input format only: one pass over its slots scatters
// shift*I + scale*M in FP64 into a band (bandwidth bw = nx*ny for the 7-point
// grid in natural order).  The table stays out of the elimination: keys
// r*N + c of one row are contiguous, so at load 0.7 the rows' runs of slots
// merge and a table lookup walks thousands of slots.  The factorization is
// Gaussian elimination with partial pivoting in FP64 (LAPACK's banded LU,
// dgbtrf): per pivot row one launch chooses the pivot, exchanges the two
// rows and forms the multipliers, a second applies the rank-1 update to the
// (bw x 2bw) block below and right of it.  The solve (one block, FP64)
// replays the exchanges and Gauss transforms on b and back-substitutes.
#include "common.cuh"

namespace piro {
namespace {

constexpr int64_t kEmpty = -1, kDeleted = -2;

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

// Where methods::lookupandset would put key now: -1 if present; the first
// deleted slot on the probe path, else the empty slot that ends it; -2 if
// the table has neither.
__device__ __forceinline__ int64_t ht_candidate(int64_t key, const int64_t *keys, int64_t ts)
{
    int64_t h = key % ts, first_deleted = -1;
    for (int64_t a = 0; a <= ts; ++a) {
        const int64_t k = keys[h];
        if (k == key) return -1;
        if (k == kEmpty) return first_deleted != -1 ? first_deleted : h;
        if (k == kDeleted && first_deleted == -1) first_deleted = h;
        h = h + 1 == ts ? 0 : h + 1;
    }
    return first_deleted != -1 ? first_deleted : -2;
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

// ---------------------------------------------------------------- the reference's factorization

// Pre-round values: prow[j] = a(ro, ro+j), j < ncol; fac[i] = a(ro+1+i, ro), i < nrow.
__global__ void k_lu_gather(int64_t N, int64_t ro, int64_t ncol, int64_t nrow, const int64_t *__restrict__ keys,
                            const float *__restrict__ vals, int64_t ts, float *__restrict__ prow,
                            float *__restrict__ fac)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ncol + nrow;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t s;
        if (t < ncol)
            prow[t] = ht_find(ro * N + ro + t, keys, vals, ts, &s);
        else
            fac[t - ncol] = ht_find((ro + 1 + t - ncol) * N + ro, keys, vals, ts, &s);
    }
}

// The fill-in for pivot row ro (one thread, the reference's insertion order).
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

// Elimination round ro over rows ro+1 .. N-1 and columns ro .. N-1.
__global__ void k_lu_round(int64_t N, int64_t ro, int64_t *keys, float *vals, int64_t ts,
                           const float *__restrict__ prow, const float *__restrict__ fac)
{
    const float piv = prow[0];
    if (piv == 0.0f) return;
    const int64_t ncol = N - ro, items = (ncol - 1) * ncol;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < items; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ncol, j = t % ncol;
        const float factor = fac[i];
        if (factor == 0.0f) continue;
        int64_t hk;
        float val = ht_find((ro + 1 + i) * N + ro + j, keys, vals, ts, &hk);
        if (hk < 0) continue;
        val = __fsub_rn(val, __fmul_rn(__fdiv_rn(factor, piv), prow[j]));
        vals[hk] = val;
        if ((double)fabsf(val) < 1e-6) keys[hk] = kDeleted;
    }
}

// The whole factorization in one block, the table in shared memory (when
// keys, values and the round's gathers fit): the same gather, fill-in and
// elimination per round, separated by __syncthreads instead of launches, and
// every probe served by shared memory instead of a dependent L2 load.
__global__ void __launch_bounds__(1024) k_lu_reference_smem(int64_t N, int64_t *__restrict__ keys_g,
                                                            float *__restrict__ vals_g, int64_t ts, int *err)
{
    extern __shared__ __align__(16) unsigned char lu_smem[];
    int64_t *keys = reinterpret_cast<int64_t *>(lu_smem);
    float *vals = reinterpret_cast<float *>(keys + ts);
    float *prow = vals + ts;
    float *fac = prow + N;
    int32_t *cols = reinterpret_cast<int32_t *>(fac + N);
    __shared__ int s_err, s_nc;
    __shared__ int32_t s_cand[1024];
    for (int64_t s = threadIdx.x; s < ts; s += blockDim.x) {
        keys[s] = keys_g[s];
        vals[s] = vals_g[s];
    }
    if (threadIdx.x == 0) s_err = 0;
    __syncthreads();
    for (int64_t ro = 0; ro < N - 1; ++ro) {
        const int64_t ncol = N - ro, nrow = ncol - 1;
        for (int64_t t = threadIdx.x; t < ncol + nrow; t += blockDim.x) {
            int64_t sl;
            if (t < ncol)
                prow[t] = ht_find(ro * N + ro + t, keys, vals, ts, &sl);
            else
                fac[t - ncol] = ht_find((ro + 1 + t - ncol) * N + ro, keys, vals, ts, &sl);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int nc = 0;
            for (int64_t co = ro; co < N; ++co)
                if ((double)fabsf(prow[co - ro]) > 1e-6) cols[nc++] = (int32_t)co;
            s_nc = nc;
        }
        __syncthreads();
        // Fill-in, in the reference's order (rows, then columns), by chunks of
        // blockDim pairs: every thread walks its key's probe path at once
        // (present, or the slot lookupandset would take now); then thread 0
        // places the absent keys in order.  A slot taken by an earlier key of
        // the chunk moves the placement on to the next deleted or empty slot,
        // which is where the sequential walk would stop.
        const int64_t npairs = nrow * s_nc;
        for (int64_t base = 0; base < npairs && !s_err; base += blockDim.x) {
            const int64_t p = base + threadIdx.x;
            int32_t cand = -1;
            if (p < npairs && fac[p / s_nc] != 0.0f)
                cand = (int32_t)ht_candidate((ro + 1 + p / s_nc) * N + cols[p % s_nc], keys, ts);
            s_cand[threadIdx.x] = cand;
            __syncthreads();
            if (threadIdx.x == 0) {
                const int64_t m = npairs - base < blockDim.x ? npairs - base : blockDim.x;
                for (int64_t q = 0; q < m && !s_err; ++q) {
                    const int32_t c0 = s_cand[q];
                    if (c0 == -1) continue;
                    if (c0 == -2) {
                        s_err = 1;
                        break;
                    }
                    int64_t h = c0, a = 0;
                    while (keys[h] >= 0 && a < ts) {
                        h = h + 1 == ts ? 0 : h + 1;
                        ++a;
                    }
                    if (a == ts) {
                        s_err = 1;
                        break;
                    }
                    const int64_t pq = base + q;
                    keys[h] = (ro + 1 + pq / s_nc) * N + cols[pq % s_nc];
                    vals[h] = 0.0f;
                }
            }
            __syncthreads();
        }
        if (s_err) break;
        const float piv = prow[0];
        if (piv != 0.0f) {
            for (int64_t t = threadIdx.x; t < nrow * ncol; t += blockDim.x) {
                const int64_t i = t / ncol, j = t % ncol;
                const float factor = fac[i];
                if (factor == 0.0f) continue;
                int64_t hk;
                float val = ht_find((ro + 1 + i) * N + ro + j, keys, vals, ts, &hk);
                if (hk < 0) continue;
                val = __fsub_rn(val, __fmul_rn(__fdiv_rn(factor, piv), prow[j]));
                vals[hk] = val;
                if ((double)fabsf(val) < 1e-6) keys[hk] = kDeleted;
            }
        }
        __syncthreads();
    }
    for (int64_t s = threadIdx.x; s < ts; s += blockDim.x) {
        keys_g[s] = keys[s];
        vals_g[s] = vals[s];
    }
    if (threadIdx.x == 0 && s_err) *err = 1;
}

size_t lu_reference_smem_bytes(int64_t N, int64_t ts) { return (size_t)ts * 12 + (size_t)N * 12; }
constexpr size_t kLuSmemMax = 220 * 1024;

// ---------------------------------------------------------------- banded LU with partial pivoting (FP64)
//
// A = shift*I + scale*M in FP64, bandwidths kl = ku = bw.  Row r of the band
// holds columns r - bw .. r + 2bw (W = 3bw + 1 doubles, column c at
// band[r*W + c - r + bw]): row interchanges can move entries up to 2bw right
// of the diagonal into U, as in LAPACK's banded LU (dgbtrf).  Pivot row ro,
// one launch: piv[ro] = the row p in [ro, ro+bw] with the largest |a(p, ro)|
// (the first such row on a tie), rows ro and p exchanged over columns ro ..
// ro+2bw, and the multipliers l(i) = a(ro+i, ro) / a(ro, ro) written to
// Lc[ro*bw + i - 1].  A second launch subtracts l(i) * a(ro, c) from
// a(ro+i, c) for c in (ro, ro+2bw].  The multipliers stay with the row
// positions of their step (earlier columns are never exchanged), so the
// solve applies, step by step, the exchange and then the Gauss transform to
// b, and back-substitutes with U.  A column without a nonzero in its band is
// a singular matrix (PIRO_ERR_ZERO_PIVOT).

__global__ void k_lup_diag(int64_t N, int64_t W, int64_t bw, double shift, double *__restrict__ band)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x)
        band[r * W + bw] = shift;
}

// band(r, c) = shift*[r == c] + scale*M(r, c) in FP64 for every key in the table.
__global__ void k_lup_scatter(int64_t N, int64_t bw, int64_t W, const int64_t *__restrict__ keys,
                              const float *__restrict__ vals, int64_t ts, double shift, double scale,
                              double *__restrict__ band, int *err)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ts; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = keys[s];
        if (k < 0) continue;
        const int64_t r = k / N, d = k % N - r;
        if (d > bw || d < -bw) {
            atomicCAS(err, 0, 2);
            continue;
        }
        const double v = scale * (double)vals[s];
        band[r * W + d + bw] = d == 0 ? shift + v : v;
    }
}

constexpr int kPivThreads = 1024;

// Pivot search, row exchange and multipliers of pivot row ro (one block).
__global__ void __launch_bounds__(kPivThreads) k_lup_pivot(int64_t N, int64_t bw, int64_t W,
                                                           double *__restrict__ band, double *__restrict__ Lc,
                                                           int32_t *__restrict__ piv, int64_t ro, int *err)
{
    __shared__ double s_v[32];
    __shared__ int64_t s_i[32];
    __shared__ int64_t s_p;
    if (*((volatile int *)err)) return;  // an earlier pivot was zero
    const int64_t span = N - 1 - ro < bw ? N - 1 - ro : bw;
    // largest |a(ro+t, ro)|, the smallest t on a tie
    double best = -1.0;
    int64_t bi = 0;
    for (int64_t t = threadIdx.x; t <= span; t += blockDim.x) {
        const double v = fabs(band[(ro + t) * W + bw - t]);
        if (v > best) {
            best = v;
            bi = t;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, o);
        const int64_t oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
            best = ov;
            bi = oi;
        }
    }
    if (lane == 0) {
        s_v[warp] = best;
        s_i[warp] = bi;
    }
    __syncthreads();
    if (warp == 0) {
        best = lane < (int)(blockDim.x >> 5) ? s_v[lane] : -1.0;
        bi = lane < (int)(blockDim.x >> 5) ? s_i[lane] : 0;
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int64_t oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        if (lane == 0) {
            s_p = best > 0.0 ? bi : -1;
            piv[ro] = (int32_t)(ro + (best > 0.0 ? bi : 0));
            if (best <= 0.0 && atomicCAS(err, 0, 3) == 0) err[1] = (int)ro;
        }
    }
    __syncthreads();
    const int64_t p = s_p;
    if (p < 0) return;
    // exchange rows ro and ro+p over columns ro .. ro+2bw
    const int64_t cend = N - 1 - ro < 2 * bw ? N - 1 - ro : 2 * bw;
    if (p > 0)
        for (int64_t j = threadIdx.x; j <= cend; j += blockDim.x) {
            double *a = band + ro * W + bw + j;             // a(ro, ro+j)
            double *b = band + (ro + p) * W + bw - p + j;   // a(ro+p, ro+j)
            const double t = *a;
            *a = *b;
            *b = t;
        }
    __syncthreads();
    const double pv = band[ro * W + bw];
    for (int64_t t = 1 + threadIdx.x; t <= span; t += blockDim.x) {
        double *m = band + (ro + t) * W + bw - t;  // a(ro+t, ro)
        const double l = *m / pv;
        *m = l;
        Lc[ro * bw + t - 1] = l;
    }
}

// a(ro+i, ro+j) -= l(i) * a(ro, ro+j), i in 1..span, j in 1..2bw: block y
// takes row ro+1+y, its threads the columns.
constexpr int kUpdThreads = 256;

__global__ void __launch_bounds__(kUpdThreads) k_lup_update(int64_t N, int64_t bw, int64_t W,
                                                            double *__restrict__ band, int64_t ro,
                                                            const int *__restrict__ err)
{
    if (*((volatile const int *)err)) return;
    const int64_t i = (int64_t)blockIdx.y + 1;
    const double l = band[(ro + i) * W + bw - i];
    if (l == 0.0) return;
    const int64_t cend = N - 1 - ro < 2 * bw ? N - 1 - ro : 2 * bw;
    const double *u = band + ro * W + bw;          // u[j] = a(ro, ro+j)
    double *a = band + (ro + i) * W + bw - i;      // a[j] = a(ro+i, ro+j)
    for (int64_t j = 1 + (int64_t)blockIdx.x * kUpdThreads + threadIdx.x; j <= cend; j += (int64_t)gridDim.x * kUpdThreads)
        a[j] = fma(-l, u[j], a[j]);
}

// Solve with the factor (one block): y = b in FP64; per step ro the row
// exchange and the Gauss transform y[ro+t] -= l(t) y[ro]; then x from U,
// row by row from the last (each row a block-wide dot product over its at
// most 2bw entries right of the diagonal); x demoted to FP32.
__global__ void __launch_bounds__(kPivThreads) k_lup_solve(int64_t N, int64_t bw, int64_t W,
                                                           const double *__restrict__ band,
                                                           const double *__restrict__ Lc,
                                                           const int32_t *__restrict__ piv, const float *__restrict__ b,
                                                           double *__restrict__ y, float *__restrict__ x)
{
    __shared__ double s_w[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t r = threadIdx.x; r < N; r += blockDim.x) y[r] = (double)b[r];
    __syncthreads();
    for (int64_t ro = 0; ro < N; ++ro) {
        const int64_t p = piv[ro];
        if (p != ro && threadIdx.x == 0) {
            const double t = y[ro];
            y[ro] = y[p];
            y[p] = t;
        }
        __syncthreads();
        const double yr = y[ro];
        const int64_t span = N - 1 - ro < bw ? N - 1 - ro : bw;
        if (yr != 0.0)
            for (int64_t t = 1 + threadIdx.x; t <= span; t += blockDim.x) y[ro + t] = fma(-Lc[ro * bw + t - 1], yr, y[ro + t]);
        __syncthreads();
    }
    // back substitution: y[r] becomes x[r]
    for (int64_t r = N - 1; r >= 0; --r) {
        const int64_t cend = N - 1 - r < 2 * bw ? N - 1 - r : 2 * bw;
        const double *u = band + r * W + bw;  // u[j] = U(r, r+j)
        double s = 0.0;
        for (int64_t j = 1 + threadIdx.x; j <= cend; j += blockDim.x) s = fma(u[j], y[r + j], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) s_w[warp] = s;
        __syncthreads();
        if (warp == 0) {
            s = lane < (int)(blockDim.x >> 5) ? s_w[lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) y[r] = (y[r] - s) / u[0];
        }
        __syncthreads();
    }
    for (int64_t r = threadIdx.x; r < N; r += blockDim.x) x[r] = (float)y[r];
}

// Device layout of the factor buffer: band double[N][3bw+1], Lc double[N][bw],
// y double[N] (the solve's workspace), piv int32[N], err int[2].
struct LupLayout {
    int64_t W;
    size_t band, lc, y, piv, err, total;  // byte offsets
};

int lup_layout(int64_t N, int64_t bw, LupLayout *L)
{
    if (N < 1 || bw < 1) return PIRO_ERR_ARG;
    L->W = 3 * bw + 1;
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    L->band = 0;
    L->lc = up(sizeof(double) * (size_t)N * (size_t)L->W);
    L->y = L->lc + up(sizeof(double) * (size_t)N * (size_t)bw);
    L->piv = L->y + up(sizeof(double) * (size_t)N);
    L->err = L->piv + up(sizeof(int32_t) * (size_t)N);
    L->total = L->err + 256;
    return PIRO_OK;
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_ht_lu_reference(int64_t N, int64_t *keys, float *vals, int64_t ts, piro_stream_t stream)
{
    PIRO_ARG(N >= 1 && keys && vals && ts > 0 && N <= 46340, "piro_ht_lu_reference: bad arguments");
    cudaStream_t st = as_stream(stream);
    float *prow = nullptr;
    int32_t *cols = nullptr;
    int *err = nullptr;
    cudaError_t e = cudaMalloc(&prow, sizeof(float) * (size_t)(2 * N));
    if (e == cudaSuccess) e = cudaMalloc(&err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&cols, sizeof(int32_t) * (size_t)N);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    float *fac = prow + N;
    const size_t smem = lu_reference_smem_bytes(N, ts);
    const bool one_block = smem <= kLuSmemMax;
    if (e == cudaSuccess && one_block) {
        e = cudaFuncSetAttribute(k_lu_reference_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            k_lu_reference_smem<<<1, 1024, smem, st>>>(N, keys, vals, ts, err);
            e = cudaGetLastError();
        }
    }
    for (int64_t ro = 0; !one_block && ro < N - 1 && e == cudaSuccess; ++ro) {
        const int64_t ncol = N - ro, nrow = ncol - 1;
        k_lu_gather<<<grid_for(ncol + nrow, 256, 4), 256, 0, st>>>(N, ro, ncol, nrow, keys, vals, ts, prow, fac);
        k_lu_fill<<<1, 1, 0, st>>>(N, ro, keys, vals, ts, prow, fac, cols, err);
        k_lu_round<<<grid_for(nrow * ncol, 256, 4), 256, 0, st>>>(N, ro, keys, vals, ts, prow, fac);
        e = cudaGetLastError();
    }
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(prow);
    cudaFree(cols);
    cudaFree(err);
    if (e != cudaSuccess) {
        set_error("piro_ht_lu_reference: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    if (herr) {
        set_error("piro_ht_lu_reference: the hash table has no room for the fill-in (raise its size)");
        return PIRO_ERR_TABLE_FULL;
    }
    return PIRO_OK;
}

extern "C" int piro_ht_lu_band_bytes(int64_t N, int64_t bw, size_t *bytes)
{
    LupLayout L;
    PIRO_ARG(bytes && N >= 1 && bw >= 1 && bw <= N && lup_layout(N, bw, &L) == PIRO_OK,
             "piro_ht_lu_band_bytes: bad arguments");
    *bytes = L.total;
    return PIRO_OK;
}

extern "C" int piro_ht_lu_factor(int64_t N, int64_t bw, const int64_t *keys, const float *vals, int64_t ts,
                                 float shift, float scale, void *band, size_t band_bytes, piro_stream_t stream)
{
    LupLayout L;
    PIRO_ARG(keys && vals && ts > 0 && band && N >= 1 && bw >= 1 && bw <= N && N < ((int64_t)1 << 31) &&
                 lup_layout(N, bw, &L) == PIRO_OK,
             "piro_ht_lu_factor: bad arguments");
    PIRO_ARG(band_bytes >= L.total, "piro_ht_lu_factor: band buffer too small (piro_ht_lu_band_bytes)");
    PIRO_ARG(bw <= 65535, "piro_ht_lu_factor: bandwidth above 65535");
    cudaStream_t st = as_stream(stream);
    char *base = static_cast<char *>(band);
    double *AB = reinterpret_cast<double *>(base + L.band);
    double *Lc = reinterpret_cast<double *>(base + L.lc);
    int32_t *piv = reinterpret_cast<int32_t *>(base + L.piv);
    int *err = reinterpret_cast<int *>(base + L.err);
    const int64_t W = L.W;
    PIRO_CUDA(cudaMemsetAsync(AB, 0, sizeof(double) * (size_t)N * (size_t)W, st));
    PIRO_CUDA(cudaMemsetAsync(err, 0, 2 * sizeof(int), st));
    k_lup_diag<<<grid_for(N, 256, 8), 256, 0, st>>>(N, W, bw, (double)shift, AB);
    k_lup_scatter<<<grid_for(ts, 256, 8), 256, 0, st>>>(N, bw, W, keys, vals, ts, (double)shift, (double)scale, AB,
                                                        err);
    PIRO_CHECK_LAUNCH("k_lup_scatter");
    int herr[2] = {0, 0};
    PIRO_CUDA(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (herr[0] == 2) {
        set_error("piro_ht_lu_factor: the table holds an entry outside the bandwidth %lld", (long long)bw);
        return PIRO_ERR_ARG;
    }
    for (int64_t ro = 0; ro < N; ++ro) {
        k_lup_pivot<<<1, kPivThreads, 0, st>>>(N, bw, W, AB, Lc, piv, ro, err);
        const int64_t span = N - 1 - ro < bw ? N - 1 - ro : bw;
        const int64_t cend = N - 1 - ro < 2 * bw ? N - 1 - ro : 2 * bw;
        if (span > 0 && cend > 0) {
            const dim3 grid((unsigned)cdiv(cend, kUpdThreads), (unsigned)span);
            k_lup_update<<<grid, kUpdThreads, 0, st>>>(N, bw, W, AB, ro, err);
        }
    }
    PIRO_CHECK_LAUNCH("k_lup_update");
    PIRO_CUDA(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (herr[0] == 3) {
        set_error("piro_ht_lu_factor: singular matrix: column %d has no nonzero at or below the diagonal", herr[1]);
        return PIRO_ERR_ZERO_PIVOT;
    }
    return PIRO_OK;
}

extern "C" int piro_ht_lu_solve(int64_t N, int64_t bw, void *band, size_t band_bytes, const float *b, float *x,
                                piro_stream_t stream)
{
    LupLayout L;
    PIRO_ARG(band && b && x && N >= 1 && bw >= 1 && bw <= N && lup_layout(N, bw, &L) == PIRO_OK,
             "piro_ht_lu_solve: bad arguments");
    PIRO_ARG(band_bytes >= L.total, "piro_ht_lu_solve: band buffer too small (piro_ht_lu_band_bytes)");
    cudaStream_t st = as_stream(stream);
    char *base = static_cast<char *>(band);
    k_lup_solve<<<1, kPivThreads, 0, st>>>(N, bw, L.W, reinterpret_cast<const double *>(base + L.band),
                                          reinterpret_cast<const double *>(base + L.lc),
                                          reinterpret_cast<const int32_t *>(base + L.piv), b,
                                          reinterpret_cast<double *>(base + L.y), x);
    PIRO_CHECK_LAUNCH("k_lup_solve");
    return PIRO_OK;
}

extern "C" int piro_ht_lu_pivots(int64_t N, int64_t bw, const void *band, size_t band_bytes, int32_t *piv_host)
{
    LupLayout L;
    PIRO_ARG(band && piv_host && N >= 1 && bw >= 1 && bw <= N && lup_layout(N, bw, &L) == PIRO_OK &&
                 band_bytes >= L.total,
             "piro_ht_lu_pivots: bad arguments");
    PIRO_CUDA(cudaMemcpy(piv_host, static_cast<const char *>(band) + L.piv, sizeof(int32_t) * (size_t)N,
                         cudaMemcpyDeviceToHost));
    return PIRO_OK;
}

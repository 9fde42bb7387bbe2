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
// dgbtrf), by panels of 16 columns: one block factors the panel in shared
// memory, then the exchanges and the pivot rows' U part right of it, then a
// tiled update of the (bw x 2bw) block below and right of it (the column-by-
// column form -- one pivot launch and one rank-1 update launch per row --
// remains, and gives the same bits).  The solve (one block, FP64) replays the
// exchanges and Gauss transforms on b and back-substitutes.
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

// The same factorization by panels of nb columns (LAPACK's blocked dgbtrf
// scheme), bit for bit the result of the column-by-column launches above:
//   1. k_lupb_panel (one block): the panel's rows j0 .. j0+nb-1+bw and
//      columns j0 .. j0+nb-1 in shared memory; per column the pivot search,
//      the exchange inside the panel, the multipliers (to the band and Lc)
//      and the rank-1 update of the panel's later columns, each element by
//      the same fma as the column launches.  The exchanges of the columns
//      right of the panel are deferred; Lw gets the multipliers as the later
//      exchanges of the panel see them (the multiplier of step k for the row
//      that ends at position r is the one stored at the position that row
//      held at step k).
//   2. k_lupb_rows (a thread per column right of the panel): the panel's nb
//      exchanges in order, then the pivot rows j0 .. j0+nb-1 updated with
//      Lw (forward substitution with the unit lower triangle).
//   3. k_lupb_update (64 x 64 tiles): a(r, c) -= sum over k of Lw(r, k) *
//      a(j0+k, c) for the rows below the panel, k ascending, as the column
//      launches apply their steps.
// Every update is skipped where the column launches skip it: a zero
// multiplier, or a column more than 2bw right of the step's pivot.
constexpr int kLuNbMax = 16;
constexpr int kLuTile = 64;

__device__ __forceinline__ double *band_at(double *band, int64_t W, int64_t bw, int64_t r, int64_t c)
{
    return band + r * W + (c - r + bw);
}

__device__ __forceinline__ bool in_band(int64_t bw, int64_t r, int64_t c)
{
    const int64_t d = c - r + bw;
    return d >= 0 && d <= 3 * bw;
}

constexpr int kPanelThreads = 1024;

__global__ void __launch_bounds__(kPanelThreads) k_lupb_panel(int64_t N, int64_t bw, int64_t W,
                                                            double *__restrict__ band, double *__restrict__ Lc,
                                                            int32_t *__restrict__ piv, double *__restrict__ Lw,
                                                            int64_t j0, int nbp, int nb, int *err)
{
    extern __shared__ double s_p[];  // [R][ld], ld = nb + 1: a column read across rows is bank-conflict free
    __shared__ double s_v[32];
    __shared__ int s_i[32];
    __shared__ int s_prow;
    __shared__ int32_t s_piv[kLuNbMax];
    __shared__ double s_pr[kLuNbMax];  // the pivot row (after its exchange), columns jj .. of the step
    if (*((volatile int *)err)) return;
    const int ld = nb + 1;
    const int64_t rmax = j0 + nbp - 1 + bw < N - 1 ? j0 + nbp - 1 + bw : N - 1;
    const int R = (int)(rmax - j0 + 1);
    for (int idx = threadIdx.x; idx < R * nbp; idx += blockDim.x) {
        const int r = idx / nbp, cc = idx - r * nbp;
        const int64_t gr = j0 + r, gc = j0 + cc;
        s_p[r * ld + cc] = in_band(bw, gr, gc) ? *band_at(band, W, bw, gr, gc) : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // argmax of |column jj| over rows jj .. jj+span (first on a tie), from the
    // per-thread candidates (best, bi) of the caller; the result in s_prow
    auto pick = [&](double best, int bi, int jj) {
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
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
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ov > best || (ov == best && oi < bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            const int64_t j = j0 + jj;
            if (lane == 0) {
                s_prow = best > 0.0 ? bi : -1;
                piv[j] = (int32_t)(j + (best > 0.0 ? bi : 0));
                s_piv[jj] = (int32_t)(j + (best > 0.0 ? bi : 0));
                if (best <= 0.0 && atomicCAS(err, 0, 3) == 0) err[1] = (int)j;
            }
            // the pivot row as the step's exchange leaves it: row jj + p over the
            // columns jj .. jj + cend of the panel
            const int p = __shfl_sync(0xffffffffu, bi, 0);
            const int64_t cend = N - 1 - j < 2 * bw ? N - 1 - j : 2 * bw;
            const int ccend = (int)(jj + cend < nbp - 1 ? jj + cend : nbp - 1);
            const int cc = jj + lane;
            if (cc <= ccend) s_pr[cc] = s_p[(jj + p) * ld + cc];
        }
        __syncthreads();
    };
    {   // the first column's pivot
        const int span0 = (int)(N - 1 - j0 < bw ? N - 1 - j0 : bw);
        double best = -1.0;
        int bi = 0;
        for (int t = threadIdx.x; t <= span0; t += blockDim.x) {
            const double v = fabs(s_p[t * ld]);
            if (v > best) {
                best = v;
                bi = t;
            }
        }
        pick(best, bi, 0);
    }
    for (int jj = 0; jj < nbp; ++jj) {
        const int64_t j = j0 + jj;
        const int span = (int)(N - 1 - j < bw ? N - 1 - j : bw);
        const int64_t cend = N - 1 - j < 2 * bw ? N - 1 - j : 2 * bw;  // columns j .. j+cend take part
        const int p = s_prow;
        if (p < 0) return;  // singular: the later launches see *err and return
        const int ccend = (int)(jj + cend < nbp - 1 ? jj + cend : nbp - 1);  // last panel column of this step
        // per row below the pivot: the multiplier, the update of the row's later
        // panel columns, and the row's candidate for the next column's pivot.
        // The exchange happens here: the thread of row jj + p takes row jj's
        // entries as its own and writes the pivot row (s_pr) to position jj; no
        // other thread reads either position in this phase.
        const double pv = s_pr[jj];
        const bool next = jj + 1 < nbp;
        const int span_n = next ? (int)(N - 1 - (j + 1) < bw ? N - 1 - (j + 1) : bw) : -1;  // next column's rows
        double best = -1.0;
        int bi = 0;
        for (int t = 1 + threadIdx.x; t <= span || (next && t <= span_n + 1); t += blockDim.x) {
            double *row = s_p + (jj + t) * ld;
            if (t <= span) {
                if (t == p)
                    for (int cc = jj; cc <= ccend; ++cc) {
                        row[cc] = s_p[jj * ld + cc];
                        s_p[jj * ld + cc] = s_pr[cc];
                    }
                const double l = row[jj] / pv;
                row[jj] = l;
                Lc[j * bw + t - 1] = l;
                if (l != 0.0)
                    for (int cc = jj + 1; cc <= ccend; ++cc) row[cc] = fma(-l, s_pr[cc], row[cc]);
            }
            if (next && t <= span_n + 1) {  // row j + t is candidate t - 1 of column j + 1
                const double v = fabs(row[jj + 1]);
                if (v > best) {
                    best = v;
                    bi = t - 1;
                }
            }
        }
        if (next) pick(best, bi, jj + 1);
        else __syncthreads();
    }
    for (int idx = threadIdx.x; idx < R * nbp; idx += blockDim.x) {
        const int r = idx / nbp, cc = idx - r * nbp;
        const int64_t gr = j0 + r, gc = j0 + cc;
        if (in_band(bw, gr, gc)) *band_at(band, W, bw, gr, gc) = s_p[r * ld + cc];
    }
    // Lw[r][k]: the multiplier of step k for the row that ends at position j0 + r
    for (int idx = threadIdx.x; idx < R * nbp; idx += blockDim.x) {
        const int r = idx / nbp, k = idx - r * nbp;
        int64_t q = j0 + r;
        for (int kk = nbp - 1; kk > k; --kk) {
            const int64_t pk = s_piv[kk];
            if (q == j0 + kk) q = pk;
            else if (q == pk) q = j0 + kk;
        }
        const int64_t rel = q - (j0 + k);
        const int64_t span_k = N - 1 - (j0 + k) < bw ? N - 1 - (j0 + k) : bw;
        Lw[(int64_t)r * kLuNbMax + k] = rel >= 1 && rel <= span_k ? s_p[(q - j0) * ld + k] : 0.0;
    }
}

// Right of the panel: the deferred exchanges, then the pivot rows' U part.
__global__ void k_lupb_rows(int64_t N, int64_t bw, int64_t W, double *__restrict__ band,
                            const int32_t *__restrict__ piv, const double *__restrict__ Lw, int64_t j0, int nbp,
                            const int *err)
{
    if (*((volatile const int *)err)) return;
    const int64_t cmax = j0 + nbp - 1 + 2 * bw < N - 1 ? j0 + nbp - 1 + 2 * bw : N - 1;
    const int64_t c = j0 + nbp + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c > cmax) return;
    for (int k = 0; k < nbp; ++k) {
        const int64_t j = j0 + k, p = piv[j];
        if (p != j && c <= j + 2 * bw) {
            double *a = band_at(band, W, bw, j, c), *b = band_at(band, W, bw, p, c);
            const double t = *a;
            *a = *b;
            *b = t;
        }
    }
    for (int i = 1; i < nbp; ++i) {
        double *a = band_at(band, W, bw, j0 + i, c);
        if (!in_band(bw, j0 + i, c)) continue;
        double acc = *a;
        for (int k = 0; k < i; ++k) {
            const double l = Lw[(int64_t)i * kLuNbMax + k];
            if (l != 0.0 && c <= j0 + k + 2 * bw) acc = fma(-l, *band_at(band, W, bw, j0 + k, c), acc);
        }
        *a = acc;
    }
}

// Rows below the panel: 64 x 64 tiles, 256 threads, 4 x 4 elements each
// (rows ty + 16 m, columns tx + 16 n: consecutive threads on consecutive
// columns).
__global__ void __launch_bounds__(256) k_lupb_update(int64_t N, int64_t bw, int64_t W, double *__restrict__ band,
                                                     const double *__restrict__ Lw, int64_t j0, int nbp,
                                                     const int *err)
{
    __shared__ double s_l[kLuTile][kLuNbMax + 1];
    __shared__ double s_u[kLuNbMax][kLuTile];
    if (*((volatile const int *)err)) return;
    const int64_t rfirst = j0 + nbp;
    const int64_t rmax = j0 + nbp - 1 + bw < N - 1 ? j0 + nbp - 1 + bw : N - 1;
    const int64_t cmax = j0 + nbp - 1 + 2 * bw < N - 1 ? j0 + nbp - 1 + 2 * bw : N - 1;
    const int64_t r0 = rfirst + (int64_t)blockIdx.y * kLuTile, c0 = rfirst + (int64_t)blockIdx.x * kLuTile;
    if (r0 > rmax || c0 > cmax) return;
    for (int idx = threadIdx.x; idx < kLuTile * kLuNbMax; idx += blockDim.x) {
        const int r = idx / kLuNbMax, k = idx - r * kLuNbMax;
        const int64_t gr = r0 + r;
        s_l[r][k] = (k < nbp && gr <= rmax) ? Lw[(gr - j0) * kLuNbMax + k] : 0.0;
    }
    for (int idx = threadIdx.x; idx < kLuNbMax * kLuTile; idx += blockDim.x) {
        const int k = idx / kLuTile, cc = idx - k * kLuTile;
        const int64_t gc = c0 + cc;
        s_u[k][cc] = (k < nbp && gc <= cmax && gc <= j0 + k + 2 * bw) ? *band_at(band, W, bw, j0 + k, gc) : 0.0;
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // all 16 elements loaded first (16 loads in flight per thread), then the
    // steps in order on the 16 accumulators
    double acc[4][4];
    unsigned ok = 0, upd = 0;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const int64_t gr = r0 + ty + 16 * m, gc = c0 + tx + 16 * n;
            const bool e = gr <= rmax && gc <= cmax && in_band(bw, gr, gc);
            acc[m][n] = e ? *band_at(band, W, bw, gr, gc) : 0.0;
            ok |= e ? 1u << (4 * m + n) : 0u;
        }
    for (int k = 0; k < nbp; ++k) {
        double l[4], u[4];
        bool cu[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) l[m] = s_l[ty + 16 * m][k];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            u[n] = s_u[k][tx + 16 * n];
            cu[n] = c0 + tx + 16 * n <= j0 + k + 2 * bw;
        }
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < 4; ++n)
                if (l[m] != 0.0 && cu[n]) {
                    acc[m][n] = fma(-l[m], u[n], acc[m][n]);
                    upd |= 1u << (4 * m + n);
                }
    }
    upd &= ok;
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int n = 0; n < 4; ++n)
            if (upd & (1u << (4 * m + n)))
                *band_at(band, W, bw, r0 + ty + 16 * m, c0 + tx + 16 * n) = acc[m][n];
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

// The solve by the same 16-row panels.  Lp holds, per panel of 16 steps
// starting at j0, the multipliers as the panel's later exchanges see them
// ([bw + 16][16] doubles per panel, row r = position j0 + r), built once per
// factorization from Lc and the pivots.  The forward pass per panel: the 16
// exchanges on y, the unit lower triangle (one thread, steps in order), then
// the rows below it (a thread per row, steps in order); the backward pass per
// panel from the last: for each of its rows the dot product with the solved
// x right of the panel (a warp per row), then the triangle (one thread).  Two
// block barriers per panel and pass, against two per row in k_lup_solve.
constexpr int kLuSolveNb = 16;

__global__ void k_lup_lw_from_lc(int64_t N, int64_t bw, const double *__restrict__ Lc,
                                 const int32_t *__restrict__ piv, double *__restrict__ Lp)
{
    const int64_t R = bw + kLuSolveNb;
    const int64_t npan = cdiv(N, kLuSolveNb);
    const int64_t total = npan * R * kLuSolveNb;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pi = idx / (R * kLuSolveNb);
        const int64_t rem = idx - pi * R * kLuSolveNb;
        const int r = (int)(rem / kLuSolveNb), k = (int)(rem - (int64_t)r * kLuSolveNb);
        const int64_t j0 = pi * kLuSolveNb;
        const int nbp = (int)(N - j0 < kLuSolveNb ? N - j0 : kLuSolveNb);
        double v = 0.0;
        if (k < nbp && j0 + r < N) {
            int64_t q = j0 + r;
            for (int kk = nbp - 1; kk > k; --kk) {
                const int64_t pk = piv[j0 + kk];
                if (q == j0 + kk) q = pk;
                else if (q == pk) q = j0 + kk;
            }
            const int64_t rel = q - (j0 + k);
            const int64_t span_k = N - 1 - (j0 + k) < bw ? N - 1 - (j0 + k) : bw;
            if (rel >= 1 && rel <= span_k) v = Lc[(j0 + k) * bw + rel - 1];
        }
        Lp[idx] = v;
    }
}

__global__ void __launch_bounds__(kPivThreads) k_lup_solve_panels(int64_t N, int64_t bw, int64_t W,
                                                                  const double *__restrict__ band,
                                                                  const double *__restrict__ Lp,
                                                                  const int32_t *__restrict__ piv,
                                                                  const float *__restrict__ b, double *__restrict__ y,
                                                                  float *__restrict__ x)
{
    // The sequential parts of a panel (its exchanges, its triangle) run in one
    // thread on shared-memory copies that the block loads in parallel first,
    // so that no dependent chain waits on global memory.
    constexpr int P = kLuSolveNb;
    __shared__ double s_y[P];        // y of the panel's rows
    __shared__ double s_t[P][P + 1]; // the panel's triangle: Lw (forward) or U (backward)
    __shared__ double s_far[P];      // y at each step's pivot row, before the panel's exchanges
    __shared__ int64_t s_pos[P];     // rows outside the panel that the exchanges touch, and their values
    __shared__ double s_val[P];
    __shared__ int32_t s_piv[P];
    __shared__ double s_dot[P];
    const int64_t R = bw + P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int64_t r = threadIdx.x; r < N; r += blockDim.x) y[r] = (double)b[r];
    __syncthreads();
    const int64_t npan = cdiv(N, P);
    for (int64_t pi = 0; pi < npan; ++pi) {
        const int64_t j0 = pi * P;
        const int nbp = (int)(N - j0 < P ? N - j0 : P);
        const double *lw = Lp + pi * R * P;
        // parallel loads: pivots, y of the panel and of the pivot rows, the triangle of Lw
        if (threadIdx.x < nbp) {
            const int32_t p = piv[j0 + threadIdx.x];
            s_piv[threadIdx.x] = p;
            s_y[threadIdx.x] = y[j0 + threadIdx.x];
            s_far[threadIdx.x] = y[p];
        }
        for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
            const int i = t / P, k = t - i * P;
            s_t[i][k] = (i < nbp && k < i) ? lw[i * P + k] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int nfar = 0;
            for (int k = 0; k < nbp; ++k) {
                const int64_t p = s_piv[k];
                if (p == j0 + k) continue;
                double *vb;
                if (p < j0 + nbp) {
                    vb = &s_y[p - j0];
                } else {
                    int f = 0;
                    while (f < nfar && s_pos[f] != p) ++f;
                    if (f == nfar) {  // first touch in this panel: y[p] as loaded
                        s_pos[f] = p;
                        s_val[f] = s_far[k];
                        ++nfar;
                    }
                    vb = &s_val[f];
                }
                const double t = s_y[k];
                s_y[k] = *vb;
                *vb = t;
            }
            for (int f = 0; f < nfar; ++f) y[s_pos[f]] = s_val[f];
        }
        __syncwarp();
        if (warp == 0) {
            // the unit lower triangle by columns: lane i takes row i, step k's
            // y_k reaches the lanes by a shuffle (each row's updates in k order)
            double yi = lane < nbp ? s_y[lane] : 0.0;
            for (int k = 0; k < nbp - 1; ++k) {
                const double yk = __shfl_sync(0xffffffffu, yi, k);
                const double l = lane > k && lane < nbp ? s_t[lane][k] : 0.0;
                if (l != 0.0 && yk != 0.0) yi = fma(-l, yk, yi);
            }
            if (lane < nbp) s_y[lane] = yi;
        }
        __syncthreads();
        if (threadIdx.x < nbp) y[j0 + threadIdx.x] = s_y[threadIdx.x];
        const int64_t rmax = j0 + nbp - 1 + bw < N - 1 ? j0 + nbp - 1 + bw : N - 1;
        for (int64_t r = j0 + nbp + threadIdx.x; r <= rmax; r += blockDim.x) {
            double acc = y[r];
            for (int k = 0; k < nbp; ++k) {
                const double l = lw[(r - j0) * P + k];
                if (l != 0.0 && s_y[k] != 0.0) acc = fma(-l, s_y[k], acc);
            }
            y[r] = acc;
        }
        __syncthreads();
    }
    // back substitution, panels from the last; y[r] becomes x[r]
    for (int64_t pi = npan - 1; pi >= 0; --pi) {
        const int64_t j0 = pi * P;
        const int nbp = (int)(N - j0 < P ? N - j0 : P);
        const int64_t jend = j0 + nbp;  // first column right of the panel
        for (int i = warp; i < nbp; i += nwarp) {
            const int64_t r = j0 + i;
            const int64_t cmax = r + 2 * bw < N - 1 ? r + 2 * bw : N - 1;
            double sum = 0.0;
            for (int64_t c = jend + lane; c <= cmax; c += 32) sum = fma(band[r * W + (c - r + bw)], y[c], sum);
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) s_dot[i] = sum;
        }
        // U of the panel's rows and columns (diagonal included), and their y
        for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
            const int i = t / P, c = t - i * P;
            const int64_t r = j0 + i, gc = j0 + c;
            s_t[i][c] = (i < nbp && c < nbp && c >= i && gc <= r + 2 * bw) ? band[r * W + (gc - r + bw)] : 0.0;
        }
        if (threadIdx.x < nbp) s_y[threadIdx.x] = y[j0 + threadIdx.x];
        __syncthreads();
        if (warp == 0) {
            // U by columns from the last: lane i holds row i's sum; x_c, once
            // solved, reaches the lanes above it by a shuffle
            double sum = lane < nbp ? s_dot[lane] : 0.0, yi = lane < nbp ? s_y[lane] : 0.0;
            for (int c = nbp - 1; c >= 0; --c) {
                if (lane == c) yi = (yi - sum) / s_t[c][c];
                const double xc = __shfl_sync(0xffffffffu, yi, c);
                if (lane < c) sum = fma(s_t[lane][c], xc, sum);
            }
            if (lane < nbp) s_y[lane] = yi;
        }
        __syncthreads();
        if (threadIdx.x < nbp) y[j0 + threadIdx.x] = s_y[threadIdx.x];
        __syncthreads();
    }
    for (int64_t r = threadIdx.x; r < N; r += blockDim.x) x[r] = (float)y[r];
}

// The same solve with y kept in shared memory: a ring of WS = 2bw + 16
// doubles holds rows [j0, j0 + WS) while panel j0 is worked on (every row a
// panel step touches lies within bw + 15 of j0 in the forward pass and within
// 2bw + 15 in the backward pass); rows leave for global memory as the panels
// move on and enter from b (forward) or from the forward result (backward).
// Only the multipliers, the pivots and U's rows are read from global memory.
// Same arithmetic as k_lup_solve_panels, bit for bit.
__global__ void __launch_bounds__(kPivThreads) k_lup_solve_ring(int64_t N, int64_t bw, int64_t W,
                                                                const double *__restrict__ band,
                                                                const double *__restrict__ Lp,
                                                                const int32_t *__restrict__ piv,
                                                                const float *__restrict__ b, double *__restrict__ y,
                                                                float *__restrict__ x)
{
    constexpr int P = kLuSolveNb;
    extern __shared__ double s_ring[];
    __shared__ double s_y[P];
    __shared__ double s_t[P][P + 1];
    __shared__ int32_t s_piv[P];
    __shared__ double s_dot[P];
    const uint32_t WS = (uint32_t)(2 * bw + P);
    auto slot = [WS](int64_t r) { return (uint32_t)r % WS; };  // rows < 2^31
    const uint32_t step_b = blockDim.x % WS, step_w = 32u % WS;  // ring moves of a block / warp stride
    const int64_t R = bw + P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int64_t npan = cdiv(N, P);
    for (int64_t r = threadIdx.x; r < N && r < (int64_t)WS; r += blockDim.x) s_ring[r] = (double)b[r];
    __syncthreads();
    for (int64_t pi = 0; pi < npan; ++pi) {
        const int64_t j0 = pi * P;
        const int nbp = (int)(N - j0 < P ? N - j0 : P);
        const double *lw = Lp + pi * R * P;
        if (threadIdx.x < nbp) s_piv[threadIdx.x] = piv[j0 + threadIdx.x];
        for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
            const int i = t / P, k = t - i * P;
            s_t[i][k] = (i < nbp && k < i) ? lw[i * P + k] : 0.0;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < nbp; ++k) {
                const int64_t p = s_piv[k];
                if (p == j0 + k) continue;
                double *a = &s_ring[slot(j0 + k)], *c = &s_ring[slot(p)];
                const double t = *a;
                *a = *c;
                *c = t;
            }
        __syncwarp();
        if (warp == 0) {
            double yi = lane < nbp ? s_ring[slot(j0 + lane)] : 0.0;
            for (int k = 0; k < nbp - 1; ++k) {
                const double yk = __shfl_sync(0xffffffffu, yi, k);
                const double l = lane > k && lane < nbp ? s_t[lane][k] : 0.0;
                if (l != 0.0 && yk != 0.0) yi = fma(-l, yk, yi);
            }
            if (lane < nbp) {
                s_y[lane] = yi;
                s_ring[slot(j0 + lane)] = yi;
            }
        }
        __syncthreads();
        const int64_t rmax = j0 + nbp - 1 + bw < N - 1 ? j0 + nbp - 1 + bw : N - 1;
        uint32_t sr = slot(j0 + nbp + threadIdx.x);
        for (int64_t r = j0 + nbp + threadIdx.x; r <= rmax; r += blockDim.x) {
            double *yr = &s_ring[sr];
            sr += step_b;
            sr = sr >= WS ? sr - WS : sr;
            double acc = *yr;
            for (int k = 0; k < nbp; ++k) {
                const double l = lw[(r - j0) * P + k];
                if (l != 0.0 && s_y[k] != 0.0) acc = fma(-l, s_y[k], acc);
            }
            *yr = acc;
        }
        __syncthreads();
        // rows j0 .. j0+nbp-1 are done with the forward pass; rows WS further on enter
        if (threadIdx.x < nbp) {
            const int64_t r = j0 + threadIdx.x, rn = r + WS;
            y[r] = s_ring[slot(r)];
            if (rn < N) s_ring[slot(rn)] = (double)b[rn];
        }
    }
    __syncthreads();
    // back substitution, panels from the last; the ring holds rows [j0, j0 + WS)
    for (int64_t pi = npan - 1; pi >= 0; --pi) {
        const int64_t j0 = pi * P;
        const int nbp = (int)(N - j0 < P ? N - j0 : P);
        const int64_t jend = j0 + nbp;
        if (pi == npan - 1) {
            for (int64_t r = j0 + threadIdx.x; r < N; r += blockDim.x) s_ring[slot(r)] = y[r];
        } else if (threadIdx.x < nbp) {  // row r + WS (solved) leaves, row r (forward result) enters
            const int64_t r = j0 + threadIdx.x, ro = r + WS;
            if (ro < N) y[ro] = s_ring[slot(ro)];
            s_ring[slot(r)] = y[r];
        }
        __syncthreads();
        for (int i = warp; i < nbp; i += nwarp) {
            const int64_t r = j0 + i;
            const int64_t cmax = r + 2 * bw < N - 1 ? r + 2 * bw : N - 1;
            const double *u = band + r * W + (bw - r);  // u[c] = U(r, c)
            double sum = 0.0;
            int64_t c = jend + lane;
            uint32_t sc = slot(c);
#pragma unroll 4
            for (; c <= cmax; c += 32) {
                sum = fma(u[c], s_ring[sc], sum);
                sc += step_w;
                sc = sc >= WS ? sc - WS : sc;
            }
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
            if (lane == 0) s_dot[i] = sum;
        }
        for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
            const int i = t / P, c = t - i * P;
            const int64_t r = j0 + i, gc = j0 + c;
            s_t[i][c] = (i < nbp && c < nbp && c >= i && gc <= r + 2 * bw) ? band[r * W + (gc - r + bw)] : 0.0;
        }
        __syncthreads();
        if (warp == 0) {
            double sum = lane < nbp ? s_dot[lane] : 0.0, yi = lane < nbp ? s_ring[slot(j0 + lane)] : 0.0;
            for (int c = nbp - 1; c >= 0; --c) {
                if (lane == c) yi = (yi - sum) / s_t[c][c];
                const double xc = __shfl_sync(0xffffffffu, yi, c);
                if (lane < c) sum = fma(s_t[lane][c], xc, sum);
            }
            if (lane < nbp) s_ring[slot(j0 + lane)] = yi;
        }
        __syncthreads();
    }
    for (int64_t r = threadIdx.x; r < N && r < (int64_t)WS; r += blockDim.x) y[r] = s_ring[slot(r)];
    __syncthreads();
    for (int64_t r = threadIdx.x; r < N; r += blockDim.x) x[r] = (float)y[r];
}

// Device layout of the factor buffer: band double[N][3bw+1], Lc double[N][bw],
// y double[N] (the solve's workspace), piv int32[N], err int[2], Lw
// double[bw + 16][16] (the blocked factorization's panel multipliers), Lp
// double[ceil(N/16)][bw + 16][16] (the solve's panel multipliers).
struct LupLayout {
    int64_t W;
    size_t band, lc, y, piv, err, lw, lp, total;  // byte offsets
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
    L->lw = L->err + 256;
    L->lp = L->lw + up(sizeof(double) * (size_t)(bw + kLuNbMax) * kLuNbMax);
    L->total = L->lp + up(sizeof(double) * (size_t)cdiv(N, kLuSolveNb) * (size_t)(bw + kLuSolveNb) * kLuSolveNb);
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
    // panel width: the widest of 16, 8, 4 whose panel (bw + nb rows) fits in
    // 200 KB of shared memory; PIRO_LU_UNBLOCKED=1 forces the column launches
    int nb = 0;
    for (int t = kLuNbMax; t >= 4 && !nb; t /= 2)
        if ((size_t)(bw + t) * (t + 1) * sizeof(double) <= 200 * 1024) nb = t;
    const char *ub = getenv("PIRO_LU_UNBLOCKED");
    if (ub && ub[0] == '1') nb = 0;
    if (nb) {
        double *Lw = reinterpret_cast<double *>(base + L.lw);
        const size_t smem = (size_t)(bw + nb) * (nb + 1) * sizeof(double);
        PIRO_CUDA(cudaFuncSetAttribute(k_lupb_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (int64_t j0 = 0; j0 < N; j0 += nb) {
            const int nbp = (int)(N - j0 < nb ? N - j0 : nb);
            k_lupb_panel<<<1, kPanelThreads, smem, st>>>(N, bw, W, AB, Lc, piv, Lw, j0, nbp, nb, err);
            const int64_t rmax = j0 + nbp - 1 + bw < N - 1 ? j0 + nbp - 1 + bw : N - 1;
            const int64_t cmax = j0 + nbp - 1 + 2 * bw < N - 1 ? j0 + nbp - 1 + 2 * bw : N - 1;
            const int64_t ncols = cmax - (j0 + nbp) + 1, nrows = rmax - (j0 + nbp) + 1;
            if (ncols > 0) {
                k_lupb_rows<<<(unsigned)cdiv(ncols, 128), 128, 0, st>>>(N, bw, W, AB, piv, Lw, j0, nbp, err);
                if (nrows > 0)
                    k_lupb_update<<<dim3((unsigned)cdiv(ncols, kLuTile), (unsigned)cdiv(nrows, kLuTile)), 256, 0,
                                    st>>>(N, bw, W, AB, Lw, j0, nbp, err);
            }
        }
        PIRO_CHECK_LAUNCH("k_lupb_update");
    } else {
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
    }
    PIRO_CUDA(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (herr[0] == 3) {
        set_error("piro_ht_lu_factor: singular matrix: column %d has no nonzero at or below the diagonal", herr[1]);
        return PIRO_ERR_ZERO_PIVOT;
    }
    const int64_t lp_items = cdiv(N, kLuSolveNb) * (bw + kLuSolveNb) * kLuSolveNb;
    k_lup_lw_from_lc<<<grid_for(lp_items, 256, 8), 256, 0, st>>>(N, bw, Lc, piv,
                                                                   reinterpret_cast<double *>(base + L.lp));
    PIRO_CHECK_LAUNCH("k_lup_lw_from_lc");
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
    const char *ub = getenv("PIRO_LU_UNBLOCKED");
    if (ub && ub[0] == '1') {
        k_lup_solve<<<1, kPivThreads, 0, st>>>(N, bw, L.W, reinterpret_cast<const double *>(base + L.band),
                                              reinterpret_cast<const double *>(base + L.lc),
                                              reinterpret_cast<const int32_t *>(base + L.piv), b,
                                              reinterpret_cast<double *>(base + L.y), x);
        PIRO_CHECK_LAUNCH("k_lup_solve");
    } else if ((size_t)(2 * bw + kLuSolveNb) * sizeof(double) <= 160 * 1024 &&
               !(getenv("PIRO_LU_NO_RING") && getenv("PIRO_LU_NO_RING")[0] == '1')) {
        const size_t smem = (size_t)(2 * bw + kLuSolveNb) * sizeof(double);
        PIRO_CUDA(cudaFuncSetAttribute(k_lup_solve_ring, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_lup_solve_ring<<<1, kPivThreads, smem, st>>>(N, bw, L.W, reinterpret_cast<const double *>(base + L.band),
                                                       reinterpret_cast<const double *>(base + L.lp),
                                                       reinterpret_cast<const int32_t *>(base + L.piv), b,
                                                       reinterpret_cast<double *>(base + L.y), x);
        PIRO_CHECK_LAUNCH("k_lup_solve_ring");
    } else {
        k_lup_solve_panels<<<1, kPivThreads, 0, st>>>(N, bw, L.W, reinterpret_cast<const double *>(base + L.band),
                                                     reinterpret_cast<const double *>(base + L.lp),
                                                     reinterpret_cast<const int32_t *>(base + L.piv), b,
                                                     reinterpret_cast<double *>(base + L.y), x);
        PIRO_CHECK_LAUNCH("k_lup_solve_panels");
    }
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

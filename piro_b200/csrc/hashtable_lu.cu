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
// shift*I + scale*M into a dense band (row r, column c at
// band[r*(2bw+1) + c - r + bw]; bw = nx*ny for the 7-point grid in natural
// order).  Elimination without pivoting fills in nothing outside the band,
// and in the band no lookup probes a cluster: keys r*N + c of one row are
// contiguous, so at load 0.7 the rows' runs of slots merge and a table lookup
// walks thousands of slots.  The LU runs in place in the band, one launch per
// pivot row over the (bw x bw) block below and right of it; the multipliers
// of a column are stored by the next launch, which no longer reads that
// column.  The substitution is one cooperative launch: per block of 32 rows,
// the worker CTAs form the partial sums of the NEXT block over the solved
// part of its band while CTA 0 finishes the current block (its sums, the
// contribution of the block just solved, and the 32x32 triangle in one warp);
// one grid barrier per block, every wait bounded.
#include "common.cuh"

namespace piro {
namespace {

constexpr int64_t kEmpty = -1, kDeleted = -2;
constexpr int kTri = 32;          // rows per substitution block
constexpr int kSolveThreads = 256;
constexpr int kMaxCta = 1024;     // partial-sum slots per buffer
constexpr long long kSpinLimit = 1ll << 22;  // a stuck barrier ends with an error, not a hang

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

// ---------------------------------------------------------------- banded LU and substitution

__global__ void k_band_diag(int64_t N, int64_t W, int64_t bw, float shift, float *__restrict__ band)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x)
        band[r * W + bw] = shift;
}

// band(r, c) = shift*[r == c] + scale*M(r, c) for every key in the table.
__global__ void k_band_scatter(int64_t N, int64_t bw, int64_t W, const int64_t *__restrict__ keys,
                               const float *__restrict__ vals, int64_t ts, float shift, float scale,
                               float *__restrict__ band, int *err)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ts; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = keys[s];
        if (k < 0) continue;
        const int64_t r = k / N, d = k % N - r;
        if (d > bw || d < -bw) {
            atomicCAS(err, 0, 2);
            continue;
        }
        const float v = __fmul_rn(scale, vals[s]);
        band[r * W + d + bw] = d == 0 ? __fadd_rn(shift, v) : v;
    }
}

// Pivot row ro: a(r, c) -= (a(r, ro)/a(ro, ro)) * a(ro, c) for r, c in
// (ro, ro+span]; block (x, y) takes row ro+1+y, columns kRoundCols*x ..; and
// the multipliers of column ro-1 divided in place (no item of this round
// reads that column).
constexpr int kRoundThreads = 256, kRoundCols = 1024;

__global__ void __launch_bounds__(kRoundThreads) k_band_round(int64_t N, int64_t bw, int64_t W,
                                                              float *__restrict__ band, int64_t ro, int *err)
{
    const float piv = band[ro * W + bw];
    if (piv == 0.0f) {
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && atomicCAS(err, 0, 3) == 0) err[1] = (int)ro;
        return;
    }
    const int64_t span = N - 1 - ro < bw ? N - 1 - ro : bw;
    if (ro > 0 && blockIdx.x == 0) {
        const int64_t pspan = N - ro < bw ? N - ro : bw;
        const float pp = band[(ro - 1) * W + bw];
        for (int64_t t = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; t < pspan; t += (int64_t)gridDim.y * blockDim.x) {
            float *m = band + (ro + t) * W + (bw - 1 - t);  // a(ro+t, ro-1)
            *m = __fdiv_rn(*m, pp);
        }
    }
    const int64_t i = (int64_t)blockIdx.y + 1;
    if (i > span) return;
    const float f = band[(ro + i) * W + bw - i];  // a(ro+i, ro)
    if (f == 0.0f) return;
    const float m = __fdiv_rn(f, piv);
    const float *u = band + ro * W + bw;          // u[j] = a(ro, ro+j)
    float *a = band + (ro + i) * W + (bw - i);    // a[j] = a(ro+i, ro+j)
    const int64_t j0 = (int64_t)blockIdx.x * kRoundCols + 1;
    const int64_t j1 = j0 + kRoundCols <= span + 1 ? j0 + kRoundCols : span + 1;
#pragma unroll 4
    for (int64_t j = j0 + threadIdx.x; j < j1; j += kRoundThreads) a[j] = __fsub_rn(a[j], __fmul_rn(m, u[j]));
}

struct BarState {
    unsigned count, gen;
    int err, pad;
};

__device__ __forceinline__ bool grid_barrier(BarState *st, int *s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &st->gen;
        volatile int *verr = &st->err;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&st->count, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(&st->count, 0u);
            __threadfence();
            atomicAdd(&st->gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == g) {
                if (*verr || ++spins > kSpinLimit) {
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (*verr) ok = 0;
        if (!ok) atomicExch(&st->err, 1);
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct SolveArgs {
    int64_t N, bw, W;
    const float *band;
    const float *b;
    float *x;
    float *part;  // [2][kMaxCta][kTri]
    BarState *st;
};

constexpr int64_t kMinCols = 64;  // columns per worker at least: few partials for CTA 0 to add

// Columns that the workers sum for block kn (all rows of the band solved
// before the block that precedes kn in the sweep) and their split.
struct Split {
    int64_t c0, c1, chunk, nact;
};

__device__ __forceinline__ Split worker_split(const SolveArgs &A, int64_t kn, bool fwd, int workers)
{
    const int64_t Rn = kn * kTri;
    Split sp;
    if (fwd) {
        sp.c0 = Rn - A.bw > 0 ? Rn - A.bw : 0;
        sp.c1 = Rn - kTri;
    } else {
        sp.c0 = Rn + 2 * kTri < A.N ? Rn + 2 * kTri : A.N;
        sp.c1 = Rn + kTri + A.bw < A.N ? Rn + kTri + A.bw : A.N;
    }
    const int64_t len = sp.c1 > sp.c0 ? sp.c1 - sp.c0 : 0;
    const int64_t even = cdiv(len, workers);
    sp.chunk = even > kMinCols ? even : kMinCols;
    sp.nact = cdiv(len, sp.chunk);
    return sp;
}

// Partial sums of block rows [R, R+nb) over columns [c0, c1) (this worker's
// slice), each row restricted to its band.
__device__ __forceinline__ void block_partials(const SolveArgs &A, int64_t R, int nb, int64_t c0, int64_t c1,
                                               bool forward, float *out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < kTri; i += kSolveThreads / 32) {
        float s = 0.0f;
        if (i < nb) {
            const int64_t r = R + i;
            const int64_t lo = forward ? (c0 > r - A.bw ? c0 : r - A.bw) : c0;
            const int64_t hi = forward ? c1 : (c1 < r + A.bw + 1 ? c1 : r + A.bw + 1);
            const float *row = A.band + r * A.W + A.bw - r;
            for (int64_t c = lo + lane; c < hi; c += 32) s += __ldg(row + c) * __ldcg(A.x + c);
        }
        s = warp_sum(s);
        if (lane == 0) out[i] = s;
    }
}

__global__ void __launch_bounds__(kSolveThreads) k_band_solve(SolveArgs A)
{
    __shared__ float s_tri[kTri][kTri + 1];
    __shared__ float s_sum[kTri];
    __shared__ int s_ok;
    const int64_t N = A.N, bw = A.bw, W = A.W;
    const int64_t nblk = cdiv(N, kTri);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int workers = (int)gridDim.x - 1;
    for (int sweep = 0; sweep < 2; ++sweep) {
        const bool fwd = sweep == 0;
        for (int64_t it = 0; it < nblk; ++it) {
            const int64_t k = fwd ? it : nblk - 1 - it;
            const int64_t R = k * kTri;
            const int nb = (int)(N - R < kTri ? N - R : kTri);
            const int buf = (int)(it & 1);
            if (blockIdx.x > 0) {
                // partial sums of the next block over the blocks solved before this one
                const int64_t w = blockIdx.x - 1;
                if (it + 1 < nblk) {
                    const int64_t kn = fwd ? k + 1 : k - 1, Rn = kn * kTri;
                    const Split sp = worker_split(A, kn, fwd, workers);
                    if (w < sp.nact) {
                        const int64_t a0 = sp.c0 + w * sp.chunk, a1 = a0 + sp.chunk < sp.c1 ? a0 + sp.chunk : sp.c1;
                        block_partials(A, Rn, (int)(N - Rn < kTri ? N - Rn : kTri), a0, a1, fwd,
                                       A.part + ((size_t)(buf ^ 1) * kMaxCta + blockIdx.x) * kTri);
                    }
                }
            } else {
                // block k: the workers' sums, the block solved last, the triangle
                const bool has_prev = it > 0;
                const int64_t nact = has_prev ? worker_split(A, k, fwd, workers).nact : 0;
                const int64_t Rp = (fwd ? k - 1 : k + 1) * kTri;
                float acc[kTri / (kSolveThreads / 32)];
#pragma unroll
                for (int q = 0; q < kTri / (kSolveThreads / 32); ++q) {
                    const int i = warp + q * (kSolveThreads / 32);
                    float s = 0.0f;
                    if (i < nb && has_prev) {
                        const float *pp = A.part + (size_t)buf * kMaxCta * kTri + i;
                        if (lane < nact) s += __ldcg(pp + (size_t)(1 + lane) * kTri);
                        for (int64_t g = 33 + lane; g <= nact; g += 32) s += __ldcg(pp + (size_t)g * kTri);
                        const int64_t r = R + i, c = Rp + lane;
                        const bool in = fwd ? (c >= r - bw) : (c < N && c <= r + bw);
                        if (in) s += __ldg(A.band + r * W + (c - r + bw)) * __ldcg(A.x + c);
                    }
                    acc[q] = s;
                }
#pragma unroll
                for (int q = 0; q < kTri / (kSolveThreads / 32); ++q) {
                    const float s = warp_sum(acc[q]);
                    if (lane == 0) s_sum[warp + q * (kSolveThreads / 32)] = s;
                }
                for (int t = threadIdx.x; t < kTri * kTri; t += kSolveThreads) {
                    const int i = t / kTri, j = t % kTri;
                    const bool in = i < nb && j < nb && (fwd ? (j < i && i - j <= bw) : (j >= i && j - i <= bw));
                    s_tri[i][j] = in ? __ldg(A.band + (R + i) * W + (j - i + bw)) : 0.0f;
                }
                __syncthreads();
                if (warp == 0) {
                    float v = lane < nb ? (fwd ? __ldg(A.b + R + lane) : __ldcg(A.x + R + lane)) - s_sum[lane] : 0.0f;
                    if (fwd) {
                        for (int j = 0; j < nb; ++j) {
                            const float xj = __shfl_sync(0xffffffffu, v, j);
                            if (lane > j) v -= s_tri[lane][j] * xj;
                        }
                    } else {
                        for (int j = nb - 1; j >= 0; --j) {
                            if (lane == j) v = v / s_tri[j][j];
                            const float xj = __shfl_sync(0xffffffffu, v, j);
                            if (lane < j) v -= s_tri[lane][j] * xj;
                        }
                    }
                    if (lane < nb) __stcg(A.x + R + lane, v);
                }
            }
            if (!grid_barrier(A.st, &s_ok)) return;
        }
    }
}

int band_layout(int64_t N, int64_t bw, int64_t *W, size_t *band_floats)
{
    if (N < 1 || bw < 1) return PIRO_ERR_ARG;
    if (bw > N - 1) bw = N - 1 > 0 ? N - 1 : 1;
    *W = 2 * bw + 1;
    *band_floats = (size_t)N * (size_t)(*W);
    return PIRO_OK;
}

constexpr size_t kScratchBytes = sizeof(float) * 2 * kMaxCta * kTri + 256;  // partial sums, barrier state

size_t scratch_offset(size_t band_floats) { return (sizeof(float) * band_floats + 255) / 256 * 256; }

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
    int64_t W;
    size_t nf;
    PIRO_ARG(bytes && band_layout(N, bw, &W, &nf) == PIRO_OK, "piro_ht_lu_band_bytes: bad arguments");
    *bytes = scratch_offset(nf) + kScratchBytes;
    return PIRO_OK;
}

extern "C" int piro_ht_lu_factor(int64_t N, int64_t bw, const int64_t *keys, const float *vals, int64_t ts,
                                 float shift, float scale, void *band, size_t band_bytes, piro_stream_t stream)
{
    int64_t W;
    size_t nf;
    PIRO_ARG(keys && vals && ts > 0 && band && band_layout(N, bw, &W, &nf) == PIRO_OK && N < ((int64_t)1 << 31),
             "piro_ht_lu_factor: bad arguments");
    PIRO_ARG(band_bytes >= scratch_offset(nf) + kScratchBytes, "piro_ht_lu_factor: band buffer too small");
    PIRO_ARG((W - 1) / 2 <= 65535, "piro_ht_lu_factor: bandwidth above 65535");
    bw = (W - 1) / 2;
    cudaStream_t st = as_stream(stream);
    float *AB = static_cast<float *>(band);
    int *err = reinterpret_cast<int *>(static_cast<char *>(band) + scratch_offset(nf));
    PIRO_CUDA(cudaMemsetAsync(AB, 0, sizeof(float) * nf, st));
    PIRO_CUDA(cudaMemsetAsync(err, 0, 2 * sizeof(int), st));
    k_band_diag<<<grid_for(N, 256, 8), 256, 0, st>>>(N, W, bw, shift, AB);
    k_band_scatter<<<grid_for(ts, 256, 8), 256, 0, st>>>(N, bw, W, keys, vals, ts, shift, scale, AB, err);
    PIRO_CHECK_LAUNCH("k_band_scatter");
    int herr[2] = {0, 0};
    PIRO_CUDA(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (herr[0] == 2) {
        set_error("piro_ht_lu_factor: the table holds an entry outside the bandwidth %lld", (long long)bw);
        return PIRO_ERR_ARG;
    }
    for (int64_t ro = 0; ro < N; ++ro) {
        const int64_t span = N - 1 - ro < bw ? N - 1 - ro : bw;
        const dim3 grid((unsigned)(span > 0 ? cdiv(span, kRoundCols) : 1), (unsigned)(span > 0 ? span : 1));
        k_band_round<<<grid, kRoundThreads, 0, st>>>(N, bw, W, AB, ro, err);
    }
    PIRO_CHECK_LAUNCH("k_band_round");
    PIRO_CUDA(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (herr[0] == 3) {
        set_error("piro_ht_lu_factor: zero pivot at row %d (elimination without pivoting)", herr[1]);
        return PIRO_ERR_ZERO_PIVOT;
    }
    return PIRO_OK;
}

extern "C" int piro_ht_lu_solve(int64_t N, int64_t bw, void *band, size_t band_bytes, const float *b, float *x,
                                piro_stream_t stream)
{
    int64_t W;
    size_t nf;
    PIRO_ARG(band && b && x && b != x && band_layout(N, bw, &W, &nf) == PIRO_OK, "piro_ht_lu_solve: bad arguments");
    PIRO_ARG(band_bytes >= scratch_offset(nf) + kScratchBytes, "piro_ht_lu_solve: band buffer too small");
    cudaStream_t st = as_stream(stream);
    static int grid[kMaxDevices] = {0};
    static DeviceOnce once;
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    const int rc = device_once(once, dev, [dev]() -> int {
        int per_sm = 0;
        PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_band_solve, kSolveThreads, 0));
        const int g = sm_count();  // at most one CTA per SM
        if (per_sm < 1) {
            set_error("piro_ht_lu_solve: the solve kernel cannot be resident");
            return PIRO_ERR_CUDA;
        }
        grid[dev] = g < 2 ? 2 : (g > kMaxCta ? kMaxCta : g);
        return PIRO_OK;
    });
    if (rc != PIRO_OK) return rc;
    char *scratch = static_cast<char *>(band) + scratch_offset(nf);
    SolveArgs A;
    A.N = N;
    A.bw = (W - 1) / 2;
    A.W = W;
    A.band = static_cast<const float *>(band);
    A.b = b;
    A.x = x;
    A.part = reinterpret_cast<float *>(scratch + 256);
    A.st = reinterpret_cast<BarState *>(scratch + 64);
    PIRO_CUDA(cudaMemsetAsync(A.st, 0, sizeof(BarState), st));
    void *args[] = {&A};
    // CTA 0 and enough workers for kMinCols columns each
    int64_t g = 1 + cdiv(A.bw, kMinCols);
    g = g < 2 ? 2 : (g > grid[dev] ? grid[dev] : g);
    PIRO_CUDA(cudaLaunchCooperativeKernel((const void *)k_band_solve, dim3((unsigned)g), dim3(kSolveThreads), args, 0, st));
    BarState h;
    PIRO_CUDA(cudaMemcpyAsync(&h, A.st, sizeof(BarState), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (h.err) {
        set_error("piro_ht_lu_solve: grid barrier timed out");
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

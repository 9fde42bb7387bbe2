// hashtable.cu -- parallel build of PIRO's open-addressing sparse-matrix table
// with slots identical to the reference's sequential insertion.
//
// The reference inserts every nonzero in row-major order with linear probing
// (methods::sethash, src/methods.cpp:74-118, driven by
// src/operatorlaplacian.cpp:190-203): key = row*N + col, home slot key % TS,
// first free slot from the home; a repeated key keeps its slot and takes the
// later value.  That layout is first-come-first-served by insertion time t
// (the nonzero's position in the CSR arrays).
//
// A first-come-first-served linear-probing table is the unique table in which
// every key's probe path from its home to its slot passes only keys inserted
// earlier.  Threads therefore insert concurrently with time priority: a probe
// that meets a later-inserted key swaps itself in with atomicCAS and carries
// the evicted key onward (ordered hashing, Amble & Knuth 1974, with insertion
// time as the order).  The table converges to that unique layout whatever the
// interleaving.  During the build each slot holds the insertion time t in the
// int64 key array itself; a final pass turns t into (key, value).
#include "common.cuh"

namespace piro {
namespace {

__global__ void k_ht_clear(int64_t ts, int64_t *__restrict__ slots)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ts; s += (int64_t)gridDim.x * blockDim.x)
        slots[s] = -1;
}

// One thread per row; each first occurrence of a column in the row is inserted
// with priority t (its CSR position).  probe_cap bounds the work of a thread.
__global__ void k_ht_insert(int64_t N, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                            int64_t ts, unsigned long long *__restrict__ slots, int64_t probe_cap,
                            int *__restrict__ err)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t j0 = rowptr[r], j1 = rowptr[r + 1];
        for (int32_t j = j0; j < j1; ++j) {
            const int32_t c = col[j];
            bool dup = false;
            for (int32_t q = j0; q < j; ++q)
                if (col[q] == c) { dup = true; break; }
            if (dup) continue;
            unsigned long long cur = (unsigned long long)j;
            int64_t key = r * N + c;
            int64_t h = key % ts;
            int64_t probes = 0;
            while (true) {
                if (++probes > probe_cap) { atomicExch(err, 1); return; }
                const unsigned long long old = *((volatile unsigned long long *)slots + h);
                if (old == ~0ull) {
                    if (atomicCAS(slots + h, ~0ull, cur) == ~0ull) break;
                    continue;  // lost the race: look at the slot again
                }
                if (old > cur) {
                    // a later insertion holds the slot: take it, carry the evictee on
                    if (atomicCAS(slots + h, old, cur) == old) {
                        cur = old;
                        h = h + 1 == ts ? 0 : h + 1;
                    }
                    continue;
                }
                h = h + 1 == ts ? 0 : h + 1;
            }
        }
    }
}

// Row containing nonzero t: largest r with rowptr[r] <= t.
__device__ __forceinline__ int64_t row_of(int64_t t, const int32_t *__restrict__ rowptr, int64_t N)
{
    int64_t lo = 0, hi = N;  // rowptr[lo] <= t < rowptr[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (rowptr[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_ht_finalize(int64_t N, const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                              const float *__restrict__ val, int64_t ts, int64_t *__restrict__ keys,
                              float *__restrict__ vals)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ts; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = keys[s];
        if (t < 0) {
            vals[s] = 0.0f;
            continue;
        }
        const int64_t r = row_of(t, rowptr, N);
        const int32_t c = col[t];
        float v = val[t];
        for (int32_t j = (int32_t)t + 1; j < rowptr[r + 1]; ++j)
            if (col[j] == c) v = val[j];  // sethash overwrites on a repeated key
        keys[s] = r * N + c;
        vals[s] = v;
    }
}

bool is_prime(int64_t n)
{
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (int64_t f = 3; f * f <= n; f += 2)
        if (n % f == 0) return false;
    return true;
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_ht_table_size(int64_t nnz, int64_t N, int policy, float a, float b, float c, float lf, int64_t *ts)
{
    PIRO_ARG(ts && nnz >= 0 && N > 0 && lf > 0.0f, "piro_ht_table_size: bad arguments");
    if (policy == 0) {
        // src/operatorlaplacian.cpp:184-185: float load = a*pow(N, b) + c in
        // double (pow of an int and a float promotes), stored as float; then
        // (int)(sparsecount / (load * lf)) in float.
        const float load = (float)((double)a * pow((double)(int)N, (double)b) + (double)c);
        const float q = (float)(int)nnz / (load * lf);
        const int64_t t = (int64_t)(int)q;
        if (t <= 0 || !(q < 2147483647.0f)) {
            piro::set_error("piro_ht_table_size: reference formula gives %lld slots for N=%lld", (long long)t,
                            (long long)N);
            return PIRO_ERR_TABLE_SIZE;
        }
        *ts = t;
        return PIRO_OK;
    }
    if (policy == 1) {
        int64_t t = (int64_t)ceil((double)nnz / (double)lf);
        if (t < 2) t = 2;
        while (!is_prime(t)) ++t;
        *ts = t;
        return PIRO_OK;
    }
    piro::set_error("piro_ht_table_size: policy %d not in {0 reference, 1 prime}", policy);
    return PIRO_ERR_ARG;
}

extern "C" int piro_ht_build_workspace(int64_t ts, size_t *bytes)
{
    PIRO_ARG(bytes && ts > 0, "piro_ht_build_workspace: bad arguments");
    *bytes = 256;  // the table-full flag; slots are built in place in keys[]
    return PIRO_OK;
}

extern "C" int piro_ht_build(int64_t N, const int32_t *rowptr, const int32_t *col, const float *val, int64_t nnz,
                             int64_t ts, int64_t *keys, float *vals, void *work, size_t work_bytes, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rowptr && col && val && keys && vals && ts > 0 && nnz >= 0, "piro_ht_build: bad arguments");
    PIRO_ARG(work && work_bytes >= sizeof(int), "piro_ht_build: workspace too small");
    PIRO_ARG(N <= INT64_MAX / N, "piro_ht_build: row*N+col overflows int64");
    cudaStream_t s = as_stream(stream);
    int *err = static_cast<int *>(work);
    PIRO_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    k_ht_clear<<<grid_for(ts, 256, 8), 256, 0, s>>>(ts, keys);
    PIRO_CHECK_LAUNCH("k_ht_clear");
    // every carried key moves forward at most ts slots between evictions and
    // is evicted at most once per earlier key; cap generously, then report full
    const int64_t cap = 4 * ts + 1024;
    k_ht_insert<<<grid_for(N, 128, 8), 128, 0, s>>>(N, rowptr, col, ts, reinterpret_cast<unsigned long long *>(keys),
                                                    cap, err);
    PIRO_CHECK_LAUNCH("k_ht_insert");
    int h_err = 0;
    PIRO_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    PIRO_CUDA(cudaStreamSynchronize(s));
    if (h_err) {
        piro::set_error("piro_ht_build: table of %lld slots is full (nnz %lld)", (long long)ts, (long long)nnz);
        return PIRO_ERR_TABLE_FULL;
    }
    k_ht_finalize<<<grid_for(ts, 256, 8), 256, 0, s>>>(N, rowptr, col, val, ts, keys, vals);
    PIRO_CHECK_LAUNCH("k_ht_finalize");
    return PIRO_OK;
}

// spmv.cu -- time-step kernels: CSR SpMV with the forward-Euler update fused
// in its epilogue, the backward-Euler residual form, COO SpMV by warp-segmented
// reduction, HT SpMV by row lookups, the matrix-free 7-point stencil, setBC and
// the elementwise kernels.
//
// CSR layout in HBM: rowptr int32[N+1], col int32[nnz], val float[nnz].  The
// CSR kernels are HBM-bound (8 bytes per nonzero + 12 per row) and share the
// row loop of csr_tile.cuh: one row per thread in storage order -- the
// reference's summation order -- so results are bit-exact with SpMVCSR.cl.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "csr_tile.cuh"

#include <algorithm>

namespace piro {
int scan_rowptr_inplace(int64_t N, int32_t *rowptr, void *work, size_t work_bytes, cudaStream_t s);
size_t scan_workspace_bytes(int64_t N);
}  // namespace piro

namespace piro {
namespace {

// mode 0: SpMVCSR (out = u + sum), mode 1: SpMVCSR_I1 (out = u - sum).
template <int kMode>
// Matrix row `row` is grid row row0 + row (interior test) and reads/writes
// u[ubase + row] / out[ubase + row]; columns index u directly.  (The whole
// grid: row0 = ubase = 0; a z-slab with one halo plane below: row0 = first
// owned row, ubase = nx*ny.)
struct FeRow {
    GridDiv g;
    float dt;
    const float *__restrict__ u;
    float *__restrict__ out;
    int64_t row0, ubase;
    const float *__restrict__ bc;  // kMode 2: the saved face values (may be NULL)
    float result;
    // SpMVCSR.cl's `result += deltat * A[k] * B[col]`, left to right
    __device__ __forceinline__ float term(int32_t c, float v) const { return mul_rn(mul_rn(dt, v), __ldg(u + c)); }
    static __device__ __forceinline__ float accum(float s, float t) { return add_rn(s, t); }
    __device__ __forceinline__ void finish(int64_t row, float s)
    {
        result = s;
        end(row);
    }
    __device__ __forceinline__ void end(int64_t row)
    {
        const int64_t k = ubase + row;
        if (kMode == 2) {
            // the whole next field: interior rows the step, face cells (one
            // coordinate on the boundary: exactly bc::initbc's face lists) their
            // saved value, edges and corners 0 -- zero-filled partD, SpMVCSR,
            // then setBC, in one pass
            int x, y, z;
            g.coords((uint32_t)(row0 + row), x, y, z);
            const int ex = (x == 0 || x == g.nx - 1) + (y == 0 || y == g.ny - 1) + (z == 0 || z == g.nz - 1);
            out[k] = ex == 0 ? add_rn(result, u[k]) : (ex == 1 && bc) ? bc[k] : 0.0f;
        } else if (g.interior(row0 + row)) {
            out[k] = kMode == 0 ? add_rn(result, u[k]) : sub_rn(u[k], result);
        }
    }
};

template <int kMode>
__global__ void __launch_bounds__(kRowThreads) k_csr_step(GridDiv g, int64_t N, const int32_t *__restrict__ rowptr,
                                                          const int32_t *__restrict__ col,
                                                          const float *__restrict__ val, float dt,
                                                          const float *__restrict__ u, float *__restrict__ out,
                                                          int64_t row0, int64_t ubase)
{
    FeRow<kMode> op{g, dt, u, out, row0, ubase, nullptr, 0.0f};
    csr_for_rows_adaptive(N, rowptr, col, val, op);
}

__global__ void __launch_bounds__(kRowThreads) k_csr_step_bc(GridDiv g, int64_t N, const int32_t *__restrict__ rowptr,
                                                             const int32_t *__restrict__ col,
                                                             const float *__restrict__ val, float dt,
                                                             const float *__restrict__ u, const float *__restrict__ bc,
                                                             float *__restrict__ out)
{
    FeRow<2> op{g, dt, u, out, 0, 0, bc, 0.0f};
    csr_for_rows_adaptive(N, rowptr, col, val, op);
}

// COO with a row index: rowstart[r] = the first entry of row r in the
// row-sorted entry arrays (rowstart[N] = nnz), built once per operator; then
// the step is the CSR row loop over cols/vals (each row's entries summed in
// storage order), out = dt*sum or u + dt*sum on every row (SpMVCOO then
// addVectors).  err: rows not sorted, or out of range.
__global__ void k_coo_rowstart(int64_t N, int64_t nnz, const int32_t *__restrict__ rows, int32_t *__restrict__ rowstart,
                               int *err)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r1 = rows[k], r0 = k > 0 ? rows[k - 1] : -1;
        if (r1 < r0 || r1 < 0 || r1 >= N) {
            atomicExch(err, 1);
            continue;
        }
        for (int64_t r = r0 + 1; r <= r1; ++r) rowstart[r] = (int32_t)k;
        if (k == nnz - 1)
            for (int64_t r = r1 + 1; r <= N; ++r) rowstart[r] = (int32_t)nnz;
    }
}

struct CooRow {
    float dt;
    const float *__restrict__ u;
    float *__restrict__ out;
    int fe;
    float acc;
    // SpMVCOO.cl's `result += values[k] * B[cols[k]]` over the row's entries
    __device__ __forceinline__ float term(int32_t c, float v) const { return __fmul_rn(v, __ldg(u + c)); }
    static __device__ __forceinline__ float accum(float s, float t) { return __fadd_rn(s, t); }
    __device__ __forceinline__ void finish(int64_t row, float s)
    {
        const float c = __fmul_rn(dt, s);
        out[row] = fe ? __fadd_rn(__ldg(u + row), c) : c;
    }
};

__global__ void __launch_bounds__(kRowThreads) k_coo_rows(int64_t N, const int32_t *__restrict__ rowstart,
                                                          const int32_t *__restrict__ cols,
                                                          const float *__restrict__ vals, float dt, int fe,
                                                          const float *__restrict__ u, float *__restrict__ out)
{
    CooRow op{dt, u, out, fe, 0.0f};
    csr_for_rows_adaptive(N, rowstart, cols, vals, op);
}

// COO: each warp takes 32 consecutive entries per pass; a segmented inclusive
// scan over equal row ids gives each row's partial sum in the segment's last
// lane.  Rows wholly inside the warp's span are stored; rows cut by the span
// edges are atomically added (at most two contributions for rows of <= 32
// entries, so the result does not depend on their order).  acc must be zero.
// The segments are only whole rows when the row ids ascend, and SpMVCOO.cl
// (which scans every entry for each row) matches no row outside [0, N): an
// entry whose row or column lies outside [0, N) adds nothing (bit 1 of *err),
// and a row id below its predecessor's sets bit 2 of *err, so the host turns
// both into an error instead of a wrong sum or an out-of-range access.
__global__ void k_coo_segsum(int64_t N, int64_t nnz, const int32_t *__restrict__ rows,
                             const int32_t *__restrict__ cols, const float *__restrict__ vals,
                             const float *__restrict__ u, float *__restrict__ acc, int *__restrict__ err)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int bad = 0;
    for (int64_t base = warp * 32; base < nnz; base += nwarps * 32) {
        const int64_t k = base + lane;
        const bool in_span = k < nnz;
        const int rraw = in_span ? __ldcs(rows + k) : INT32_MAX;
        const int craw = in_span ? __ldcs(cols + k) : 0;
        const bool valid = in_span && rraw >= 0 && rraw < N && craw >= 0 && craw < N;
        if (in_span && !valid) bad |= 1;
        // ascending row ids: compare with the previous entry (lane 0 reads it)
        int rprev = __shfl_up_sync(0xffffffffu, rraw, 1);
        if (lane == 0) rprev = k > 0 && in_span ? __ldg(rows + (k - 1)) : INT32_MIN;
        if (in_span && rraw < rprev) bad |= 2;
        int r = valid ? rraw : -1;
        float p = valid ? __fmul_rn(__ldcs(vals + k), __ldg(u + craw)) : 0.0f;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float q = __shfl_up_sync(0xffffffffu, p, o);
            const int rq = __shfl_up_sync(0xffffffffu, r, o);
            if (lane >= o && rq == r) p = __fadd_rn(q, p);
        }
        const int rnext = __shfl_down_sync(0xffffffffu, r, 1);
        const bool seg_end = valid && (lane == 31 || rnext != r);
        if (seg_end) {
            // segment start lane: first lane of this row within the warp
            const bool cut_left = (k - lane > 0) && __ldg(rows + (base - 1)) == r &&
                                  // the row reaches lane 0 of this span
                                  __ldg(rows + base) == r;
            const bool cut_right = (lane == 31) && (k + 1 < nnz) && __ldg(rows + k + 1) == r;
            if (cut_left || cut_right) atomicAdd(acc + r, p);
            else acc[r] = p;
        }
    }
    if (bad) atomicOr(err, bad);
}

// The same sum with 8 consecutive entries per lane (a warp covers a 256-entry
// span per pass), and the step finished in place: 16-byte loads of rows,
// cols and vals, runs of equal row ids summed sequentially in the lane, and
// one segmented scan per warp over the lanes' last runs instead of one per
// entry.  With ascending row ids a row's entries are contiguous, so a run
// that starts and ends inside a lane is the whole row; a lane's last run
// continues into the next lane when that lane starts with the same row, and
// the scan carries its sum there.  A row complete inside the span is
// written at once, out = dt*sum or u + dt*sum (SpMVCOO's C[row] =
// deltat*result, then addVectors); rows without entries get dt*0 (+ u).  A
// row that crosses a span boundary leaves its part in this span as
// part_first[span] (the row began in an earlier span) or part_last[span]
// (it begins here), and k_coo_span_fixup adds the parts in span order: no
// atomics, so the sums do not depend on scheduling.  Same input checks as
// k_coo_segsum.  Requires 16-byte aligned arrays.
constexpr int kCooPer = 8;
constexpr int kCooSpan = 32 * kCooPer;

template <bool kFe>
__device__ __forceinline__ float coo_finish(float sum, float dt, const float *__restrict__ u, int64_t r)
{
    const float c = __fmul_rn(dt, sum);
    return kFe ? __fadd_rn(__ldg(u + r), c) : c;
}

// rows [r0, r1) hold no entry (clamped to [0, N)); callers test for a gap first
template <bool kFe>
__device__ __forceinline__ void coo_empty_rows(int64_t r0, int64_t r1, int64_t N, float dt, const float *__restrict__ u,
                                            float *__restrict__ out)
{
    r0 = r0 < 0 ? 0 : r0;
    r1 = r1 > N ? N : r1;
    for (int64_t r = r0; r < r1; ++r) out[r] = coo_finish<kFe>(0.0f, dt, u, r);
}

template <bool kFe>
__global__ void __launch_bounds__(256, 5) k_coo_segsum8(int64_t N, int64_t nnz, const int32_t *__restrict__ rows,
                                                     const int32_t *__restrict__ cols,
                                                     const float *__restrict__ vals, const float *__restrict__ u,
                                                     float dt, float *__restrict__ out,
                                                     float *__restrict__ part_first, float *__restrict__ part_last,
                                                     int32_t *__restrict__ span_row, int32_t *__restrict__ span_whole,
                                                     int *__restrict__ err)
{
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    constexpr int kNone = INT32_MAX;  // row id of entries past the end
    int bad = 0;
    for (int64_t base = warp * kCooSpan; base < nnz; base += nwarps * kCooSpan) {
        const int64_t k0 = base + (int64_t)lane * kCooPer;
        const int64_t sidx = base / kCooSpan;
        int r[kCooPer], c[kCooPer];
        float v[kCooPer];
        if (k0 + kCooPer <= nnz) {
            const int4 *R4 = reinterpret_cast<const int4 *>(rows + k0), *C4 = reinterpret_cast<const int4 *>(cols + k0);
            const float4 *V4 = reinterpret_cast<const float4 *>(vals + k0);
#pragma unroll
            for (int h = 0; h < kCooPer / 4; ++h) {
                const int4 ra = __ldcs(R4 + h), ca = __ldcs(C4 + h);
                const float4 va = __ldcs(V4 + h);
                r[4 * h] = ra.x; r[4 * h + 1] = ra.y; r[4 * h + 2] = ra.z; r[4 * h + 3] = ra.w;
                c[4 * h] = ca.x; c[4 * h + 1] = ca.y; c[4 * h + 2] = ca.z; c[4 * h + 3] = ca.w;
                v[4 * h] = va.x; v[4 * h + 1] = va.y; v[4 * h + 2] = va.z; v[4 * h + 3] = va.w;
            }
        } else {
#pragma unroll
            for (int t = 0; t < kCooPer; ++t) {
                const int64_t k = k0 + t;
                const bool in = k < nnz;
                r[t] = in ? __ldcs(rows + k) : kNone;
                c[t] = in ? __ldcs(cols + k) : 0;
                v[t] = in ? __ldcs(vals + k) : 0.0f;
            }
        }
        // input checks: ids in [0, N), row ids ascending (within the lane and
        // from the entry before it); an entry out of range adds nothing.  A
        // lane with all 8 entries inside the array (every lane but the last
        // one of the array) skips the per-entry end test.
        const bool full = k0 + kCooPer <= nnz;
        int prev = __shfl_up_sync(0xffffffffu, r[kCooPer - 1], 1);
        if (lane == 0) prev = base > 0 ? __ldg(rows + (base - 1)) : INT32_MIN;
        const uint32_t un = (uint32_t)N;
#pragma unroll
        for (int t = 0; t < kCooPer; ++t) {
            if (!full && k0 + t >= nnz) continue;
            if (r[t] < prev) bad |= 2;
            prev = r[t];
            if ((uint32_t)r[t] >= un || (uint32_t)c[t] >= un) {  // negative ids wrap above N
                bad |= 1;
                v[t] = 0.0f;
                c[t] = 0;
            }
        }
        // runs of equal row ids: runs strictly inside the lane are whole rows
        const int first = r[0];
        int cur = r[0];
        float s_run = 0.0f, head = 0.0f;
        bool multi = false;
#pragma unroll
        for (int t = 0; t < kCooPer; ++t) {
            const float pv = (full || r[t] != kNone) ? __fmul_rn(v[t], __ldg(u + c[t])) : 0.0f;
            if (r[t] != cur) {
                if (!multi) head = s_run;                                               // the lane's first run
                else if (cur >= 0 && cur < N) out[cur] = coo_finish<kFe>(s_run, dt, u, cur);  // a whole row
                if (r[t] != kNone && r[t] > cur + 1) coo_empty_rows<kFe>((int64_t)cur + 1, r[t], N, dt, u, out);
                multi = true;
                cur = r[t];
                s_run = 0.0f;
            }
            s_run = __fadd_rn(s_run, pv);
        }
        const int last = cur;
        // inclusive segmented scan of the lanes' last runs: a lane that is one
        // run throughout continues its predecessor's run of the same row
        float carry = s_run;
        bool joins = !multi;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float cq = __shfl_up_sync(0xffffffffu, carry, o);
            const int kq = __shfl_up_sync(0xffffffffu, last, o);
            const int jq = __shfl_up_sync(0xffffffffu, (int)joins, o);
            if (lane >= o && joins && kq == last) {
                carry = __fadd_rn(cq, carry);
                joins = jq != 0;
            }
        }
        const float cin = __shfl_up_sync(0xffffffffu, carry, 1);
        const int kin = __shfl_up_sync(0xffffffffu, last, 1);
        const int next_first = __shfl_down_sync(0xffffffffu, first, 1);
        const int64_t span_end = base + kCooSpan < nnz ? base + kCooSpan : nnz;
        const int left_row = base > 0 ? __ldg(rows + (base - 1)) : INT32_MIN;   // row of the entry before the span
        const int right_row = span_end < nnz ? __ldg(rows + span_end) : kNone;  // row of the entry after it
        if (multi && first >= 0 && first < N) {
            // the lane's first run ends here: add what the lanes before carried in
            const float h = (lane > 0 && kin == first) ? __fadd_rn(cin, head) : head;
            if (first == left_row) part_first[sidx] = h;  // the tail of a row begun in an earlier span
            else out[first] = coo_finish<kFe>(h, dt, u, first);
        }
        // the lane's last run ends here unless the next lane starts with it
        const bool ends_here = lane == 31 || k0 + kCooPer >= span_end || next_first != last;
        if (ends_here && last >= 0 && last < N) {
            if (last == left_row) part_first[sidx] = carry;       // begun earlier (its tail, or the whole span)
            else if (last == right_row) part_last[sidx] = carry;  // begins here, goes on in the next span
            else out[last] = coo_finish<kFe>(carry, dt, u, last);
        }
        // rows without entries after this lane's: up to the next lane's first
        // row, or from the span's last entry to the next span's first row (to
        // N after the last entry); before the first entry, in span 0
        const int span_first = __shfl_sync(0xffffffffu, first, 0);
        if (k0 < span_end) {
            if (k0 + kCooPer >= span_end) {  // the lane with the span's last entry
                const int lr = __ldg(rows + (span_end - 1));
                const int64_t a = (int64_t)lr + 1, b = span_end < nnz ? (int64_t)right_row : N;
                if (b > a) coo_empty_rows<kFe>(a, b, N, dt, u, out);
                // for k_coo_span_fixup: the row that begins here and goes on (or -1),
                // and whether one row covers the whole span and goes on
                const bool cont_in = span_first == lr && left_row == lr, cont_out = right_row == lr;
                span_row[sidx] = cont_out && !cont_in && lr >= 0 && lr < N ? lr : -1;
                span_whole[sidx] = cont_in && cont_out ? 1 : 0;
            } else if (next_first > last + 1) {
                coo_empty_rows<kFe>((int64_t)last + 1, next_first, N, dt, u, out);
            }
        }
        if (base == 0 && lane == 0 && r[0] > 0) coo_empty_rows<kFe>(0, r[0], N, dt, u, out);
    }
    if (bad) atomicOr(err, bad);
}

// Rows that cross span boundaries, one thread per span that begins such a
// row: its part here plus the parts of the following spans, in span order,
// while the row goes on; then the finished value.
template <bool kFe>
__global__ void k_coo_span_fixup(int64_t nspan, const float *__restrict__ u, float dt,
                                 const float *__restrict__ part_first, const float *__restrict__ part_last,
                                 const int32_t *__restrict__ span_row, const int32_t *__restrict__ span_whole,
                                 float *__restrict__ out)
{
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nspan; s += (int64_t)gridDim.x * blockDim.x) {
        const int lr = span_row[s];
        if (lr < 0) continue;  // no row begins in this span and goes on
        float total = part_last[s];
        for (int64_t t = s + 1; t < nspan; ++t) {
            total = __fadd_rn(total, part_first[t]);
            if (!span_whole[t]) break;  // the row ends in span t
        }
        out[lr] = coo_finish<kFe>(total, dt, u, lr);
    }
}

// out = dt*acc (SpMVCOO's C[row] = deltat*result) or u + dt*acc.
// acc and out may be the same buffer (element-wise, same index).
__global__ void k_scale_add(int64_t n, float dt, const float *acc, const float *u, float *out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float c = __fmul_rn(dt, acc[i]);
        out[i] = u ? __fadd_rn(u[i], c) : c;
    }
}

// HT lookup with linear probing (SpMVHT.cl:1-20) from slot h on; bounded by
// ts probes.
__device__ __forceinline__ float ht_get_from(int64_t key, int64_t h, const int64_t *__restrict__ keys,
                                             const float *__restrict__ vals, int64_t ts)
{
    for (int64_t a = 0; a < ts; ++a) {
        const int64_t k = __ldg(keys + h);
        if (k == key) return __ldg(vals + h);
        if (k == -1) return 0.0f;
        h = h + 1 == ts ? 0 : h + 1;
    }
    return 0.0f;
}

// Row i of the 7-point matrix (row order[j] of thread j when ordered): the
// candidate columns c = i + off, off in
// {-nx*ny, -nx, -1, 0, 1, nx, nx*ny}, in ascending order; absent keys give 0,
// adding 0*u exactly as the reference's loop over the row does.  The keys
// i*N + c have home slots (i*N + i + off) mod ts: one 64-bit modulo per row,
// then small offsets (|off| < ts, since ts > nnz > N).  The seven first probes
// are issued together, then the seven value loads; only a collision (a first
// probe holding another key) walks on.
template <bool kOrdered>
__global__ void __launch_bounds__(256, 4) k_ht_spmv(GridDiv g, int64_t N, const int64_t *__restrict__ keys,
                          const float *__restrict__ vals, int64_t ts, ModU64 mts, float dt, int fe,
                          const int32_t *__restrict__ order, const float *__restrict__ u, float *__restrict__ out)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t sxy = (int64_t)nx * ny;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < N; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = kOrdered ? (int64_t)__ldg(order + j) : j;
        int x, y, z;
        g.coords((uint32_t)i, x, y, z);
        // the seven directions in ascending column order, each present or not
        const int64_t off[7] = {-sxy, -(int64_t)nx, -1, 0, 1, (int64_t)nx, sxy};
        const bool ok[7] = {z > 0, y > 0, x > 0, true, x < nx - 1, y < ny - 1, z < nz - 1};
        const int64_t kd = i * N + i, base = (int64_t)mts.mod((uint64_t)kd);
        auto home = [&](int t) {  // the first probe of candidate t (recomputed on a collision, not kept)
            int64_t hh = base + off[t];
            hh += hh < 0 ? ts : 0;
            hh -= hh >= ts ? ts : 0;
            return hh;
        };
        int64_t k[7];
        float v[7];
#pragma unroll
        for (int t = 0; t < 7; ++t) {
            if (ok[t]) {
                const int64_t hh = home(t);
                k[t] = __ldg(keys + hh);
                v[t] = __ldg(vals + hh);  // with the key, not after it: one round trip
            }
        }
#pragma unroll
        for (int t = 0; t < 7; ++t) {
            if (ok[t]) {
                const int64_t key = kd + off[t];
                if (k[t] == key) {
                } else if (k[t] == -1) {
                    v[t] = 0.0f;
                } else {
                    const int64_t hh = home(t);
                    v[t] = ht_get_from(key, hh + 1 == ts ? 0 : hh + 1, keys, vals, ts);
                }
            }
        }
        float sum = 0.0f;
#pragma unroll
        for (int t = 0; t < 7; ++t)
            if (ok[t]) sum = __fadd_rn(sum, __fmul_rn(v[t], __ldg(u + i + off[t])));
        const float c = __fmul_rn(dt, sum);
        out[i] = fe ? __fadd_rn(u[i], c) : c;
    }
}

// The same step in two passes, so that neither u nor out is touched in the
// scattered home-slot order.  Pass 1 (rows in home-slot order) streams the
// table through its moving window and writes each row's seven values, absent
// keys as 0, into a 32-byte record stage[8 i .. 8 i + 7] (two full 16-byte
// stores: whole sectors, no read-modify-write of a partly written sector).
// Pass 2 (rows in index order) reads the records and u coalesced and writes
// out coalesced.  The per-row arithmetic is the one above, term for term.
__global__ void __launch_bounds__(256, 4) k_ht_stage(GridDiv g, int64_t N, const int64_t *__restrict__ keys,
                           const float *__restrict__ vals, int64_t ts, ModU64 mts, const int32_t *__restrict__ order,
                           float4 *__restrict__ stage)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t sxy = (int64_t)nx * ny;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int32_t next_i = j < N ? __ldg(order + j) : 0;  // the row of the next iteration, loaded one ahead
    for (; j < N; j += stride) {
        const int64_t i = next_i;
        if (j + stride < N) next_i = __ldg(order + j + stride);
        int x, y, z;
        g.coords((uint32_t)i, x, y, z);
        const int64_t off[7] = {-sxy, -(int64_t)nx, -1, 0, 1, (int64_t)nx, sxy};
        const bool ok[7] = {z > 0, y > 0, x > 0, true, x < nx - 1, y < ny - 1, z < nz - 1};
        const int64_t kd = i * N + i, base = (int64_t)mts.mod((uint64_t)kd);
        auto home = [&](int t) {  // the first probe of candidate t (recomputed on a collision, not kept)
            int64_t hh = base + off[t];
            hh += hh < 0 ? ts : 0;
            hh -= hh >= ts ? ts : 0;
            return hh;
        };
        int64_t k[7];
        float v[8];
        v[7] = 0.0f;
#pragma unroll
        for (int t = 0; t < 7; ++t) {
            v[t] = 0.0f;
            if (ok[t]) {
                const int64_t hh = home(t);
                k[t] = __ldg(keys + hh);
                v[t] = __ldg(vals + hh);  // with the key: one round trip
            }
        }
#pragma unroll
        for (int t = 0; t < 7; ++t) {
            if (ok[t]) {
                const int64_t key = kd + off[t];
                if (k[t] == key) {
                } else if (k[t] == -1) {
                    v[t] = 0.0f;
                } else {
                    const int64_t hh = home(t);
                    v[t] = ht_get_from(key, hh + 1 == ts ? 0 : hh + 1, keys, vals, ts);
                }
            }
        }
        stage[2 * i] = make_float4(v[0], v[1], v[2], v[3]);
        stage[2 * i + 1] = make_float4(v[4], v[5], v[6], v[7]);
    }
}

__global__ void k_ht_stage_apply(GridDiv g, float dt, int fe, const float4 *__restrict__ stage,
                                 const float *__restrict__ u, float *__restrict__ out)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sxy = nx * ny;
    const int N = sxy * nz;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        int x, y, z;
        g.coords((uint32_t)i, x, y, z);
        const float4 lo = __ldcs(stage + 2 * (int64_t)i), hi = __ldcs(stage + 2 * (int64_t)i + 1);
        const float v[7] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z};
        const int off[7] = {-sxy, -nx, -1, 0, 1, nx, sxy};
        const bool ok[7] = {z > 0, y > 0, x > 0, true, x < nx - 1, y < ny - 1, z < nz - 1};
        float sum = 0.0f;
#pragma unroll
        for (int t = 0; t < 7; ++t)
            if (ok[t]) sum = __fadd_rn(sum, __fmul_rn(v[t], __ldg(u + i + off[t])));
        const float c = __fmul_rn(dt, sum);
        out[i] = fe ? __fadd_rn(u[i], c) : c;
    }
}

// Rows by home slot: rows whose keys sit close in the table run close in
// time, so that the table is read as a moving window of about +-nx*ny slots
// (resident in L2) instead of at random.  Counting sort on buckets of
// kOrderBucket slots of the home slot (i*N + i) mod ts; the order inside a
// bucket is whatever the atomics give (each row's result does not depend on
// it).
constexpr int kOrderShift = 7;  // 128-slot buckets

__global__ void k_order_count(int64_t N, int64_t ts, int32_t *__restrict__ cnt)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + 1 + (((i * N + i) % ts) >> kOrderShift), 1);
}

__global__ void k_order_scatter(int64_t N, int64_t ts, int32_t *__restrict__ cursor, int32_t *__restrict__ order)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        order[atomicAdd(cursor + (((i * N + i) % ts) >> kOrderShift), 1)] = (int32_t)i;
}

// Matrix-free 7-point update: one (x, y) column per thread over a run of
// kStZ planes, 32 x 8 columns per block.  u at z-1, z, z+1 rolls through
// registers, so a cell costs six new loads (x and y neighbours from L1/L2,
// z+1, alpha) and HBM sees each u and alpha value about once: 12 bytes per
// cell.  Coordinates come from the block indices (no division).
__device__ __forceinline__ float st_update(float c, float xm, float xp, float ym, float yp, float zm, float zp,
                                           float a, float idx2, float idy2, float idz2, float dt)
{
    const float c2 = __fmul_rn(2.0f, c);
    const float lx = __fmul_rn(__fsub_rn(__fadd_rn(xp, xm), c2), idx2);
    const float ly = __fmul_rn(__fsub_rn(__fadd_rn(yp, ym), c2), idy2);
    const float lz = __fmul_rn(__fsub_rn(__fadd_rn(zp, zm), c2), idz2);
    const float lap = __fadd_rn(__fadd_rn(lx, ly), lz);
    return __fadd_rn(c, __fmul_rn(dt, __fmul_rn(a, lap)));
}

constexpr int kStX = 32, kStY = 8, kStZ = 8;

__global__ void __launch_bounds__(kStX *kStY) k_stencil(int nx, int ny, int nz, float idx2, float idy2, float idz2,
                                                        float dt, const float *__restrict__ alpha,
                                                        const float *__restrict__ u, float *__restrict__ out)
{
    const int x = blockIdx.x * kStX + threadIdx.x, y = blockIdx.y * kStY + threadIdx.y;
    if (x >= nx || y >= ny) return;
    const int z0 = blockIdx.z * kStZ;
    const int z1 = min(z0 + kStZ, nz);
    const int64_t sxy = (int64_t)nx * ny;
    const bool in_xy = x > 0 && x < nx - 1 && y > 0 && y < ny - 1;
    int64_t id = (int64_t)z0 * sxy + (int64_t)y * nx + x;
    float zm = z0 > 0 ? __ldg(u + id - sxy) : 0.0f;
    float c = __ldg(u + id);
    for (int z = z0; z < z1; ++z, id += sxy) {
        const float zp = z + 1 < nz ? __ldg(u + id + sxy) : 0.0f;
        if (in_xy && z > 0 && z < nz - 1) {
            const float a = alpha ? __ldg(alpha + id) : 1.0f;
            __stcs(out + id, st_update(c, __ldg(u + id - 1), __ldg(u + id + 1), __ldg(u + id - nx), __ldg(u + id + nx),
                                       zm, zp, a, idx2, idy2, idz2, dt));
        } else {
            __stcs(out + id, c);
        }
        zm = c;
        c = zp;
    }
}

// The same update on groups of 4 x-adjacent cells taken in memory order, one
// group per thread (nx % 4 == 0: a group never spans two x-lines; 16-byte
// aligned arrays; N < 2^32 for 32-bit coordinates).  Every load is issued at
// once (u, alpha and the y/z neighbours as float4, the two x halo cells as
// scalars); the whole grid sweeps memory in address order, so the z+-1
// planes are still in L2 when read and HBM sees each u and alpha value once.
// Measured on B200 at 256^3: 5.15 TB/s against 3.3 for the z-marching form,
// whose per-plane loads leave too few bytes in flight.
__global__ void __launch_bounds__(256) k_stencil4(int nx, int ny, int nz, float idx2, float idy2, float idz2, float dt,
                                                  const float *__restrict__ alpha, const float *__restrict__ u,
                                                  float *__restrict__ out)
{
    const uint32_t sxy = (uint32_t)nx * (uint32_t)ny, nv = (sxy * (uint32_t)nz) >> 2;
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const uint32_t id = v << 2;
    const uint32_t z = id / sxy, rem = id - z * sxy, y = rem / (uint32_t)nx;
    const int x0 = (int)(rem - y * (uint32_t)nx);
    const float4 c = __ldg(reinterpret_cast<const float4 *>(u) + v);
    float4 r = c;
    if (y > 0 && y < (uint32_t)ny - 1 && z > 0 && z < (uint32_t)nz - 1) {
        const float4 a = alpha ? __ldg(reinterpret_cast<const float4 *>(alpha) + v) : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        const float4 ym = __ldg(reinterpret_cast<const float4 *>(u + id - nx));
        const float4 yp = __ldg(reinterpret_cast<const float4 *>(u + id + nx));
        const float4 zm = __ldg(reinterpret_cast<const float4 *>(u + id - sxy));
        const float4 zp = __ldg(reinterpret_cast<const float4 *>(u + id + sxy));
        const float xl = x0 > 0 ? __ldg(u + id - 1) : 0.0f, xr = x0 + 4 < nx ? __ldg(u + id + 4) : 0.0f;
        const float cs[6] = {xl, c.x, c.y, c.z, c.w, xr};
        const float ymv[4] = {ym.x, ym.y, ym.z, ym.w}, ypv[4] = {yp.x, yp.y, yp.z, yp.w};
        const float zmv[4] = {zm.x, zm.y, zm.z, zm.w}, zpv[4] = {zp.x, zp.y, zp.z, zp.w};
        const float av[4] = {a.x, a.y, a.z, a.w};
        float rv[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int x = x0 + t;
            rv[t] = (x > 0 && x < nx - 1)
                        ? st_update(cs[t + 1], cs[t], cs[t + 2], ymv[t], ypv[t], zmv[t], zpv[t], av[t], idx2, idy2, idz2, dt)
                        : cs[t + 1];
        }
        r = make_float4(rv[0], rv[1], rv[2], rv[3]);
    }
    __stcs(reinterpret_cast<float4 *>(out) + v, r);
}

__global__ void k_set_bc(int64_t q, const uint32_t *__restrict__ idx, const float *__restrict__ src,
                         float *__restrict__ dst)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < q; t += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t i = idx[t];
        dst[i] = src[i];
    }
}

__global__ void k_vec_op(int op, int64_t n, const float *__restrict__ b, const float *__restrict__ c,
                         float *__restrict__ a)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = b[i], y = c[i];
        a[i] = op == 0 ? __fadd_rn(x, y) : op == 1 ? __fsub_rn(x, y) : op == 2 ? __fmul_rn(x, y) : __fdiv_rn(x, y);
    }
}

__global__ void k_vec_op_scalar(int op, int64_t n, float s, const float *__restrict__ c, float *__restrict__ a)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float y = c[i];
        a[i] = op == 0 ? __fadd_rn(s, y) : op == 1 ? __fsub_rn(y, s) : op == 2 ? __fmul_rn(s, y) : __fdiv_rn(y, s);
    }
}

__global__ void k_vec_urf(int64_t n, float *__restrict__ a, float *__restrict__ c, float urf)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float t = a[i];
        const float an = __fadd_rn(t, __fmul_rn(c[i], urf));
        a[i] = an;
        c[i] = __fsub_rn(an, t);
    }
}

bool grid_ok(int nx, int ny, int nz)
{
    return nx >= 3 && ny >= 3 && nz >= 3 && (int64_t)nx * ny * nz < ((int64_t)1 << 31);
}

template <int kMode>
int launch_csr_step(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val, float dt,
                    const float *u, float *out, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz), "csr step: grid sizes must be >= 3");
    PIRO_ARG(rowptr && col && val && u && out, "csr step: null pointer");
    PIRO_ARG(u != out, "csr step: u and out must differ (the reference writes a fresh buffer)");
    const int64_t N = (int64_t)nx * ny * nz;
    k_csr_step<kMode><<<csr_rows_grid(N), kRowThreads, 0, as_stream(stream)>>>(GridDiv(nx, ny, nz), N, rowptr, col,
                                                                              val, dt, u, out, 0, 0);
    PIRO_CHECK_LAUNCH("k_csr_step");
    return PIRO_OK;
}


// The matrix-free update with TMA tile staging, for 16 <= nx <= 256 with
// nx % 4 == 0 and 2048 % nx == 0.  A CTA owns TY = 2048 / nx full x-rows and
// marches a run of z planes.  One producer warp (its lane 0) issues, per
// plane, one 3-D TMA load of u's rows y0-1 .. y0+TY (the y halo; coordinates
// outside the grid arrive as zeros and feed only boundary cells, which copy u)
// and one of alpha's TY rows, into a ring of kTmaStages stages: "full"
// mbarriers complete on the copies' bytes, "empty" mbarriers on the arrival
// of all 16 consumer warps, so a stage is refilled as soon as the last warp
// has read it and no warp ever waits for another at a CTA barrier.  Consumer
// warps read planes z-1, z, z+1 from shared memory, so u crosses HBM about
// once (plus two halo planes per run; the y halo rows are L2 hits, since the
// CTAs of neighbouring row blocks run together).  Each consumer thread
// updates 4 x-adjacent cells of one row (x neighbours by warp shuffle) and
// stores them as one float4.  The TMA x coordinate is always 0, so every copy
// starts on a 16-byte boundary.  Every wait is bounded (a.spin polls,
// piro_set_wait_limit): a timed-out wait sets *err and its warp leaves.
// Before the producer leaves -- at the end of the run, or on a timeout -- it
// waits for each stage's latest copy with its own full bound (kTmaSpin), so no
// copy lands after the CTA has left, however early the consumers gave up.
constexpr int kTmaThreads = 512, kTmaStages = 6, kTmaWarps = kTmaThreads / 32;
constexpr long long kTmaSpin = 1ll << 22;

struct StencilTma {
    int nx, ny, nz, ty, zchunk, has_alpha;
    float idx2, idy2, idz2, dt;
    float *out;
    int *err;
    long long spin;  // polls per stage wait
};

__device__ __forceinline__ uint32_t st_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool st_bar_wait(uint32_t bar, uint32_t parity, long long limit)
{
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kTmaThreads + 32, 2) k_stencil_tma(const __grid_constant__ CUtensorMap umap,
                                                                      const __grid_constant__ CUtensorMap amap,
                                                                      StencilTma a)
{
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t full[kTmaStages], empty[kTmaStages];
    const int nx = a.nx, TY = a.ty, tid = threadIdx.x;
    const int y0 = blockIdx.x * TY;
    const int z0 = blockIdx.y * a.zchunk, z1 = z0 + a.zchunk < a.nz ? z0 + a.zchunk : a.nz;
    const int ufl = (TY + 2) * nx, sfl = ufl + (a.has_alpha ? TY * nx : 0);
    const int nload = z1 - z0 + 2;  // planes z0-1 .. z1; load k lives in stage k % kTmaStages
    if (tid == 0) {
        for (int s = 0; s < kTmaStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(st_smem(&full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(st_smem(&empty[s])), "r"(kTmaWarps)
                         : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid >= kTmaThreads) {  // producer warp
        if (tid != kTmaThreads) return;
        int L = 0;
        bool ok = true;
        for (; L < nload; ++L) {
            const int s = L % kTmaStages, zz = z0 - 1 + L;
            // the stage's previous load (L - S) is released once every consumer warp has read it
            if (L >= kTmaStages && !st_bar_wait(st_smem(&empty[s]), (uint32_t)((L / kTmaStages - 1) & 1), a.spin)) {
                ok = false;
                break;
            }
            const bool with_a = a.has_alpha && zz >= z0 && zz < z1;
            const uint32_t bar = st_smem(&full[s]);
            const uint32_t bytes = (uint32_t)(4 * ufl) + (with_a ? (uint32_t)(4 * TY * nx) : 0u);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
                "%5}], [%2];" ::"r"(st_smem(sm + s * sfl)),
                "l"(reinterpret_cast<uint64_t>(&umap)), "r"(bar), "r"(0), "r"(y0 - 1), "r"(zz)
                : "memory");
            if (with_a)
                asm volatile(
                    "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
                    "%4, %5}], [%2];" ::"r"(st_smem(sm + s * sfl + ufl)),
                    "l"(reinterpret_cast<uint64_t>(&amap)), "r"(bar), "r"(0), "r"(y0), "r"(zz)
                    : "memory");
        }
        if (!ok) atomicExch(a.err, 1);
        // each stage's latest load is the only one that can still be in flight
        for (int j = L - kTmaStages < 0 ? 0 : L - kTmaStages; j < L; ++j)
            (void)st_bar_wait(st_smem(&full[j % kTmaStages]), (uint32_t)((j / kTmaStages) & 1), kTmaSpin);
        return;
    }
    const int gpr = nx >> 2;  // float4 groups per row
    const int r = tid / gpr, x0 = (tid - r * gpr) << 2;
    const int y = y0 + r, lane = tid & 31;
    const bool row_ok = r < TY && y < a.ny;
    const int64_t sxy = (int64_t)nx * a.ny;
    int waited = 0;
    for (int k = 1; k + 1 < nload; ++k) {  // plane z = z0 - 1 + k from loads k-1, k, k+1
        bool ok = true;
        while (ok && waited <= k + 1) {
            ok = st_bar_wait(st_smem(&full[waited % kTmaStages]), (uint32_t)((waited / kTmaStages) & 1), a.spin);
            waited += ok;
        }
        if (!__all_sync(0xffffffffu, ok)) {  // the whole warp leaves together (the shuffles below take all lanes)
            if (lane == 0) atomicExch(a.err, 1);
            break;
        }
        const int z = z0 - 1 + k;
        const float *cen = sm + (k % kTmaStages) * sfl, *bel = sm + ((k - 1) % kTmaStages) * sfl,
                    *abv = sm + ((k + 1) % kTmaStages) * sfl;
        const int o = (r + 1) * nx + x0;
        float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (row_ok) c = *reinterpret_cast<const float4 *>(cen + o);
        // x neighbours: lane - 1's last and lane + 1's first cell (same row when they are needed)
        float xl = __shfl_up_sync(0xffffffffu, c.w, 1), xr = __shfl_down_sync(0xffffffffu, c.x, 1);
        if (row_ok) {
            if (lane == 0 && x0 > 0) xl = cen[o - 1];
            if (lane == 31 && x0 + 4 < nx) xr = cen[o + 4];
            float4 res = c;
            if (y > 0 && y < a.ny - 1 && z > 0 && z < a.nz - 1) {
                const float4 ym = *reinterpret_cast<const float4 *>(cen + o - nx);
                const float4 yp = *reinterpret_cast<const float4 *>(cen + o + nx);
                const float4 zm = *reinterpret_cast<const float4 *>(bel + o);
                const float4 zp = *reinterpret_cast<const float4 *>(abv + o);
                const float4 al = a.has_alpha ? *reinterpret_cast<const float4 *>(cen + ufl + r * nx + x0)
                                              : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
                const float cs[6] = {xl, c.x, c.y, c.z, c.w, xr};
                const float ymv[4] = {ym.x, ym.y, ym.z, ym.w}, ypv[4] = {yp.x, yp.y, yp.z, yp.w};
                const float zmv[4] = {zm.x, zm.y, zm.z, zm.w}, zpv[4] = {zp.x, zp.y, zp.z, zp.w};
                const float av[4] = {al.x, al.y, al.z, al.w};
                float rv[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int x = x0 + t;
                    rv[t] = (x > 0 && x < nx - 1) ? st_update(cs[t + 1], cs[t], cs[t + 2], ymv[t], ypv[t], zmv[t],
                                                              zpv[t], av[t], a.idx2, a.idy2, a.idz2, a.dt)
                                                  : cs[t + 1];
                }
                res = make_float4(rv[0], rv[1], rv[2], rv[3]);
            }
            __stcs(reinterpret_cast<float4 *>(a.out + (int64_t)z * sxy + (int64_t)y * nx + x0), res);
        }
        // load k - 1 is read for the last time here: this warp releases its stage
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(st_smem(&empty[(k - 1) % kTmaStages]))
                         : "memory");
    }
}

// Per device: the flag a timed-out stage wait of k_stencil_tma sets, and the
// CTAs of it resident per SM.
struct StencilTmaDevice {
    int *err_flag = nullptr;
    int per_sm = 0;
};
StencilTmaDevice stencil_tma_dev[kMaxDevices];
DeviceOnce stencil_tma_once;

size_t stencil_tma_smem(int nx) { return sizeof(float) * kTmaStages * (size_t)((2 * (2048 / nx) + 2) * nx); }

bool stencil_tma_fits(int nx, int ny, int nz, const float *alpha, const float *u, const float *out)
{
    const uintptr_t al = reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(out) |
                         reinterpret_cast<uintptr_t>(alpha);
    return nx >= 16 && nx <= 256 && nx % 4 == 0 && 2048 % nx == 0 && (al & 15) == 0 &&
           (int64_t)nx * ny * nz < ((int64_t)1 << 31);
}

int encode_plane_map(CUtensorMap *m, const float *base, int nx, int ny, int nz, int rows)
{
    // the driver entry point, resolved once for all host threads
    static std::once_flag resolved;
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    std::call_once(resolved, []() {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess && fn)
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!encode) {
        set_error("cuTensorMapEncodeTiled is not available");
        return PIRO_ERR_CUDA;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)nx * ny * 4};
    const cuuint32_t box[3] = {(cuuint32_t)nx, (cuuint32_t)rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

int stencil_tma_setup(int dev)
{
    return device_once(stencil_tma_once, dev, [dev]() -> int {
        StencilTmaDevice &d = stencil_tma_dev[dev];
        // the largest stage ring (nx = 256) sets the attribute for every nx
        PIRO_CUDA(cudaFuncSetAttribute(k_stencil_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)stencil_tma_smem(256)));
        PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.per_sm, k_stencil_tma, kTmaThreads + 32,
                                                                stencil_tma_smem(256)));
        if (!d.err_flag) {
            PIRO_CUDA(cudaMalloc(&d.err_flag, sizeof(int)));
            PIRO_CUDA(cudaMemset(d.err_flag, 0, sizeof(int)));
        }
        return PIRO_OK;
    });
}

int stencil_tma_step(int nx, int ny, int nz, float idx2, float idy2, float idz2, float dt, const float *alpha,
                     const float *u, float *out, cudaStream_t st)
{
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    int rc = stencil_tma_setup(dev);
    if (rc != PIRO_OK) return rc;
    const StencilTmaDevice &d = stencil_tma_dev[dev];
    const int TY = 2048 / nx;
    const int ytiles = (int)cdiv(ny, TY);
    // one wave: about (resident CTAs) / (row blocks) z runs per row block
    const int wave = (d.per_sm > 0 ? d.per_sm : 1) * sm_count();
    int runs = wave / ytiles;
    runs = runs < 1 ? 1 : (runs > nz ? nz : runs);
    const int zchunk = (int)cdiv(nz, runs);
    runs = (int)cdiv(nz, zchunk);
    CUtensorMap umap, amap;
    rc = encode_plane_map(&umap, u, nx, ny, nz, TY + 2);
    if (!rc) rc = encode_plane_map(&amap, alpha ? alpha : u, nx, ny, nz, TY);
    if (rc) return rc;
    StencilTma a{nx, ny, nz, TY, zchunk, alpha ? 1 : 0, idx2, idy2, idz2, dt, out, d.err_flag, wait_limit(kTmaSpin)};
    k_stencil_tma<<<dim3((unsigned)ytiles, (unsigned)runs), kTmaThreads + 32, stencil_tma_smem(nx), st>>>(umap, amap,
                                                                                                        a);
    PIRO_CHECK_LAUNCH("k_stencil_tma");
    return PIRO_OK;
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_csr_fe_step(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                                float dt, const float *u, float *out, piro_stream_t stream)
{
    return launch_csr_step<0>(nx, ny, nz, rowptr, col, val, dt, u, out, stream);
}

extern "C" int piro_csr_fe_step_rows(int nx, int ny, int nz, int64_t row0, int64_t nrows, const int32_t *rowptr,
                                     const int32_t *col, const float *val, float dt, const float *u, int64_t ubase,
                                     float *out, piro_stream_t stream)
{
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(grid_ok(nx, ny, nz) && rowptr && col && val && u && out && u != out && row0 >= 0 && nrows > 0 &&
                 row0 + nrows <= N && ubase >= 0,
             "piro_csr_fe_step_rows: bad arguments");
    k_csr_step<0><<<csr_rows_grid(nrows), kRowThreads, 0, as_stream(stream)>>>(GridDiv(nx, ny, nz), nrows, rowptr,
                                                                              col, val, dt, u, out, row0, ubase);
    PIRO_CHECK_LAUNCH("k_csr_step");
    return PIRO_OK;
}

extern "C" int piro_csr_i1(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                           float dt, const float *u, float *out, piro_stream_t stream)
{
    return launch_csr_step<1>(nx, ny, nz, rowptr, col, val, dt, u, out, stream);
}

// Per device: the input-check flags of k_coo_segsum.


static std::mutex coo_scratch_mu[kMaxDevices];
static void *coo_scratch_buf[kMaxDevices] = {};
static size_t coo_scratch_cap[kMaxDevices] = {};

static int coo_common(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals, float dt,
                      const float *u, float *out, bool fe, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && N < INT32_MAX && nnz >= 0 && (nnz == 0 || (rows && cols && vals)) && u && out,
             "coo spmv: bad arguments");
    PIRO_ARG(u != out, "coo spmv: u and out must differ");
    cudaStream_t s = as_stream(stream);
    if (nnz == 0) {  // every row empty: dt*0 (+ u)
        PIRO_CUDA(cudaMemsetAsync(out, 0, sizeof(float) * N, s));
        k_scale_add<<<grid_for(N, 256, 8), 256, 0, s>>>(N, dt, out, fe ? u : nullptr, out);
        PIRO_CHECK_LAUNCH("k_scale_add");
        return PIRO_OK;
    }
    // scratch: the input-check flag, then for the 16-byte path the per-span
    // parts and records of rows that cross spans.  One buffer per device,
    // grown on demand and held under a lock for the whole call (the call
    // ends with a stream synchronize), so calls from several host threads or
    // streams never share it while in flight.
    const bool al16 = ((reinterpret_cast<uintptr_t>(rows) | reinterpret_cast<uintptr_t>(cols) |
                        reinterpret_cast<uintptr_t>(vals)) & 15) == 0;
    const int64_t nspan = cdiv(nnz, kCooSpan);
    const size_t scratch = 256 + (al16 ? 16 * (size_t)nspan : 0);
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    PIRO_ARG(dev >= 0 && dev < kMaxDevices, "coo spmv: device index out of range");
    std::lock_guard<std::mutex> lk(coo_scratch_mu[dev]);
    if (coo_scratch_cap[dev] < scratch) {
        if (coo_scratch_buf[dev]) PIRO_CUDA(cudaFree(coo_scratch_buf[dev]));
        coo_scratch_buf[dev] = nullptr;
        coo_scratch_cap[dev] = 0;
        PIRO_CUDA(cudaMalloc(&coo_scratch_buf[dev], scratch));
        coo_scratch_cap[dev] = scratch;
    }
    void *mem = coo_scratch_buf[dev];
    int *err = static_cast<int *>(mem);
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e == cudaSuccess && al16) {
        float *parts = reinterpret_cast<float *>(static_cast<char *>(mem) + 256);
        float *part_first = parts, *part_last = parts + nspan;
        int32_t *span_row = reinterpret_cast<int32_t *>(parts + 2 * nspan);
        int32_t *span_whole = reinterpret_cast<int32_t *>(parts + 3 * nspan);
        const unsigned g1 = grid_for(cdiv(nnz, kCooPer), 256, 8), g2 = grid_for(nspan, 256, 4);
        if (fe) {
            k_coo_segsum8<true><<<g1, 256, 0, s>>>(N, nnz, rows, cols, vals, u, dt, out, part_first, part_last, span_row,
                                                   span_whole, err);
            k_coo_span_fixup<true><<<g2, 256, 0, s>>>(nspan, u, dt, part_first, part_last, span_row, span_whole, out);
        } else {
            k_coo_segsum8<false><<<g1, 256, 0, s>>>(N, nnz, rows, cols, vals, u, dt, out, part_first, part_last,
                                                    span_row, span_whole, err);
            k_coo_span_fixup<false><<<g2, 256, 0, s>>>(nspan, u, dt, part_first, part_last, span_row, span_whole, out);
        }
        e = cudaGetLastError();
    } else if (e == cudaSuccess) {
        // out doubles as the accumulator: zero it, sum into it, then scale in place.
        e = cudaMemsetAsync(out, 0, sizeof(float) * N, s);
        if (e == cudaSuccess) {
            k_coo_segsum<<<grid_for(nnz, 256, 8), 256, 0, s>>>(N, nnz, rows, cols, vals, u, out, err);
            k_scale_add<<<grid_for(N, 256, 8), 256, 0, s>>>(N, dt, out, fe ? u : nullptr, out);
            e = cudaGetLastError();
        }
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error("coo spmv: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    PIRO_ARG(!(h & 1), "coo spmv: a row or column id outside [0, N)");
    PIRO_ARG(!(h & 2), "coo spmv: row ids not sorted ascending (use piro_coo_row_index for its check)");
    return PIRO_OK;
}

extern "C" int piro_coo_spmv(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals,
                             float dt, const float *u, float *out, piro_stream_t stream)
{
    return coo_common(N, nnz, rows, cols, vals, dt, u, out, false, stream);
}

extern "C" int piro_coo_fe_step(int64_t N, int64_t nnz, const int32_t *rows, const int32_t *cols, const float *vals,
                                float dt, const float *u, float *out, piro_stream_t stream)
{
    return coo_common(N, nnz, rows, cols, vals, dt, u, out, true, stream);
}

extern "C" int piro_csr_fe_step_bc(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                                   float dt, const float *u, const float *bc, float *out, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && rowptr && col && val && u && out && u != out && bc != out,
             "piro_csr_fe_step_bc: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    k_csr_step_bc<<<csr_rows_grid(N), kRowThreads, 0, as_stream(stream)>>>(GridDiv(nx, ny, nz), N, rowptr, col, val,
                                                                            dt, u, bc, out);
    PIRO_CHECK_LAUNCH("k_csr_step_bc");
    return PIRO_OK;
}

extern "C" int piro_coo_row_index(int64_t N, int64_t nnz, const int32_t *rows, int32_t *rowstart, void *work,
                                  size_t work_bytes, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && N < INT32_MAX && nnz >= 0 && nnz < INT32_MAX && rowstart && (nnz == 0 || rows),
             "piro_coo_row_index: bad arguments");
    PIRO_ARG(work && work_bytes >= sizeof(int), "piro_coo_row_index: workspace too small");
    cudaStream_t s = as_stream(stream);
    if (nnz == 0) {
        PIRO_CUDA(cudaMemsetAsync(rowstart, 0, sizeof(int32_t) * (size_t)(N + 1), s));
        return PIRO_OK;
    }
    int *err = static_cast<int *>(work);
    PIRO_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    k_coo_rowstart<<<grid_for(nnz, 256, 8), 256, 0, s>>>(N, nnz, rows, rowstart, err);
    PIRO_CHECK_LAUNCH("k_coo_rowstart");
    int h = 0;
    PIRO_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    PIRO_CUDA(cudaStreamSynchronize(s));
    PIRO_ARG(!h, "piro_coo_row_index: rows not sorted ascending, or out of range");
    return PIRO_OK;
}

extern "C" int piro_coo_step_indexed(int64_t N, const int32_t *rowstart, const int32_t *cols, const float *vals,
                                     float dt, int fe, const float *u, float *out, piro_stream_t stream)
{
    PIRO_ARG(N > 0 && rowstart && cols && vals && u && out && u != out, "piro_coo_step_indexed: bad arguments");
    k_coo_rows<<<csr_rows_grid(N), kRowThreads, 0, as_stream(stream)>>>(N, rowstart, cols, vals, dt, fe, u, out);
    PIRO_CHECK_LAUNCH("k_coo_rows");
    return PIRO_OK;
}

extern "C" int piro_ht_spmv(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts, float dt, int fe,
                            const float *u, float *out, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && keys && vals && ts > 0 && u && out && u != out, "piro_ht_spmv: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    k_ht_spmv<false><<<grid_for(N, 256, 8), 256, 0, as_stream(stream)>>>(GridDiv(nx, ny, nz), N, keys, vals, ts,
                                                                         ModU64((uint64_t)ts), dt, fe, nullptr,
                                                                         u, out);
    PIRO_CHECK_LAUNCH("k_ht_spmv");
    return PIRO_OK;
}

extern "C" int piro_ht_row_order_workspace(int64_t N, int64_t ts, size_t *bytes)
{
    PIRO_ARG(bytes && N > 0 && ts > 0, "piro_ht_row_order_workspace: bad arguments");
    const int64_t nbk = (ts >> kOrderShift) + 1;
    *bytes = sizeof(int32_t) * (size_t)(nbk + 1) + 256 + scan_workspace_bytes(nbk);
    return PIRO_OK;
}

extern "C" int piro_ht_row_order(int64_t N, int64_t ts, int32_t *order, void *work, size_t work_bytes,
                                 piro_stream_t stream)
{
    PIRO_ARG(N > 0 && N < INT32_MAX && ts > 0 && order && work, "piro_ht_row_order: bad arguments");
    PIRO_ARG(N <= INT64_MAX / (N + 1), "piro_ht_row_order: row*N+col overflows int64");
    size_t need = 0;
    piro_ht_row_order_workspace(N, ts, &need);
    PIRO_ARG(work_bytes >= need, "piro_ht_row_order: workspace too small");
    const int64_t nbk = (ts >> kOrderShift) + 1;
    cudaStream_t s = as_stream(stream);
    int32_t *cnt = static_cast<int32_t *>(work);  // [nbk + 1]: cnt[0] = 0, bucket counts after it
    void *scan_work = static_cast<char *>(work) + (sizeof(int32_t) * (size_t)(nbk + 1) + 255) / 256 * 256;
    PIRO_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (size_t)(nbk + 1), s));
    k_order_count<<<grid_for(N, 256, 8), 256, 0, s>>>(N, ts, cnt);
    PIRO_CHECK_LAUNCH("k_order_count");
    const int rc = scan_rowptr_inplace(nbk, cnt, scan_work, scan_workspace_bytes(nbk), s);
    if (rc) return rc;
    // cnt[b] is now the first position of bucket b: use it as the cursor
    k_order_scatter<<<grid_for(N, 256, 8), 256, 0, s>>>(N, ts, cnt, order);
    PIRO_CHECK_LAUNCH("k_order_scatter");
    return PIRO_OK;
}

extern "C" int piro_ht_spmv_ordered(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts,
                                    float dt, int fe, const int32_t *order, const float *u, float *out,
                                    piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && keys && vals && ts > 0 && order && u && out && u != out,
             "piro_ht_spmv_ordered: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    k_ht_spmv<true><<<grid_for(N, 256, 8), 256, 0, as_stream(stream)>>>(GridDiv(nx, ny, nz), N, keys, vals, ts,
                                                                        ModU64((uint64_t)ts), dt, fe, order,
                                                                        u, out);
    PIRO_CHECK_LAUNCH("k_ht_spmv");
    return PIRO_OK;
}

extern "C" int piro_ht_stage_bytes(int64_t N, size_t *bytes)
{
    PIRO_ARG(bytes && N > 0, "piro_ht_stage_bytes: bad arguments");
    *bytes = 32 * (size_t)N;
    return PIRO_OK;
}

extern "C" int piro_ht_spmv_staged(int nx, int ny, int nz, const int64_t *keys, const float *vals, int64_t ts,
                                   float dt, int fe, const int32_t *order, void *stage, size_t stage_bytes,
                                   const float *u, float *out, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && keys && vals && ts > 0 && order && stage && u && out && u != out,
             "piro_ht_spmv_staged: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(N < INT32_MAX, "piro_ht_spmv_staged: more than 2^31 - 1 rows");
    PIRO_ARG(stage_bytes >= 32 * (size_t)N && ((uintptr_t)stage & 15) == 0,
             "piro_ht_spmv_staged: stage smaller than 32 bytes per row or not 16-byte aligned");
    cudaStream_t s = as_stream(stream);
    float4 *st = static_cast<float4 *>(stage);
    const GridDiv g(nx, ny, nz);
    k_ht_stage<<<grid_for(N, 256, 8), 256, 0, s>>>(g, N, keys, vals, ts, ModU64((uint64_t)ts), order, st);
    PIRO_CHECK_LAUNCH("k_ht_stage");
    k_ht_stage_apply<<<grid_for(N, 256, 8), 256, 0, s>>>(g, dt, fe, st, u, out);
    PIRO_CHECK_LAUNCH("k_ht_stage_apply");
    return PIRO_OK;
}

extern "C" int piro_stencil_fe_step(int nx, int ny, int nz, float idx2, float idy2, float idz2, float dt,
                                    const float *alpha, const float *u, float *out, piro_stream_t stream)
{
    PIRO_ARG(grid_ok(nx, ny, nz) && u && out && u != out, "piro_stencil_fe_step: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    if (stencil_tma_fits(nx, ny, nz, alpha, u, out))
        return stencil_tma_step(nx, ny, nz, idx2, idy2, idz2, dt, alpha, u, out, as_stream(stream));
    const uintptr_t al = reinterpret_cast<uintptr_t>(u) | reinterpret_cast<uintptr_t>(out) |
                         reinterpret_cast<uintptr_t>(alpha);
    if (nx % 4 == 0 && N < ((int64_t)1 << 32) && (al & 15) == 0) {
        k_stencil4<<<(unsigned)cdiv(N / 4, 256), 256, 0, as_stream(stream)>>>(nx, ny, nz, idx2, idy2, idz2, dt, alpha,
                                                                             u, out);
        PIRO_CHECK_LAUNCH("k_stencil4");
        return PIRO_OK;
    }
    const dim3 block(kStX, kStY);
    const dim3 grid((unsigned)cdiv(nx, kStX), (unsigned)cdiv(ny, kStY), (unsigned)cdiv(nz, kStZ));
    k_stencil<<<grid, block, 0, as_stream(stream)>>>(nx, ny, nz, idx2, idy2, idz2, dt, alpha, u, out);
    PIRO_CHECK_LAUNCH("k_stencil");
    return PIRO_OK;
}

extern "C" int piro_stencil_check(piro_stream_t stream)
{
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    PIRO_ARG(dev >= 0 && dev < kMaxDevices, "piro_stencil_check: device index");
    if (!stencil_tma_once.done[dev].load(std::memory_order_acquire)) return PIRO_OK;  // no staged step ran here
    int *flag = stencil_tma_dev[dev].err_flag;
    int h = 0;
    cudaStream_t st = as_stream(stream);
    PIRO_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (h) {
        PIRO_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
        set_error("piro_stencil_fe_step: a stage wait timed out");
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

extern "C" int piro_set_bc(int64_t q, const uint32_t *idx, const float *src, float *dst, piro_stream_t stream)
{
    PIRO_ARG(q >= 0 && (q == 0 || (idx && src && dst)), "piro_set_bc: bad arguments");
    if (q == 0) return PIRO_OK;
    k_set_bc<<<grid_for(q, 256, 4), 256, 0, as_stream(stream)>>>(q, idx, src, dst);
    PIRO_CHECK_LAUNCH("k_set_bc");
    return PIRO_OK;
}

extern "C" int piro_vec_op(int op, int64_t n, const float *b, const float *c, float *a, piro_stream_t stream)
{
    PIRO_ARG(op >= 0 && op <= 3 && n >= 0 && (n == 0 || (a && b && c)), "piro_vec_op: bad arguments");
    if (n == 0) return PIRO_OK;
    k_vec_op<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(op, n, b, c, a);
    PIRO_CHECK_LAUNCH("k_vec_op");
    return PIRO_OK;
}

extern "C" int piro_vec_op_scalar(int op, int64_t n, float s, const float *c, float *a, piro_stream_t stream)
{
    PIRO_ARG(op >= 0 && op <= 3 && n >= 0 && (n == 0 || (a && c)), "piro_vec_op_scalar: bad arguments");
    if (n == 0) return PIRO_OK;
    k_vec_op_scalar<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(op, n, s, c, a);
    PIRO_CHECK_LAUNCH("k_vec_op_scalar");
    return PIRO_OK;
}

extern "C" int piro_vec_urf(int64_t n, float *a, float *c, float urf, piro_stream_t stream)
{
    PIRO_ARG(n >= 0 && (n == 0 || (a && c)), "piro_vec_urf: bad arguments");
    if (n == 0) return PIRO_OK;
    k_vec_urf<<<grid_for(n, 256, 8), 256, 0, as_stream(stream)>>>(n, a, c, urf);
    PIRO_CHECK_LAUNCH("k_vec_urf");
    return PIRO_OK;
}

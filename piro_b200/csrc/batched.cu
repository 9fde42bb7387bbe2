// batched.cu -- many independent heat problems of uneven sizes stepped
// together: one persistent cooperative launch per time step (two steps per
// replayed CUDA graph), each member a constant-alpha problem on its own ghost-inclusive
// cube, forward Euler (TIMESCHEME 11, src/kernelprocess.cpp:10-40) or
// backward Euler (TIMESCHEME 12, solved as the single-grid solver does:
// FP32 Jacobi-PCG inside FP64 iterative refinement to a relative residual).
//
// Layout in HBM: every member's field is one contiguous float block of n^3
// cells (index x + y*n + z*n^2), members back to back.  Work is cut into
// tiles of kTile.. cells that never cross a member; FE tiles and BE tiles have
// their own lists.
//
// One step (k_batch_step):
//   P0   FE tiles: out = u + dt*(alpha*lap u) on interior cells (the
//        arithmetic of the matrix-free forward-Euler kernel), boundary copied;
//        BE tiles: b = u, x64 = u, d = 0.  One warp per BE member sets its
//        solver state.
//   then, until every BE member is done, rounds of four phases separated by
//   a grid barrier:
//   V1   per BE tile, by member mode: RESID -- r = b - A(x64 + d) in FP64
//        (the pending correction d of the last sweep included), partials of
//        |r64|^2, |b|^2, <r, z>, |r32|^2; CG -- p = z + beta p_old, q = A p
//        (FP32, matrix-free), partial <p, q>.  z = r / A_rr is never stored.
//   S1   one warp per member sums its tiles' partials in a fixed order and
//        decides: after RESID, done (relative residual <= rtol), stalled, or
//        a new CG sweep; in CG, the step length a.
//   V2   x64 += d, d = 0 for members that just evaluated a residual (and the
//        FP32 result for the finished ones); CG members: d += a p, r -= a q,
//        partials <r, z>, |r|^2.
//   S2   one warp per member: next beta, inner stop test, the count of
//        members still active.
// All sums are per-tile block reductions plus an in-order per-member sum, so
// results do not depend on scheduling.  The CG sums' terms are FP32 products
// (they only steer CG) added in FP64; the residual norms are FP64 throughout.  The grid barrier's waits are bounded:
// on timeout an error flag is raised and every block leaves.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace piro {
namespace {

enum : int { kResid = 1, kCgStart = 2, kCg = 3, kFinish = 4, kDone = 5 };

struct BMember {
    GridDiv g;
    int64_t off, N;      // first cell, cells
    float alpha, dt;
    float cd, co, dinv;  // FP32 inner operator: diagonal, off-diagonal, 1 / diagonal
    double cd64, co64;   // FP64 operator of the residual
    int scheme;          // 0 forward Euler, 1 backward Euler
    int tile0, ntiles;   // this member's BE tiles (BE members only)
};

struct BState {
    int mode, sweep, it, inner_total, status;
    double rz, rr0, tol2, rel, prev_rel, a, beta;
};

struct BarrierState {
    unsigned count, gen;
    int err;
    int active[2];
};

struct BArgs {
    const BMember *mem;
    int M;
    const int *fe_tile_m, *be_tile_m;  // tile -> member
    const int64_t *fe_tile_s, *be_tile_s;  // tile -> first cell within the member
    int nfe, nbe, tile;
    const float *u;
    float *out, *b, *r, *p0, *p1, *q, *d;
    double *x64;
    double *partials;  // [nbe][4]
    BState *st;
    BarrierState *bar;
    double rtol, inner_floor;
    int max_sweeps, max_inner, max_rounds;
    long long spin_limit;
};

constexpr int kThreads = 256;

__device__ __forceinline__ bool grid_sync(BarrierState *bs, long long spin_limit, int *s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &bs->gen;
        volatile int *verr = &bs->err;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&bs->count, 1u) + 1u;
        int ok = 1;
        if (arrived == gridDim.x) {
            atomicExch(&bs->count, 0u);
            __threadfence();
            atomicAdd(&bs->gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == g) {
                if (*verr || ++spins > spin_limit) {
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (*verr) ok = 0;
        if (!ok) atomicExch(&bs->err, 1);
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

__device__ __forceinline__ double block_sum(double v, double *s_warp)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s_warp[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0.0;
        t = warp_sum(t);
    }
    return t;  // thread 0
}

// kN block sums in one shared-memory round (thread 0 holds the totals).
template <int kN>
__device__ __forceinline__ void block_sums(double (&v)[kN], double *s_red)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int t = 0; t < kN; ++t) v[t] = warp_sum(v[t]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int t = 0; t < kN; ++t) s_red[t * 32 + w] = v[t];
    __syncthreads();
    if (w == 0)
#pragma unroll
        for (int t = 0; t < kN; ++t) v[t] = warp_sum(lane < nw ? s_red[t * 32 + lane] : 0.0);
}

// In-order (lane-strided, then butterfly) sum of `count` partials of stride 4
// starting at p; every lane gets the result.
__device__ __forceinline__ double warp_partial_sum(const double *p, int count)
{
    double s = 0.0;
    for (int i = threadIdx.x & 31; i < count; i += 32) s += ((volatile const double *)p)[4 * i];
    return warp_sum(s);
}

// FP32 matrix-free A v at an interior cell (A = I - dt*alpha*L, 7-point L, h = 1).
__device__ __forceinline__ float a_apply32(const BMember &m, const float *v, int64_t i, int64_t sxy)
{
    const int nx = m.g.nx;
    return m.cd * v[i] + m.co * (((v[i - 1] + v[i + 1]) + (v[i - nx] + v[i + nx])) + (v[i - sxy] + v[i + sxy]));
}

// kMinBlocks: the blocks per SM the registers are capped for (4: 64
// registers; 6 and 8 cap them at 40 and 32 for more warps per SM).
template <int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_batch_step(BArgs A)
{
    __shared__ double s_warp[32];
    __shared__ double s_red[4 * 32];
    __shared__ int s_ok;
    const int nwarps_grid = (int)(gridDim.x * (blockDim.x >> 5));
    const int gwarp = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const int lane = threadIdx.x & 31;

    // ---- P0: forward-Euler members, and the start of the backward-Euler ones
    for (int t = blockIdx.x; t < A.nfe; t += gridDim.x) {
        const BMember m = A.mem[A.fe_tile_m[t]];
        const int64_t s0 = A.fe_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
        const int64_t sxy = (int64_t)m.g.nx * m.g.ny;
        const float *u = A.u + m.off;
        float *o = A.out + m.off;
        for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const float c = u[i];
            if (m.g.interior(i)) {
                const float c2 = __fmul_rn(2.0f, c);
                const float lx = __fsub_rn(__fadd_rn(u[i + 1], u[i - 1]), c2);
                const float ly = __fsub_rn(__fadd_rn(u[i + m.g.nx], u[i - m.g.nx]), c2);
                const float lz = __fsub_rn(__fadd_rn(u[i + sxy], u[i - sxy]), c2);
                const float lap = __fadd_rn(__fadd_rn(lx, ly), lz);
                o[i] = __fadd_rn(c, __fmul_rn(m.dt, __fmul_rn(m.alpha, lap)));
            } else {
                o[i] = c;
            }
        }
    }
    for (int t = blockIdx.x; t < A.nbe; t += gridDim.x) {
        const BMember m = A.mem[A.be_tile_m[t]];
        const int64_t s0 = A.be_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
        for (int64_t i = m.off + s0 + threadIdx.x; i < m.off + s1; i += blockDim.x) {
            const float v = A.u[i];
            A.b[i] = v;
            A.x64[i] = (double)v;
            A.d[i] = 0.0f;
        }
    }
    for (int k = gwarp; k < A.M; k += nwarps_grid) {
        if (lane == 0) {
            BState s{};
            s.mode = A.mem[k].scheme == 1 ? kResid : kDone;
            s.status = A.mem[k].scheme == 1 ? PIRO_ERR_NOT_CONVERGED : PIRO_OK;
            s.prev_rel = INFINITY;
            A.st[k] = s;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        A.bar->active[0] = 0;
        A.bar->active[1] = 0;
    }
    if (!grid_sync(A.bar, A.spin_limit, &s_ok)) return;

    for (int round = 0; round < A.max_rounds; ++round) {
        // ---- V1
        for (int t = blockIdx.x; t < A.nbe; t += gridDim.x) {
            const int mi = A.be_tile_m[t];
            const BMember m = A.mem[mi];
            const BState s = A.st[mi];
            const int64_t s0 = A.be_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
            const int64_t sxy = (int64_t)m.g.nx * m.g.ny;
            double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
            if (s.mode == kResid) {
                const double *x = A.x64 + m.off;
                const float *dd = A.d + m.off, *bb = A.b + m.off;
                float *rr = A.r + m.off;
                for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
                    if (!m.g.interior(i)) {
                        rr[i] = 0.0f;
                        continue;
                    }
                    const int nx = m.g.nx;
                    const double xc = x[i] + (double)dd[i];
                    const double nb = ((x[i - 1] + (double)dd[i - 1]) + (x[i + 1] + (double)dd[i + 1])) +
                                      ((x[i - nx] + (double)dd[i - nx]) + (x[i + nx] + (double)dd[i + nx])) +
                                      ((x[i - sxy] + (double)dd[i - sxy]) + (x[i + sxy] + (double)dd[i + sxy]));
                    const double bi = (double)bb[i];
                    const double ri = bi - (m.cd64 * xc + m.co64 * nb);
                    const float rf = (float)ri;
                    rr[i] = rf;
                    v0 += ri * ri;
                    v1 += bi * bi;
                    v2 += (double)rf * (double)(rf * m.dinv);
                    v3 += (double)rf * (double)rf;
                }
            } else if (s.mode == kCg) {
                const float beta = (float)s.beta;
                const float *rr = A.r + m.off;
                const float *po = ((s.it & 1) ? A.p1 : A.p0) + m.off;
                float *pn = ((s.it & 1) ? A.p0 : A.p1) + m.off;
                float *qq = A.q + m.off;
                const int nx = m.g.nx;
                // p = z + beta p_old at the cell and its six neighbours (boundary
                // neighbours carry r = 0 and p_old = 0).  Two cells per
                // iteration (i and i + blockDim.x, the thread's cells in their
                // usual order) so that both cells' 14 loads are in flight together.
                auto pv = [&](int64_t j) { return rr[j] * m.dinv + beta * po[j]; };
                for (int64_t i = s0 + threadIdx.x; i < s1; i += 2 * blockDim.x) {
                    const int64_t i2 = i + blockDim.x;
                    const bool in1 = m.g.interior(i), in2 = i2 < s1 && m.g.interior(i2);
                    float c1 = 0.0f, nb1 = 0.0f, c2 = 0.0f, nb2 = 0.0f;
                    if (in1) {
                        c1 = pv(i);
                        nb1 = ((pv(i - 1) + pv(i + 1)) + (pv(i - nx) + pv(i + nx))) + (pv(i - sxy) + pv(i + sxy));
                    }
                    if (in2) {
                        c2 = pv(i2);
                        nb2 = ((pv(i2 - 1) + pv(i2 + 1)) + (pv(i2 - nx) + pv(i2 + nx))) + (pv(i2 - sxy) + pv(i2 + sxy));
                    }
                    float pq = 0.0f;  // the two cells' <p, q> terms in FP32, added in FP64
                    if (in1) {
                        const float qv = m.cd * c1 + m.co * nb1;
                        pn[i] = c1;
                        qq[i] = qv;
                        pq = c1 * qv;
                    } else {
                        pn[i] = 0.0f;
                        qq[i] = 0.0f;
                    }
                    if (i2 < s1) {
                        if (in2) {
                            const float qv = m.cd * c2 + m.co * nb2;
                            pn[i2] = c2;
                            qq[i2] = qv;
                            pq += c2 * qv;
                        } else {
                            pn[i2] = 0.0f;
                            qq[i2] = 0.0f;
                        }
                    }
                    v0 += (double)pq;
                }
            } else {
                continue;
            }
            if (s.mode == kResid) {
                double v[4] = {v0, v1, v2, v3};
                block_sums<4>(v, s_red);
                if (threadIdx.x == 0) {
                    double *pp = A.partials + 4 * (int64_t)t;
                    pp[0] = v[0];
                    pp[1] = v[1];
                    pp[2] = v[2];
                    pp[3] = v[3];
                }
            } else {
                const double t0 = block_sum(v0, s_warp);  // CG: <p, q> only
                if (threadIdx.x == 0) A.partials[4 * (int64_t)t] = t0;
            }
        }
        if (!grid_sync(A.bar, A.spin_limit, &s_ok)) return;
        // ---- S1
        if (blockIdx.x == 0 && threadIdx.x == 0) A.bar->active[(round + 1) & 1] = 0;
        for (int k = gwarp; k < A.M; k += nwarps_grid) {
            const BMember &m = A.mem[k];
            if (m.scheme != 1) continue;
            BState s = A.st[k];
            if (s.mode != kResid && s.mode != kCg) continue;
            const double *pp = A.partials + 4 * (int64_t)m.tile0;
            const double t0 = warp_partial_sum(pp, m.ntiles);
            const double t1 = s.mode == kResid ? warp_partial_sum(pp + 1, m.ntiles) : 0.0;
            const double t2 = s.mode == kResid ? warp_partial_sum(pp + 2, m.ntiles) : 0.0;
            const double t3 = s.mode == kResid ? warp_partial_sum(pp + 3, m.ntiles) : 0.0;
            if (lane != 0) continue;
            if (s.mode == kResid) {
                const double bn = sqrt(t1) > 0.0 ? sqrt(t1) : 1.0;
                const double rel = sqrt(t0) / bn;
                s.rel = rel;
                if (!isfinite(rel)) {
                    s.status = PIRO_STATUS_STALLED;
                    s.mode = kFinish;
                } else if (rel <= A.rtol) {
                    s.status = PIRO_OK;
                    s.mode = kFinish;
                } else if (s.sweep >= A.max_sweeps || s.inner_total >= A.max_inner) {
                    s.status = PIRO_ERR_NOT_CONVERGED;
                    s.mode = kFinish;
                } else if (s.sweep > 0 && rel > 0.5 * s.prev_rel) {
                    s.status = PIRO_STATUS_STALLED;
                    s.mode = kFinish;
                } else {
                    double itol = rel > 0.0 ? 0.5 * A.rtol / rel : 1.0;
                    itol = itol > 0.1 ? 0.1 : itol;
                    itol = itol < A.inner_floor ? A.inner_floor : itol;
                    s.tol2 = itol * itol;
                    s.rz = t2;
                    s.rr0 = t3;
                    s.beta = 0.0;
                    s.it = 0;
                    s.prev_rel = rel;
                    s.sweep += 1;
                    s.mode = t3 > 0.0 ? kCgStart : kFinish;
                }
            } else {
                const double a = s.rz / t0;
                if (!isfinite(a) || t0 <= 0.0) {
                    s.status = PIRO_STATUS_STALLED;
                    s.mode = kFinish;
                    s.a = 0.0;
                } else {
                    s.a = a;
                }
            }
            A.st[k] = s;
        }
        if (!grid_sync(A.bar, A.spin_limit, &s_ok)) return;
        // ---- V2
        for (int t = blockIdx.x; t < A.nbe; t += gridDim.x) {
            const int mi = A.be_tile_m[t];
            const BMember m = A.mem[mi];
            const BState s = A.st[mi];
            const int64_t s0 = A.be_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
            if (s.mode == kCgStart || s.mode == kFinish) {
                double *x = A.x64 + m.off;
                float *dd = A.d + m.off;
                for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
                    const double xn = x[i] + (double)dd[i];
                    x[i] = xn;
                    dd[i] = 0.0f;
                    if (s.mode == kFinish) A.out[m.off + i] = (float)xn;
                }
            } else if (s.mode == kCg) {
                // Boundary cells carry p = q = r = 0 (V1 and RESID write them so):
                // the update leaves them at zero and they add nothing to the sums,
                // so every cell is updated without a test, float4 groups where the
                // tile is 16-byte aligned (members start 64-cell aligned, tiles
                // are multiples of 64 cells), scalars for the tail.
                const float a = (float)s.a;
                const float *pn = ((s.it & 1) ? A.p0 : A.p1) + m.off;
                const float *qq = A.q + m.off;
                float *rr = A.r + m.off, *dd = A.d + m.off;
                double v0 = 0.0, v1 = 0.0;
                const int64_t g0 = s0 >> 2, g1 = s1 >> 2;  // s0 % 4 == 0
                // two float4 groups per iteration (the thread's groups in their usual
                // order): eight 16-byte loads in flight
                auto upd = [&](float4 &d4, float4 &r4, const float4 p4, const float4 q4) {
                    d4.x += a * p4.x; d4.y += a * p4.y; d4.z += a * p4.z; d4.w += a * p4.w;
                    r4.x = r4.x - a * q4.x; r4.y = r4.y - a * q4.y; r4.z = r4.z - a * q4.z; r4.w = r4.w - a * q4.w;
                    const float r2 = ((r4.x * r4.x + r4.y * r4.y) + (r4.z * r4.z + r4.w * r4.w));
                    v0 += (double)(r2 * m.dinv);  // <r, z> with z = r dinv (dinv uniform per member)
                    v1 += (double)r2;
                };
                for (int64_t gi = g0 + threadIdx.x; gi < g1; gi += 2 * blockDim.x) {
                    const int64_t gj = gi + blockDim.x;
                    const bool two = gj < g1;
                    const float4 p4 = reinterpret_cast<const float4 *>(pn)[gi];
                    const float4 q4 = reinterpret_cast<const float4 *>(qq)[gi];
                    float4 d4 = reinterpret_cast<float4 *>(dd)[gi];
                    float4 r4 = reinterpret_cast<float4 *>(rr)[gi];
                    float4 p5 = make_float4(0.f, 0.f, 0.f, 0.f), q5 = p5, d5 = p5, r5 = p5;
                    if (two) {
                        p5 = reinterpret_cast<const float4 *>(pn)[gj];
                        q5 = reinterpret_cast<const float4 *>(qq)[gj];
                        d5 = reinterpret_cast<float4 *>(dd)[gj];
                        r5 = reinterpret_cast<float4 *>(rr)[gj];
                    }
                    upd(d4, r4, p4, q4);
                    reinterpret_cast<float4 *>(dd)[gi] = d4;
                    reinterpret_cast<float4 *>(rr)[gi] = r4;
                    if (two) {
                        upd(d5, r5, p5, q5);
                        reinterpret_cast<float4 *>(dd)[gj] = d5;
                        reinterpret_cast<float4 *>(rr)[gj] = r5;
                    }
                }
                for (int64_t i = (g1 << 2) + threadIdx.x; i < s1; i += blockDim.x) {
                    dd[i] += a * pn[i];
                    const float ri = rr[i] - a * qq[i];
                    rr[i] = ri;
                    v0 += (double)ri * (double)(ri * m.dinv);
                    v1 += (double)ri * (double)ri;
                }
                double v[2] = {v0, v1};
                block_sums<2>(v, s_red);
                if (threadIdx.x == 0) {
                    double *pp = A.partials + 4 * (int64_t)t;
                    pp[0] = v[0];
                    pp[1] = v[1];
                }
            }
        }
        if (!grid_sync(A.bar, A.spin_limit, &s_ok)) return;
        // ---- S2
        for (int k = gwarp; k < A.M; k += nwarps_grid) {
            const BMember &m = A.mem[k];
            if (m.scheme != 1) continue;
            BState s = A.st[k];
            if (s.mode == kCg) {
                const double *pp = A.partials + 4 * (int64_t)m.tile0;
                const double rz = warp_partial_sum(pp, m.ntiles);
                const double rr = warp_partial_sum(pp + 1, m.ntiles);
                if (lane == 0) {
                    s.it += 1;
                    s.inner_total += 1;
                    const double beta = rz / s.rz;
                    if (!isfinite(rr) || !isfinite(beta)) {
                        s.status = PIRO_STATUS_STALLED;
                        s.mode = kResid;  // evaluate what the sweep reached
                    } else if (rr <= s.tol2 * s.rr0 || s.inner_total >= A.max_inner) {
                        s.mode = kResid;
                    } else {
                        s.beta = beta;
                        s.rz = rz;
                    }
                }
            } else if (lane == 0) {
                if (s.mode == kCgStart) s.mode = kCg;
                else if (s.mode == kFinish) s.mode = kDone;
            }
            if (lane == 0) {
                A.st[k] = s;
                if (s.mode != kDone) atomicAdd(&A.bar->active[round & 1], 1);
            }
        }
        if (!grid_sync(A.bar, A.spin_limit, &s_ok)) return;
        if (*((volatile int *)&A.bar->active[round & 1]) == 0) return;
    }
    // round cap reached: members still running keep their best iterate
    for (int t = blockIdx.x; t < A.nbe; t += gridDim.x) {
        const int mi = A.be_tile_m[t];
        const BMember m = A.mem[mi];
        if (A.st[mi].mode == kDone) continue;
        const int64_t s0 = A.be_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
        for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x)
            A.out[m.off + i] = (float)(A.x64[m.off + i] + (double)A.d[m.off + i]);
    }
}

// ---------------------------------------------------------------------------
// The grouped step (k_batch_groups): the same arithmetic as k_batch_step per
// member, without grid-wide lockstep.  Forward-Euler tiles are stepped by all
// CTAs first.  Each backward-Euler member is a job: a large member gets a
// contiguous group of CTAs (about one per average CTA's share of the cells)
// that split its cells into 64-cell aligned chunks and meet at a group
// barrier -- a monotonic arrival counter per job -- between phases; small
// members are packed onto the other CTAs (longest first, to the least loaded)
// and solved one after another with block barriers only.  No CTA waits for
// a member it does not work on, so members finish at their own pace and the
// step ends when the most loaded CTA is done.  Group sums are per-CTA block
// sums read by every CTA of the group in rank order (identical decisions in
// all of them, results independent of scheduling).  Each phase writes its own
// partial slots (RESID 0-3, the operator step 4, the update 5-6): a CTA that
// runs ahead cannot overwrite a sum another CTA of its group has not read,
// since it reaches the next writes of a slot only after that CTA arrived at
// the barrier that follows the read.
struct BJob {
    int member;
    int gbase, gsize;  // first CTA of the group and its CTAs
    int part_off;      // first double of its partials: 7 slots x gsize
};

struct GArgs {
    const BMember *mem;
    const int *fe_tile_m;
    const int64_t *fe_tile_s;
    int nfe, tile;
    const BJob *jobs;
    const int *cta_ptr, *cta_jobs;  // CTA c works on jobs cta_jobs[cta_ptr[c] .. cta_ptr[c+1])
    unsigned *job_bar;              // arrival counters (zeroed before the launch)
    double *job_part;
    const float *u;
    float *out, *b, *r, *p0, *p1, *q, *d;
    double *x64;
    BState *st;
    BarrierState *bar;  // err: a group barrier wait ran out
    double rtol, inner_floor;
    int max_sweeps, max_inner;
    long long spin_limit;
};

// Group barrier of one job: arrivals only grow within a launch; barrier k of
// the job waits for k * gsize of them.  A single-CTA group is a block barrier.
__device__ __forceinline__ bool group_sync(const GArgs &A, unsigned *count, int gsize, unsigned &target, int *s_ok)
{
    __syncthreads();
    if (gsize == 1) return true;
    target += (unsigned)gsize;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        volatile unsigned *vc = count;
        volatile int *verr = &A.bar->err;
        int ok = 1;
        long long spins = 0;
        while ((int)(*vc - target) < 0) {
            if (*verr || ++spins > A.spin_limit) {
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        if (*verr) ok = 0;
        if (!ok) atomicExch(&A.bar->err, 1);
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// kN group sums: this CTA's block sums into slots first.. (rank q), then,
// after the group barrier, every CTA adds the gsize partials of each slot in
// rank order.  Returns false if the barrier wait ran out.
template <int kN>
__device__ __forceinline__ bool group_sums(const GArgs &A, double *part, int first, int q, int gsize, unsigned *count,
                                           unsigned &target, double (&v)[kN], double *s_red, double *s_tot,
                                           int *s_ok)
{
    block_sums<kN>(v, s_red);
    if (threadIdx.x == 0)
#pragma unroll
        for (int t = 0; t < kN; ++t) part[(first + t) * gsize + q] = v[t];
    if (!group_sync(A, count, gsize, target, s_ok)) return false;
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
#pragma unroll
        for (int t = 0; t < kN; ++t) {
            double a = 0.0;
            for (int k = lane; k < gsize; k += 32) a += ((volatile const double *)part)[(first + t) * gsize + k];
            a = warp_sum(a);
            if (lane == 0) s_tot[t] = a;
        }
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < kN; ++t) v[t] = s_tot[t];
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(kThreads, 4) k_batch_groups(GArgs A)
{
    __shared__ double s_red[4 * 32];
    __shared__ double s_tot[4];
    __shared__ int s_ok;
    // forward-Euler members: one pass over their tiles by every CTA
    for (int t = blockIdx.x; t < A.nfe; t += gridDim.x) {
        const BMember m = A.mem[A.fe_tile_m[t]];
        const int64_t s0 = A.fe_tile_s[t], s1 = min(s0 + (int64_t)A.tile, m.N);
        const int64_t sxy = (int64_t)m.g.nx * m.g.ny;
        const float *u = A.u + m.off;
        float *o = A.out + m.off;
        for (int64_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const float c = u[i];
            if (m.g.interior(i)) {
                const float c2 = __fmul_rn(2.0f, c);
                const float lx = __fsub_rn(__fadd_rn(u[i + 1], u[i - 1]), c2);
                const float ly = __fsub_rn(__fadd_rn(u[i + m.g.nx], u[i - m.g.nx]), c2);
                const float lz = __fsub_rn(__fadd_rn(u[i + sxy], u[i - sxy]), c2);
                const float lap = __fadd_rn(__fadd_rn(lx, ly), lz);
                o[i] = __fadd_rn(c, __fmul_rn(m.dt, __fmul_rn(m.alpha, lap)));
            } else {
                o[i] = c;
            }
        }
    }
    // backward-Euler jobs of this CTA
    for (int jj = A.cta_ptr[blockIdx.x]; jj < A.cta_ptr[blockIdx.x + 1]; ++jj) {
        const BJob J = A.jobs[A.cta_jobs[jj]];
        const BMember m = A.mem[J.member];
        const int G = J.gsize, q = (int)blockIdx.x - J.gbase;
        unsigned *count = A.job_bar + A.cta_jobs[jj];
        double *part = A.job_part + J.part_off;
        unsigned target = 0;
        const int64_t chunk = cdiv(cdiv(m.N, G), 64) * 64;
        const int64_t c0 = min((int64_t)q * chunk, m.N), c1 = min(c0 + chunk, m.N);
        const int64_t sxy = (int64_t)m.g.nx * m.g.ny;
        const int nx = m.g.nx;
        const float *uu = A.u + m.off;
        float *bb = A.b + m.off, *rr = A.r + m.off, *dd = A.d + m.off, *qq = A.q + m.off, *oo = A.out + m.off;
        double *x = A.x64 + m.off;
        for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
            const float v = uu[i];
            bb[i] = v;
            x[i] = (double)v;
            dd[i] = 0.0f;
        }
        BState s{};
        s.status = PIRO_ERR_NOT_CONVERGED;
        s.prev_rel = INFINITY;
        bool ok = group_sync(A, count, G, target, &s_ok);
        bool finished = false;
        while (ok && !finished) {
            // RESID: r = b - A (x64 + d) in FP64 on the chunk
            double v[4] = {0.0, 0.0, 0.0, 0.0};
            for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
                if (!m.g.interior(i)) {
                    rr[i] = 0.0f;
                    continue;
                }
                const double xc = x[i] + (double)dd[i];
                const double nb = ((x[i - 1] + (double)dd[i - 1]) + (x[i + 1] + (double)dd[i + 1])) +
                                  ((x[i - nx] + (double)dd[i - nx]) + (x[i + nx] + (double)dd[i + nx])) +
                                  ((x[i - sxy] + (double)dd[i - sxy]) + (x[i + sxy] + (double)dd[i + sxy]));
                const double bi = (double)bb[i];
                const double ri = bi - (m.cd64 * xc + m.co64 * nb);
                const float rf = (float)ri;
                rr[i] = rf;
                v[0] += ri * ri;
                v[1] += bi * bi;
                v[2] += (double)rf * (double)(rf * m.dinv);
                v[3] += (double)rf * (double)rf;
            }
            if (!(ok = group_sums<4>(A, part, 0, q, G, count, target, v, s_red, s_tot, &s_ok))) break;
            const double bn = sqrt(v[1]) > 0.0 ? sqrt(v[1]) : 1.0;
            const double rel = sqrt(v[0]) / bn;
            s.rel = rel;
            if (!isfinite(rel)) {
                s.status = PIRO_STATUS_STALLED;
                finished = true;
            } else if (rel <= A.rtol) {
                s.status = PIRO_OK;
                finished = true;
            } else if (s.sweep >= A.max_sweeps || s.inner_total >= A.max_inner) {
                s.status = PIRO_ERR_NOT_CONVERGED;
                finished = true;
            } else if (s.sweep > 0 && rel > 0.5 * s.prev_rel) {
                s.status = PIRO_STATUS_STALLED;
                finished = true;
            }
            // the pending correction joins x (read next by the sweep after this one)
            for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
                const double xn = x[i] + (double)dd[i];
                x[i] = xn;
                dd[i] = 0.0f;
                if (finished) oo[i] = (float)xn;
            }
            if (finished || v[3] <= 0.0) {
                if (!finished) {
                    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) oo[i] = (float)x[i];
                    finished = true;
                }
                break;
            }
            double itol = rel > 0.0 ? 0.5 * A.rtol / rel : 1.0;
            itol = itol > 0.1 ? 0.1 : itol;
            itol = itol < A.inner_floor ? A.inner_floor : itol;
            s.tol2 = itol * itol;
            s.rz = v[2];
            s.rr0 = v[3];
            s.beta = 0.0;
            s.it = 0;
            s.prev_rel = rel;
            s.sweep += 1;
            // CG on the correction d
            while (true) {
                // V1: p = z + beta p_old (z = r / A_rr), q = A p, <p, q>
                const float beta = (float)s.beta;
                const float *po = ((s.it & 1) ? A.p1 : A.p0) + m.off;
                float *pn = ((s.it & 1) ? A.p0 : A.p1) + m.off;
                double w[1] = {0.0};
                for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
                    if (!m.g.interior(i)) {
                        pn[i] = 0.0f;
                        qq[i] = 0.0f;
                        continue;
                    }
                    auto pv = [&](int64_t j) { return rr[j] * m.dinv + beta * po[j]; };
                    const float c = pv(i);
                    const float nb = ((pv(i - 1) + pv(i + 1)) + (pv(i - nx) + pv(i + nx))) + (pv(i - sxy) + pv(i + sxy));
                    const float qv = m.cd * c + m.co * nb;
                    pn[i] = c;
                    qq[i] = qv;
                    w[0] += (double)(c * qv);
                }
                if (!(ok = group_sums<1>(A, part, 4, q, G, count, target, w, s_red, s_tot, &s_ok))) break;
                const double a = s.rz / w[0];
                if (!isfinite(a) || w[0] <= 0.0) {
                    // breakdown: the member ends with the correction it has (as k_batch_step's S1)
                    s.status = PIRO_STATUS_STALLED;
                    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
                        const double xn = x[i] + (double)dd[i];
                        x[i] = xn;
                        dd[i] = 0.0f;
                        oo[i] = (float)xn;
                    }
                    finished = true;
                    break;
                }
                // V2: d += a p, r -= a q; <r, z>, |r|^2 (boundary cells carry p = q = r = 0)
                const float fa = (float)a;
                double u2[2] = {0.0, 0.0};
                const int64_t g0 = c0 >> 2, g1 = c1 >> 2;  // c0 % 4 == 0
                for (int64_t gi = g0 + threadIdx.x; gi < g1; gi += blockDim.x) {
                    const float4 p4 = reinterpret_cast<const float4 *>(pn)[gi];
                    const float4 q4 = reinterpret_cast<const float4 *>(qq)[gi];
                    float4 d4 = reinterpret_cast<float4 *>(dd)[gi];
                    float4 r4 = reinterpret_cast<float4 *>(rr)[gi];
                    d4.x += fa * p4.x; d4.y += fa * p4.y; d4.z += fa * p4.z; d4.w += fa * p4.w;
                    r4.x = r4.x - fa * q4.x; r4.y = r4.y - fa * q4.y; r4.z = r4.z - fa * q4.z; r4.w = r4.w - fa * q4.w;
                    reinterpret_cast<float4 *>(dd)[gi] = d4;
                    reinterpret_cast<float4 *>(rr)[gi] = r4;
                    const float r2 = ((r4.x * r4.x + r4.y * r4.y) + (r4.z * r4.z + r4.w * r4.w));
                    u2[0] += (double)(r2 * m.dinv);
                    u2[1] += (double)r2;
                }
                for (int64_t i = (g1 << 2) + threadIdx.x; i < c1; i += blockDim.x) {
                    dd[i] += fa * pn[i];
                    const float ri = rr[i] - fa * qq[i];
                    rr[i] = ri;
                    u2[0] += (double)ri * (double)(ri * m.dinv);
                    u2[1] += (double)ri * (double)ri;
                }
                if (!(ok = group_sums<2>(A, part, 5, q, G, count, target, u2, s_red, s_tot, &s_ok))) break;
                s.it += 1;
                s.inner_total += 1;
                const double beta_n = u2[0] / s.rz;
                if (!isfinite(u2[1]) || !isfinite(beta_n)) {
                    s.status = PIRO_STATUS_STALLED;
                    break;
                }
                if (u2[1] <= s.tol2 * s.rr0 || s.inner_total >= A.max_inner) break;
                s.beta = beta_n;
                s.rz = u2[0];
            }
            // the update's group sum was the barrier: every CTA's d and r are
            // written before the residual reads its neighbours
            if (!ok) break;
        }
        if (q == 0 && threadIdx.x == 0) {
            s.mode = kDone;
            A.st[J.member] = s;
        }
        if (!ok) return;
    }
}

}  // namespace
}  // namespace piro

using namespace piro;

struct piro_batch {
    int M = 0;
    int64_t Ntot = 0;
    std::vector<BMember> mem;
    BMember *d_mem = nullptr;
    int tile = 4096;
    int nfe = 0, nbe = 0;
    int *d_fe_m = nullptr, *d_be_m = nullptr;
    int64_t *d_fe_s = nullptr, *d_be_s = nullptr;
    float *f[2] = {nullptr, nullptr};  // fields: current and next
    int cur = 0;
    float *b = nullptr, *r = nullptr, *p0 = nullptr, *p1 = nullptr, *q = nullptr, *d = nullptr;
    double *x64 = nullptr, *partials = nullptr;
    BState *st = nullptr;
    BarrierState *bar = nullptr;
    cudaStream_t stream = nullptr;
    unsigned grid = 0;
    int blocks_per_sm = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t own = nullptr;      // non-blocking stream for graph capture
    cudaGraphExec_t pair = nullptr;  // two steps (f[0] -> f[1] -> f[0]) as one graph
    double pair_rtol = 0.0;
    long long pair_spin = -1;  // the wait limit the pair graph was captured with
    double step_ms = 0.0;
    long long steps = 0;
    double rtol = 1e-8;
    // the grouped step (k_batch_groups): used when grouped = 1
    int grouped = 0;
    unsigned grid_g = 0;
    int njobs = 0;
    BJob *d_jobs = nullptr;
    int *d_cta_ptr = nullptr, *d_cta_jobs = nullptr;
    unsigned *d_job_bar = nullptr;
    double *d_job_part = nullptr;
};

static void batch_free_groups(piro_batch *s)
{
    cudaFree(s->d_jobs);
    cudaFree(s->d_cta_ptr);
    cudaFree(s->d_cta_jobs);
    cudaFree(s->d_job_bar);
    cudaFree(s->d_job_part);
    s->d_jobs = nullptr;
    s->d_cta_ptr = s->d_cta_jobs = nullptr;
    s->d_job_bar = nullptr;
    s->d_job_part = nullptr;
    s->njobs = 0;
    s->grid_g = 0;
}

// Jobs of the grouped step for a grid of sm_count * blocks_per_sm CTAs: with
// T the backward-Euler cells per CTA on average, a member of at least 2T
// cells gets floor(cells / T) CTAs of its own (T grows until the groups
// leave a CTA for the small members); the others go, largest first, to the
// least loaded of the remaining CTAs.
static int batch_groups_setup(piro_batch *s, int blocks_per_sm)
{
    batch_free_groups(s);
    int per_sm = 0;
    PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_groups, kThreads, 0));
    if (per_sm < 1) {
        set_error("piro_batch: the grouped step cannot be resident");
        return PIRO_ERR_CUDA;
    }
    const int C = sm_count() * std::min(per_sm, blocks_per_sm);
    std::vector<int> be;
    double total = 0.0;
    for (int k = 0; k < s->M; ++k)
        if (s->mem[k].scheme == 1) {
            be.push_back(k);
            total += (double)s->mem[k].N;
        }
    std::sort(be.begin(), be.end(), [&](int a, int b) { return s->mem[a].N > s->mem[b].N || (s->mem[a].N == s->mem[b].N && a < b); });
    double T = std::max(total / C, 1.0);
    std::vector<int> gsz(be.size(), 1);
    for (int guard = 0; guard < 64; ++guard) {
        int used = 0, small = 0;
        for (size_t i = 0; i < be.size(); ++i) {
            const int g = (int)std::floor((double)s->mem[be[i]].N / T);
            gsz[i] = g >= 2 ? g : 1;
            if (gsz[i] > 1) used += gsz[i];
            else ++small;
        }
        if (used + (small > 0 ? 1 : 0) <= C) break;
        T *= 1.25;
    }
    std::vector<BJob> jobs;
    std::vector<std::vector<int>> cta(C);
    int next = 0, part = 0;
    for (size_t i = 0; i < be.size(); ++i) {
        if (gsz[i] < 2) continue;
        BJob J{be[i], next, gsz[i], part};
        for (int c = next; c < next + gsz[i]; ++c) cta[c].push_back((int)jobs.size());
        jobs.push_back(J);
        next += gsz[i];
        part += 7 * gsz[i];
    }
    std::vector<double> load(C, 0.0);
    for (size_t i = 0; i < be.size(); ++i) {
        if (gsz[i] >= 2) continue;
        int best = next;
        for (int c = next + 1; c < C; ++c)
            if (load[c] < load[best]) best = c;
        BJob J{be[i], best, 1, part};
        cta[best].push_back((int)jobs.size());
        jobs.push_back(J);
        load[best] += (double)s->mem[be[i]].N;
        part += 7;
    }
    std::vector<int> ptr(C + 1, 0), list;
    for (int c = 0; c < C; ++c) {
        ptr[c] = (int)list.size();
        list.insert(list.end(), cta[c].begin(), cta[c].end());
    }
    ptr[C] = (int)list.size();
    auto up = [](void **dst, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, bytes > 0 ? bytes : 8);
        if (e == cudaSuccess && bytes > 0) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    cudaError_t e = up((void **)&s->d_jobs, jobs.data(), jobs.size() * sizeof(BJob));
    if (e == cudaSuccess) e = up((void **)&s->d_cta_ptr, ptr.data(), ptr.size() * sizeof(int));
    if (e == cudaSuccess) e = up((void **)&s->d_cta_jobs, list.data(), list.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_job_bar, sizeof(unsigned) * std::max<size_t>(1, jobs.size()));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_job_part, sizeof(double) * std::max(1, part));
    if (e != cudaSuccess) {
        batch_free_groups(s);
        set_error("piro_batch: grouped step setup failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    s->njobs = (int)jobs.size();
    s->grid_g = (unsigned)C;
    return PIRO_OK;
}

static void batch_drop_graph(piro_batch *s)
{
    if (s->pair) cudaGraphExecDestroy(s->pair);
    s->pair = nullptr;
}

static void batch_free_tiles(piro_batch *s)
{
    batch_drop_graph(s);
    cudaFree(s->d_fe_m);
    cudaFree(s->d_be_m);
    cudaFree(s->d_fe_s);
    cudaFree(s->d_be_s);
    cudaFree(s->partials);
    s->d_fe_m = s->d_be_m = nullptr;
    s->d_fe_s = s->d_be_s = nullptr;
    s->partials = nullptr;
}

// Cut the members into tiles of `tile` cells and size the cooperative grid.
// The k_batch_step instance for a launch of blocks_per_sm blocks per SM.
static const void *batch_kernel(int blocks_per_sm)
{
    if (blocks_per_sm >= 8) return (const void *)k_batch_step<8>;
    if (blocks_per_sm >= 6) return (const void *)k_batch_step<6>;
    return (const void *)k_batch_step<4>;
}

static int batch_tiles(piro_batch *s, int tile, int blocks_per_sm)
{
    batch_free_tiles(s);
    std::vector<int> fm, bm;
    std::vector<int64_t> fs, bsv;
    for (int k = 0; k < s->M; ++k) {
        BMember &m = s->mem[k];
        const int nt = (int)cdiv(m.N, tile);
        if (m.scheme == 1) {
            m.tile0 = (int)bm.size();
            m.ntiles = nt;
        } else {
            m.tile0 = 0;
            m.ntiles = 0;
        }
        for (int t = 0; t < nt; ++t) {
            if (m.scheme == 1) {
                bm.push_back(k);
                bsv.push_back((int64_t)t * tile);
            } else {
                fm.push_back(k);
                fs.push_back((int64_t)t * tile);
            }
        }
    }
    s->tile = tile;
    s->nfe = (int)fm.size();
    s->nbe = (int)bm.size();
    auto up = [](void **dst, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, bytes > 0 ? bytes : 8);
        if (e == cudaSuccess && bytes > 0) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
        return e;
    };
    cudaError_t e = up((void **)&s->d_fe_m, fm.data(), fm.size() * sizeof(int));
    if (e == cudaSuccess) e = up((void **)&s->d_fe_s, fs.data(), fs.size() * sizeof(int64_t));
    if (e == cudaSuccess) e = up((void **)&s->d_be_m, bm.data(), bm.size() * sizeof(int));
    if (e == cudaSuccess) e = up((void **)&s->d_be_s, bsv.data(), bsv.size() * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&s->partials, sizeof(double) * 4 * (size_t)std::max(1, s->nbe));
    if (e == cudaSuccess) e = cudaMemcpy(s->d_mem, s->mem.data(), sizeof(BMember) * s->M, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error("piro_batch: tile setup failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    int dev = 0, per_sm = 0, coop = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    PIRO_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel(blocks_per_sm), kThreads, 0));
    if (!coop || per_sm < 1) {
        set_error("piro_batch: cooperative launch is not available");
        return PIRO_ERR_CUDA;
    }
    const int bps = std::min(per_sm, blocks_per_sm);
    s->blocks_per_sm = bps;
    s->grid = (unsigned)(sm_count() * bps);
    return PIRO_OK;
}

extern "C" int piro_batch_create(int count, const int *n, const float *alpha, const float *dt, const int *scheme,
                                 piro_stream_t stream, piro_batch **out)
{
    PIRO_ARG(out && count > 0 && n && alpha && dt && scheme, "piro_batch_create: bad arguments");
    *out = nullptr;
    piro_batch *s = new piro_batch();
    s->M = count;
    s->mem.resize(count);
    int64_t off = 0;
    for (int k = 0; k < count; ++k) {
        if (n[k] < 3 || (int64_t)n[k] * n[k] * n[k] >= ((int64_t)1 << 31) || (scheme[k] != 0 && scheme[k] != 1) ||
            !(alpha[k] > 0.0f) || !(dt[k] > 0.0f)) {
            delete s;
            set_error("piro_batch_create: member %d: bad size, scheme, alpha or dt", k);
            return PIRO_ERR_ARG;
        }
        BMember &m = s->mem[k];
        m.g = GridDiv(n[k], n[k], n[k]);
        m.N = (int64_t)n[k] * n[k] * n[k];
        m.off = off;
        off += cdiv(m.N, 64) * 64;  // 256-byte aligned members
        m.alpha = alpha[k];
        m.dt = dt[k];
        m.scheme = scheme[k];
        // A = I - dt*alpha*L (h = 1): FP32 coefficients as the single-grid
        // stencil solver forms them, FP64 ones for the residual
        volatile float a6 = alpha[k] * -6.0f;  // one rounding per operation, no contraction
        volatile float t6 = -dt[k] * a6;
        m.cd = 1.0f + t6;
        volatile float a1 = alpha[k] * 1.0f;
        m.co = -dt[k] * a1;
        m.dinv = 1.0f / m.cd;
        m.cd64 = 1.0 + 6.0 * (double)dt[k] * (double)alpha[k];
        m.co64 = -(double)dt[k] * (double)alpha[k];
    }
    s->Ntot = off;
    const size_t N = (size_t)off;
    s->stream = as_stream(stream);
    cudaError_t e = cudaMalloc(&s->d_mem, sizeof(BMember) * count);
    if (e == cudaSuccess) e = cudaMalloc(&s->f[0], N * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->f[1], N * sizeof(float));
    for (float **p : {&s->b, &s->r, &s->p0, &s->p1, &s->q, &s->d})
        if (e == cudaSuccess) e = cudaMalloc(p, N * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->x64, N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->st, sizeof(BState) * count);
    if (e == cudaSuccess) e = cudaMalloc(&s->bar, sizeof(BarrierState));
    if (e == cudaSuccess) e = cudaMemset(s->bar, 0, sizeof(BarrierState));
    for (float *p : {s->f[0], s->f[1], s->b, s->r, s->p0, s->p1, s->q, s->d})
        if (e == cudaSuccess) e = cudaMemset(p, 0, N * sizeof(float));
    if (e == cudaSuccess) e = cudaEventCreate(&s->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->e1);
    if (e != cudaSuccess) {
        piro_batch_destroy(s);
        set_error("piro_batch_create: allocation failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_NOMEM;
    }
    int rc = batch_tiles(s, 4096, 2);
    if (rc) {
        piro_batch_destroy(s);
        return rc;
    }
    *out = s;
    return PIRO_OK;
}

extern "C" int piro_batch_layout(piro_batch *s, int64_t *offsets, int64_t *total_cells)
{
    PIRO_ARG(s, "piro_batch_layout: bad arguments");
    if (offsets)
        for (int k = 0; k < s->M; ++k) offsets[k] = s->mem[k].off;
    if (total_cells) *total_cells = s->Ntot;
    return PIRO_OK;
}

extern "C" int piro_batch_set_fields(piro_batch *s, const float *u, int from_host)
{
    PIRO_ARG(s && u, "piro_batch_set_fields: bad arguments");
    PIRO_CUDA(cudaMemcpyAsync(s->f[s->cur], u, sizeof(float) * (size_t)s->Ntot,
                              from_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s->stream));
    PIRO_CUDA(cudaStreamSynchronize(s->stream));
    return PIRO_OK;
}

extern "C" int piro_batch_get_fields(piro_batch *s, float *u, int to_host)
{
    PIRO_ARG(s && u, "piro_batch_get_fields: bad arguments");
    PIRO_CUDA(cudaMemcpyAsync(u, s->f[s->cur], sizeof(float) * (size_t)s->Ntot,
                              to_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s->stream));
    PIRO_CUDA(cudaStreamSynchronize(s->stream));
    return PIRO_OK;
}

extern "C" int piro_batch_field_ptr(piro_batch *s, float **u)
{
    PIRO_ARG(s && u, "piro_batch_field_ptr: bad arguments");
    *u = s->f[s->cur];
    return PIRO_OK;
}

static int batch_launch_groups(piro_batch *s, const float *u, float *out, cudaStream_t st)
{
    GArgs A;
    A.mem = s->d_mem;
    A.fe_tile_m = s->d_fe_m;
    A.fe_tile_s = s->d_fe_s;
    A.nfe = s->nfe;
    A.tile = s->tile;
    A.jobs = s->d_jobs;
    A.cta_ptr = s->d_cta_ptr;
    A.cta_jobs = s->d_cta_jobs;
    A.job_bar = s->d_job_bar;
    A.job_part = s->d_job_part;
    A.u = u;
    A.out = out;
    A.b = s->b;
    A.r = s->r;
    A.p0 = s->p0;
    A.p1 = s->p1;
    A.q = s->q;
    A.d = s->d;
    A.x64 = s->x64;
    A.st = s->st;
    A.bar = s->bar;
    A.rtol = s->rtol;
    A.inner_floor = 1e-6;
    A.max_sweeps = 20;
    A.max_inner = 20000;
    A.spin_limit = wait_limit(1ll << 22);  // ~2 s of polling per barrier wait
    void *args[] = {&A};
    PIRO_CUDA(cudaMemsetAsync(s->bar, 0, sizeof(BarrierState), st));
    PIRO_CUDA(cudaMemsetAsync(s->d_job_bar, 0, sizeof(unsigned) * (size_t)std::max(1, s->njobs), st));
    PIRO_CUDA(cudaLaunchCooperativeKernel((const void *)k_batch_groups, dim3(s->grid_g), dim3(kThreads), args, 0, st));
    return PIRO_OK;
}

static int batch_launch(piro_batch *s, const float *u, float *out, cudaStream_t st)
{
    if (s->grouped) return batch_launch_groups(s, u, out, st);
    BArgs A;
    A.mem = s->d_mem;
    A.M = s->M;
    A.fe_tile_m = s->d_fe_m;
    A.be_tile_m = s->d_be_m;
    A.fe_tile_s = s->d_fe_s;
    A.be_tile_s = s->d_be_s;
    A.nfe = s->nfe;
    A.nbe = s->nbe;
    A.tile = s->tile;
    A.u = u;
    A.out = out;
    A.b = s->b;
    A.r = s->r;
    A.p0 = s->p0;
    A.p1 = s->p1;
    A.q = s->q;
    A.d = s->d;
    A.x64 = s->x64;
    A.partials = s->partials;
    A.st = s->st;
    A.bar = s->bar;
    A.rtol = s->rtol;
    A.inner_floor = 1e-6;
    A.max_sweeps = 20;
    A.max_inner = 20000;
    A.max_rounds = 40000;
    A.spin_limit = wait_limit(1ll << 22);  // ~2 s of polling per barrier wait
    void *args[] = {&A};
    // a launch whose barrier wait gave up leaves count, gen and err behind
    PIRO_CUDA(cudaMemsetAsync(s->bar, 0, sizeof(BarrierState), st));
    PIRO_CUDA(cudaLaunchCooperativeKernel(batch_kernel(s->blocks_per_sm), dim3(s->grid), dim3(kThreads), args, 0, st));
    return PIRO_OK;
}

// Two steps, f[0] -> f[1] -> f[0], captured once as a CUDA graph (two
// cooperative kernel nodes) and replayed; re-captured when the tiling or the
// tolerance changes.
static int batch_pair_graph(piro_batch *s)
{
    if (s->pair && s->pair_rtol == s->rtol && s->pair_spin == wait_limit(1ll << 22)) return PIRO_OK;
    batch_drop_graph(s);
    if (!s->own) PIRO_CUDA(cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking));
    PIRO_CUDA(cudaStreamBeginCapture(s->own, cudaStreamCaptureModeThreadLocal));
    int rc = batch_launch(s, s->f[0], s->f[1], s->own);
    if (!rc) rc = batch_launch(s, s->f[1], s->f[0], s->own);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->own, &g);
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        set_error("piro_batch: graph capture of the step failed");
        return rc ? rc : PIRO_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&s->pair, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        s->pair = nullptr;
        set_error("piro_batch: graph instantiation failed: %s", cudaGetErrorString(ei));
        return PIRO_ERR_CUDA;
    }
    s->pair_rtol = s->rtol;
    s->pair_spin = wait_limit(1ll << 22);
    return PIRO_OK;
}

extern "C" int piro_batch_step(piro_batch *s, int steps, double rtol, double *ms)
{
    PIRO_ARG(s && steps >= 0 && rtol > 0.0, "piro_batch_step: bad arguments");
    s->rtol = rtol;
    int k = 0;
    if (steps >= 2) {
        int rc = batch_pair_graph(s);
        if (rc) return rc;
    }
    PIRO_CUDA(cudaEventRecord(s->e0, s->stream));
    if (s->cur == 1 && k < steps) {  // realign to f[0] so the pair graph applies
        int rc = batch_launch(s, s->f[1], s->f[0], s->stream);
        if (rc) return rc;
        s->cur = 0;
        ++k;
    }
    for (; k + 2 <= steps; k += 2) PIRO_CUDA(cudaGraphLaunch(s->pair, s->stream));
    if (k < steps) {
        int rc = batch_launch(s, s->f[0], s->f[1], s->stream);
        if (rc) return rc;
        s->cur = 1;
    }
    PIRO_CUDA(cudaEventRecord(s->e1, s->stream));
    PIRO_CUDA(cudaStreamSynchronize(s->stream));
    BarrierState hb;
    PIRO_CUDA(cudaMemcpy(&hb, s->bar, sizeof(hb), cudaMemcpyDeviceToHost));
    if (hb.err) {
        set_error("piro_batch_step: grid barrier timed out");
        return PIRO_ERR_CUDA;
    }
    float t = 0.0f;
    PIRO_CUDA(cudaEventElapsedTime(&t, s->e0, s->e1));
    s->step_ms += t;
    s->steps += steps;
    if (ms) *ms = t;
    return PIRO_OK;
}

extern "C" int piro_batch_member_info(piro_batch *s, int *status, int *sweeps, int *inner, double *rel)
{
    PIRO_ARG(s, "piro_batch_member_info: bad arguments");
    std::vector<BState> h(s->M);
    PIRO_CUDA(cudaMemcpy(h.data(), s->st, sizeof(BState) * s->M, cudaMemcpyDeviceToHost));
    for (int k = 0; k < s->M; ++k) {
        if (status) status[k] = h[k].status;
        if (sweeps) sweeps[k] = h[k].sweep;
        if (inner) inner[k] = h[k].inner_total;
        if (rel) rel[k] = s->mem[k].scheme == 1 ? h[k].rel : 0.0;
    }
    return PIRO_OK;
}

// Autotuner: time one step (from the current fields, result discarded) for
// each tile size and blocks-per-SM candidate of the lockstep step and for the
// grouped step at 2 and 4 CTAs per SM, and keep the fastest.
extern "C" int piro_batch_autotune(piro_batch *s, double rtol, int *tile_out, int *blocks_per_sm_out)
{
    PIRO_ARG(s && rtol > 0.0, "piro_batch_autotune: bad arguments");
    s->rtol = rtol;
    s->grouped = 0;  // the lockstep candidates first
    const int tiles[] = {2048, 4096, 8192, 16384};
    const int bps[] = {1, 2, 4, 6, 8};
    double best = INFINITY;
    int bt = s->tile, bb = s->blocks_per_sm;
    for (int t : tiles)
        for (int b : bps) {
            int rc = batch_tiles(s, t, b);
            if (rc) return rc;
            if (s->blocks_per_sm != b) continue;  // occupancy does not allow it
            float ms = INFINITY;
            for (int rep = 0; rep < 2; ++rep) {  // second run timed
                PIRO_CUDA(cudaEventRecord(s->e0, s->stream));
                rc = batch_launch(s, s->f[s->cur], s->f[s->cur ^ 1], s->stream);
                if (rc) return rc;
                PIRO_CUDA(cudaEventRecord(s->e1, s->stream));
                PIRO_CUDA(cudaStreamSynchronize(s->stream));
                PIRO_CUDA(cudaEventElapsedTime(&ms, s->e0, s->e1));
            }
            if (ms < best) {
                best = ms;
                bt = t;
                bb = b;
            }
        }
    // the grouped step (FE tiles of the best tiling), 2 or 4 CTAs per SM
    int rc = batch_tiles(s, bt, bb);
    if (rc) return rc;
    int bg = 0;
    for (int b : {2, 4}) {
        rc = batch_groups_setup(s, b);
        if (rc) return rc;
        s->grouped = 1;
        float ms = INFINITY;
        for (int rep = 0; rep < 2; ++rep) {
            PIRO_CUDA(cudaEventRecord(s->e0, s->stream));
            rc = batch_launch(s, s->f[s->cur], s->f[s->cur ^ 1], s->stream);
            if (rc) {
                s->grouped = 0;
                return rc;
            }
            PIRO_CUDA(cudaEventRecord(s->e1, s->stream));
            PIRO_CUDA(cudaStreamSynchronize(s->stream));
            PIRO_CUDA(cudaEventElapsedTime(&ms, s->e0, s->e1));
        }
        s->grouped = 0;
        if (ms < best) {
            best = ms;
            bg = b;
        }
    }
    if (bg) {
        rc = batch_groups_setup(s, bg);
        if (rc) return rc;
        s->grouped = 1;
        bb = bg;
    } else {
        batch_free_groups(s);
    }
    batch_drop_graph(s);
    if (tile_out) *tile_out = bt;
    if (blocks_per_sm_out) *blocks_per_sm_out = bb;
    return PIRO_OK;
}

extern "C" int piro_batch_schedule(piro_batch *s, int *grouped)
{
    PIRO_ARG(s && grouped, "piro_batch_schedule: bad arguments");
    *grouped = s->grouped;
    return PIRO_OK;
}

extern "C" int piro_batch_set_schedule(piro_batch *s, int grouped, int blocks_per_sm)
{
    PIRO_ARG(s && (grouped == 0 || grouped == 1) && blocks_per_sm >= 1, "piro_batch_set_schedule: bad arguments");
    batch_drop_graph(s);
    if (grouped) {
        int rc = batch_groups_setup(s, blocks_per_sm);
        if (rc) return rc;
    } else {
        int rc = batch_tiles(s, s->tile, blocks_per_sm);
        if (rc) return rc;
        batch_free_groups(s);
    }
    s->grouped = grouped;
    return PIRO_OK;
}

extern "C" int piro_batch_destroy(piro_batch *s)
{
    if (!s) return PIRO_OK;
    batch_free_groups(s);
    batch_free_tiles(s);
    cudaFree(s->d_mem);
    cudaFree(s->f[0]);
    cudaFree(s->f[1]);
    for (float *p : {s->b, s->r, s->p0, s->p1, s->q, s->d}) cudaFree(p);
    cudaFree(s->x64);
    cudaFree(s->st);
    cudaFree(s->bar);
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    if (s->own) cudaStreamDestroy(s->own);
    delete s;
    return PIRO_OK;
}

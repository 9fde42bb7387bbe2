// slab.cu -- z-slab domain decomposition of one grid over ranks: the kernels
// of the backward-Euler solve on one slab (FP64 residual, FP32 CG steps,
// refinement update) for A = I - dt*diag(alpha)*L with the central 7-point L.
//
// Slab layout: a rank owns grid planes [z0, z1); its arrays hold planes
// z0-1 .. z1 (one halo plane each side, nz_l = z1 - z0 + 2 planes; the halo
// below plane 0 and above plane nz-1 of the grid is never read by an owned
// interior row).  Local cell l is grid cell l + (z0 - 1)*nx*ny.  The host
// exchanges halo planes (z before each CG operator apply, x64 after each
// refinement update) and all-reduces the FP64 partial sums each kernel
// returns; these kernels only touch owned cells (and, for p, the halo planes,
// which every rank forms identically from the exchanged z).
//
// Coefficients per cell are the FP32 values csrgeam2 gives the assembled A
// (diagonal fl(1 + fl(-dt*fl(alpha*vself))), off-diagonal fl(-dt*fl(alpha*vnb)))
// promoted to FP64 for the residual, as the single-grid solver's CSR residual.
// Couplings to boundary cells use the stencil value (PIRO's 10.0 entries,
// stencils.cpp:278-291, only meet nonzero boundary values).
#include <algorithm>

#include "common.cuh"

namespace piro {
namespace {

constexpr int kSlabThreads = 256;
constexpr int kSlabBlocks = 1184;  // at most 8 per SM on a 148-SM part: per-block partial sums

struct Slab {
    GridDiv g;           // the whole grid
    int64_t lbase;       // grid index of local cell 0: (z0 - 1) * nx * ny (may be negative)
    int64_t own0, own1;  // local cell range of the owned planes
    float mdt, vself, vnb;
};

__device__ __forceinline__ void coef(const Slab &S, float a, float &cd, float &co)
{
    cd = __fadd_rn(1.0f, __fmul_rn(S.mdt, __fmul_rn(a, S.vself)));
    co = __fmul_rn(S.mdt, __fmul_rn(a, S.vnb));
}

// Block sums of nvals values into out[k * gridDim.x + blockIdx.x].
__device__ __forceinline__ void block_partials(double *out, int nvals, const double (&v)[4])
{
    __shared__ double s_w[4][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < nvals; ++k) {
        const double t = warp_sum(v[k]);
        if (lane == 0) s_w[k][w] = t;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        for (int k = 0; k < nvals; ++k) {
            double t = threadIdx.x < (blockDim.x >> 5) ? s_w[k][threadIdx.x] : 0.0;
            t = warp_sum(t);
            if (threadIdx.x == 0) out[(int64_t)k * gridDim.x + blockIdx.x] = t;
        }
    }
}

// r = b - A x64 (FP64) and z = r / A_rr on owned interior cells, 0 on the
// owned boundary; partials: |r64|^2, |b|^2, <r/alpha, z>, |r32|^2.
__global__ void __launch_bounds__(kSlabThreads) k_slab_residual(Slab S, const float *__restrict__ alpha,
                                                                const float *__restrict__ b,
                                                                const double *__restrict__ x, float *__restrict__ r,
                                                                float *__restrict__ z, double *__restrict__ part)
{
    const int64_t sxy = (int64_t)S.g.nx * S.g.ny;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t l = S.own0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < S.own1;
         l += (int64_t)gridDim.x * blockDim.x) {
        if (!S.g.interior(l + S.lbase)) {
            r[l] = 0.0f;
            z[l] = 0.0f;
            continue;
        }
        const float a = alpha[l];
        float cd, co;
        coef(S, a, cd, co);
        const int nx = S.g.nx;
        const double nb = ((x[l - 1] + x[l + 1]) + (x[l - nx] + x[l + nx])) + (x[l - sxy] + x[l + sxy]);
        const double bi = (double)b[l];
        const double ri = bi - ((double)cd * x[l] + (double)co * nb);
        const float rf = (float)ri;
        const float zf = rf / cd;
        r[l] = rf;
        z[l] = zf;
        v[0] += ri * ri;
        v[1] += bi * bi;
        v[2] += (double)rf / (double)a * (double)zf;
        v[3] += (double)rf * (double)rf;
    }
    block_partials(part, 4, v);
}

// Device-resident CG scalars of one slab solve (state[kSlabStateLen], the
// same on every rank since it is formed from all-reduced sums):
enum : int {
    kStRz = 0,    // <r/alpha, z> of the current iterate
    kStBeta = 1,  // direction update of the next iteration
    kStA = 2,     // step length of the last iteration
    kStStop = 3,  // inner stop: |r|^2 <= this (tol2 * rr0)
    kStDone = 4,  // nonzero: the inner solve has stopped (steps are no-ops)
    kStIters = 5, // iterations taken
    kStRr = 6,    // |r|^2 after the last iteration
    kStBroken = 7 // nonzero: a non-finite or non-positive scalar appeared
};

// p = z + beta*p_old on interior cells of the owned and halo planes (0 on the
// boundary); q = A p on owned interior cells; partial <p, q/alpha>.  With a
// device state, beta comes from it and a finished solve returns at once.
__global__ void __launch_bounds__(kSlabThreads, 4) k_slab_cg_spmv(Slab S, float beta, const double *__restrict__ state,
                                                               const float *__restrict__ alpha,
                                                               const float *__restrict__ z,
                                                               const float *__restrict__ p_old,
                                                               float *__restrict__ p_new, float *__restrict__ q,
                                                               double *__restrict__ part)
{
    if (state) {
        if (state[kStDone] != 0.0) return;
        beta = (float)state[kStBeta];
    }
    const int64_t sxy = (int64_t)S.g.nx * S.g.ny;
    const int64_t N = sxy * S.g.nz;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int64_t lo = max(S.own0 - sxy, -S.lbase), hi = min(S.own1 + sxy, N - S.lbase);
    const int nx = S.g.nx;
    const bool vec = (nx & 3) == 0 && ((lo | hi | S.own0 | S.own1 | S.lbase) & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(alpha) | reinterpret_cast<uintptr_t>(z) |
                       reinterpret_cast<uintptr_t>(p_old) | reinterpret_cast<uintptr_t>(p_new) |
                       reinterpret_cast<uintptr_t>(q)) & 15) == 0;
    if (vec) {
        // groups of 4 x-adjacent cells (nx % 4 == 0: a group never leaves its
        // x-row): z and p_old at the group and its y/z neighbours as 16-byte
        // loads, the x halo as two scalars; the same arithmetic per cell
        const float4 *Z = reinterpret_cast<const float4 *>(z), *Po = reinterpret_cast<const float4 *>(p_old);
        const int64_t rx = nx >> 2, rxy = sxy >> 2;
        for (int64_t g4 = (lo >> 2) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g4 < (hi >> 2);
             g4 += (int64_t)gridDim.x * blockDim.x) {
            const int64_t l = g4 << 2;
            int x0, y, zc;
            S.g.coords((uint32_t)(l + S.lbase), x0, y, zc);
            const bool yz = y > 0 && y < S.g.ny - 1 && zc > 0 && zc < S.g.nz - 1;
            bool in[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) in[k] = yz && x0 + k > 0 && x0 + k < nx - 1;
            const float4 zc4 = Z[g4], pc4 = Po[g4];
            const float zz[4] = {zc4.x, zc4.y, zc4.z, zc4.w}, pp[4] = {pc4.x, pc4.y, pc4.z, pc4.w};
            float pc[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) pc[k] = in[k] ? zz[k] + beta * pp[k] : 0.0f;
            reinterpret_cast<float4 *>(p_new)[g4] = make_float4(pc[0], pc[1], pc[2], pc[3]);
            if (l < S.own0 || l >= S.own1 || !(in[0] || in[1] || in[2] || in[3])) continue;
            auto vp = [&](float4 a4, float4 b4, int k) {
                const float za[4] = {a4.x, a4.y, a4.z, a4.w}, pb[4] = {b4.x, b4.y, b4.z, b4.w};
                return za[k] + beta * pb[k];
            };
            const float4 zym = Z[g4 - rx], pym = Po[g4 - rx], zyp = Z[g4 + rx], pyp = Po[g4 + rx];
            const float4 zzm = Z[g4 - rxy], pzm = Po[g4 - rxy], zzp = Z[g4 + rxy], pzp = Po[g4 + rxy];
            const float xl = x0 > 1 ? z[l - 1] + beta * p_old[l - 1] : 0.0f;
            const float xr = x0 + 4 < nx - 1 ? z[l + 4] + beta * p_old[l + 4] : 0.0f;
            const float4 al4 = reinterpret_cast<const float4 *>(alpha)[g4];
            const float al[4] = {al4.x, al4.y, al4.z, al4.w};
            float qo[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                qo[k] = 0.0f;
                if (!in[k]) continue;
                const float xm = k > 0 ? pc[k - 1] : xl, xp = k < 3 ? pc[k + 1] : xr;
                const float ym = y > 1 ? vp(zym, pym, k) : 0.0f, yp = y < S.g.ny - 2 ? vp(zyp, pyp, k) : 0.0f;
                const float zm = zc > 1 ? vp(zzm, pzm, k) : 0.0f, zp = zc < S.g.nz - 2 ? vp(zzp, pzp, k) : 0.0f;
                float cd, co;
                coef(S, al[k], cd, co);
                qo[k] = cd * pc[k] + co * (((xm + xp) + (ym + yp)) + (zm + zp));
                v[0] += (double)(pc[k] * qo[k] * rcp_approx(al[k]));  // FP32 term, FP64 sum
            }
            reinterpret_cast<float4 *>(q)[g4] = make_float4(qo[0], qo[1], qo[2], qo[3]);
        }
        block_partials(part, 1, v);
        return;
    }
    for (int64_t l = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < hi;
         l += (int64_t)gridDim.x * blockDim.x) {
        int x, y, zc;
        S.g.coords((uint32_t)(l + S.lbase), x, y, zc);
        const bool in = x > 0 && x < S.g.nx - 1 && y > 0 && y < S.g.ny - 1 && zc > 0 && zc < S.g.nz - 1;
        const float pc = in ? z[l] + beta * p_old[l] : 0.0f;
        p_new[l] = pc;
        if (!in || l < S.own0 || l >= S.own1) continue;
        // neighbours' p formed from z and p_old (p_new of other threads is not read);
        // the cell is interior, so a neighbour is interior when its one moved
        // coordinate is
        auto pv = [&](int64_t j, bool nin) { return nin ? z[j] + beta * p_old[j] : 0.0f; };
        const float a = alpha[l];
        float cd, co;
        coef(S, a, cd, co);
        const float qv =
            cd * pc + co * (((pv(l - 1, x > 1) + pv(l + 1, x < nx - 2)) +
                             (pv(l - nx, y > 1) + pv(l + nx, y < S.g.ny - 2))) +
                            (pv(l - sxy, zc > 1) + pv(l + sxy, zc < S.g.nz - 2)));
        q[l] = qv;
        v[0] += (double)(pc * qv * rcp_approx(a));
    }
    block_partials(part, 1, v);
}

// d += a p, r -= a q, z = r / A_rr on owned interior cells; partials
// <r/alpha, z>, |r|^2.  With a device state, a = rz / <p, S p> (pq: the
// all-reduced sum of the operator step) and a finished or broken-down solve
// returns at once.
__global__ void __launch_bounds__(kSlabThreads) k_slab_cg_update(Slab S, float a, const double *__restrict__ state,
                                                                 const double *__restrict__ pq,
                                                                 const float *__restrict__ alpha,
                                                                 const float *__restrict__ p,
                                                                 const float *__restrict__ q, float *__restrict__ d,
                                                                 float *__restrict__ r, float *__restrict__ z,
                                                                 double *__restrict__ part)
{
    if (state) {
        if (state[kStDone] != 0.0) return;
        const double ad = state[kStRz] / pq[0];
        if (!isfinite(ad) || !(pq[0] > 0.0)) return;  // k_slab_cg_scalars records the breakdown
        a = (float)ad;
    }
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    auto one = [&](float al, float pv, float qv, float &dv, float &rv, float &zv) {
        float cd, co;
        coef(S, al, cd, co);
        dv += a * pv;
        rv = rv - a * qv;
        zv = rv / cd;
        v[0] += (double)(rv * zv * rcp_approx(al));
        v[1] += (double)(rv * rv);
    };
    const bool vec = ((S.own0 | S.own1) & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(alpha) | reinterpret_cast<uintptr_t>(p) |
                       reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(d) |
                       reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(z)) & 15) == 0;
    if (vec) {
        // groups of 4 cells, all five inputs (and z, kept where the cell is not
        // interior) as 16-byte loads: four times the bytes in flight per thread
        for (int64_t g4 = (S.own0 >> 2) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g4 < (S.own1 >> 2);
             g4 += (int64_t)gridDim.x * blockDim.x) {
            const float4 al = reinterpret_cast<const float4 *>(alpha)[g4];
            const float4 pv = reinterpret_cast<const float4 *>(p)[g4];
            const float4 qv = reinterpret_cast<const float4 *>(q)[g4];
            float4 dv = reinterpret_cast<float4 *>(d)[g4];
            float4 rv = reinterpret_cast<float4 *>(r)[g4];
            float4 zv = reinterpret_cast<float4 *>(z)[g4];
            const int64_t l = g4 << 2;
            if (S.g.interior(l + S.lbase)) one(al.x, pv.x, qv.x, dv.x, rv.x, zv.x);
            if (S.g.interior(l + 1 + S.lbase)) one(al.y, pv.y, qv.y, dv.y, rv.y, zv.y);
            if (S.g.interior(l + 2 + S.lbase)) one(al.z, pv.z, qv.z, dv.z, rv.z, zv.z);
            if (S.g.interior(l + 3 + S.lbase)) one(al.w, pv.w, qv.w, dv.w, rv.w, zv.w);
            reinterpret_cast<float4 *>(d)[g4] = dv;
            reinterpret_cast<float4 *>(r)[g4] = rv;
            reinterpret_cast<float4 *>(z)[g4] = zv;
        }
    } else {
        for (int64_t l = S.own0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < S.own1;
             l += (int64_t)gridDim.x * blockDim.x) {
            if (!S.g.interior(l + S.lbase)) continue;
            float dv = d[l], rv = r[l], zv;
            one(alpha[l], p[l], q[l], dv, rv, zv);
            d[l] = dv;
            r[l] = rv;
            z[l] = zv;
        }
    }
    block_partials(part, 2, v);
}

// One CG iteration's scalars from its all-reduced sums (one thread): a =
// rz / pq, then beta = rz' / rz, rz = rz' from up = {rz', |r|^2}; the stop
// and breakdown tests set done.
__global__ void k_slab_cg_scalars(double *__restrict__ st, const double *__restrict__ pq,
                                  const double *__restrict__ up)
{
    if (threadIdx.x != 0 || blockIdx.x != 0 || st[kStDone] != 0.0) return;
    const double a = st[kStRz] / pq[0];
    if (!isfinite(a) || !(pq[0] > 0.0)) {
        st[kStBroken] = 1.0;
        st[kStDone] = 1.0;
        return;
    }
    st[kStA] = a;
    const double rzn = up[0], rr = up[1];
    const double beta = rzn / st[kStRz];
    st[kStIters] += 1.0;
    st[kStRr] = rr;
    if (!isfinite(rr) || !isfinite(beta)) {
        st[kStBroken] = 1.0;
        st[kStDone] = 1.0;
        return;
    }
    st[kStBeta] = beta;
    st[kStRz] = rzn;
    if (rr <= st[kStStop]) st[kStDone] = 1.0;
}

// x64 += d, d = 0 on owned interior cells.
__global__ void k_slab_x_update(Slab S, double *__restrict__ x, float *__restrict__ d)
{
    for (int64_t l = S.own0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < S.own1;
         l += (int64_t)gridDim.x * blockDim.x) {
        if (!S.g.interior(l + S.lbase)) continue;
        x[l] += (double)d[l];
        d[l] = 0.0f;
    }
}

// out[k] = in-order sum over the nblocks partials of value k (one warp per value).
__global__ void k_slab_finish(const double *__restrict__ part, int nblocks, int nvals, double *__restrict__ out)
{
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= nvals) return;
    double s = 0.0;
    for (int i = lane; i < nblocks; i += 32) s += part[(int64_t)k * nblocks + i];
    s = warp_sum(s);
    if (lane == 0) out[k] = s;
}

int slab_make(int nx, int ny, int nz, int z0, int z1, float dt, float norm, Slab *S)
{
    PIRO_ARG(nx >= 3 && ny >= 3 && nz >= 3 && z0 >= 0 && z1 > z0 && z1 <= nz && dt > 0.0f && norm > 0.0f &&
                 (int64_t)nx * ny * nz < ((int64_t)1 << 31),
             "piro_slab: bad grid, slab or coefficients");
    const int64_t sxy = (int64_t)nx * ny;
    S->g = GridDiv(nx, ny, nz);
    S->lbase = (int64_t)(z0 - 1) * sxy;
    S->own0 = sxy;
    S->own1 = (int64_t)(z1 - z0 + 1) * sxy;
    S->mdt = -dt;
    S->vself = (float)(-6.0 / (double)norm);
    S->vnb = (float)(1.0 / (double)norm);
    return PIRO_OK;
}

unsigned slab_grid() { return (unsigned)std::min(kSlabBlocks, sm_count() * 8); }

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_slab_workspace(int64_t *doubles)
{
    PIRO_ARG(doubles, "piro_slab_workspace: bad arguments");
    *doubles = 4 * (int64_t)kSlabBlocks;  // partial sums: [value][block]
    return PIRO_OK;
}

extern "C" int piro_slab_be_residual(int nx, int ny, int nz, int z0, int z1, float dt, float norm,
                                     const float *alpha, const float *b, const double *x64, float *r, float *z,
                                     double *work, double *sums, piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, dt, norm, &S);
    if (rc) return rc;
    PIRO_ARG(alpha && b && x64 && r && z && work && sums, "piro_slab_be_residual: null pointer");
    cudaStream_t st = as_stream(stream);
    const unsigned grid = slab_grid();
    k_slab_residual<<<grid, kSlabThreads, 0, st>>>(S, alpha, b, x64, r, z, work);
    PIRO_CHECK_LAUNCH("k_slab_residual");
    k_slab_finish<<<1, 32 * 4, 0, st>>>(work, (int)grid, 4, sums);
    PIRO_CHECK_LAUNCH("k_slab_finish");
    return PIRO_OK;
}

extern "C" int piro_slab_cg_spmv(int nx, int ny, int nz, int z0, int z1, float dt, float norm, float beta,
                                 const float *alpha, const float *z, const float *p_old, float *p_new, float *q,
                                 double *work, double *sums, piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, dt, norm, &S);
    if (rc) return rc;
    PIRO_ARG(alpha && z && p_old && p_new && q && work && sums && p_old != p_new, "piro_slab_cg_spmv: bad pointers");
    cudaStream_t st = as_stream(stream);
    const unsigned grid = slab_grid();
    k_slab_cg_spmv<<<grid, kSlabThreads, 0, st>>>(S, beta, nullptr, alpha, z, p_old, p_new, q, work);
    PIRO_CHECK_LAUNCH("k_slab_cg_spmv");
    k_slab_finish<<<1, 32, 0, st>>>(work, (int)grid, 1, sums);
    PIRO_CHECK_LAUNCH("k_slab_finish");
    return PIRO_OK;
}

extern "C" int piro_slab_cg_update(int nx, int ny, int nz, int z0, int z1, float dt, float norm, float a,
                                   const float *alpha, const float *p, const float *q, float *d, float *r, float *z,
                                   double *work, double *sums, piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, dt, norm, &S);
    if (rc) return rc;
    PIRO_ARG(alpha && p && q && d && r && z && work && sums, "piro_slab_cg_update: null pointer");
    cudaStream_t st = as_stream(stream);
    const unsigned grid = slab_grid();
    k_slab_cg_update<<<grid, kSlabThreads, 0, st>>>(S, a, nullptr, nullptr, alpha, p, q, d, r, z, work);
    PIRO_CHECK_LAUNCH("k_slab_cg_update");
    k_slab_finish<<<1, 64, 0, st>>>(work, (int)grid, 2, sums);
    PIRO_CHECK_LAUNCH("k_slab_finish");
    return PIRO_OK;
}

extern "C" int piro_slab_x_update(int nx, int ny, int nz, int z0, int z1, double *x64, float *d, piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, 1.0f, 1.0f, &S);
    if (rc) return rc;
    PIRO_ARG(x64 && d, "piro_slab_x_update: null pointer");
    k_slab_x_update<<<slab_grid(), kSlabThreads, 0, as_stream(stream)>>>(S, x64, d);
    PIRO_CHECK_LAUNCH("k_slab_x_update");
    return PIRO_OK;
}

extern "C" int piro_slab_cg_spmv_dev(int nx, int ny, int nz, int z0, int z1, float dt, float norm,
                                     const double *state, const float *alpha, const float *z, const float *p_old,
                                     float *p_new, float *q, double *work, double *sums, piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, dt, norm, &S);
    if (rc) return rc;
    PIRO_ARG(state && alpha && z && p_old && p_new && q && work && sums && p_old != p_new,
             "piro_slab_cg_spmv_dev: bad pointers");
    cudaStream_t st = as_stream(stream);
    const unsigned grid = slab_grid();
    k_slab_cg_spmv<<<grid, kSlabThreads, 0, st>>>(S, 0.0f, state, alpha, z, p_old, p_new, q, work);
    PIRO_CHECK_LAUNCH("k_slab_cg_spmv");
    k_slab_finish<<<1, 32, 0, st>>>(work, (int)grid, 1, sums);
    PIRO_CHECK_LAUNCH("k_slab_finish");
    return PIRO_OK;
}

extern "C" int piro_slab_cg_update_dev(int nx, int ny, int nz, int z0, int z1, float dt, float norm,
                                       const double *state, const double *pq, const float *alpha, const float *p,
                                       const float *q, float *d, float *r, float *z, double *work, double *sums,
                                       piro_stream_t stream)
{
    Slab S;
    int rc = slab_make(nx, ny, nz, z0, z1, dt, norm, &S);
    if (rc) return rc;
    PIRO_ARG(state && pq && alpha && p && q && d && r && z && work && sums, "piro_slab_cg_update_dev: null pointer");
    cudaStream_t st = as_stream(stream);
    const unsigned grid = slab_grid();
    k_slab_cg_update<<<grid, kSlabThreads, 0, st>>>(S, 0.0f, state, pq, alpha, p, q, d, r, z, work);
    PIRO_CHECK_LAUNCH("k_slab_cg_update");
    k_slab_finish<<<1, 64, 0, st>>>(work, (int)grid, 2, sums);
    PIRO_CHECK_LAUNCH("k_slab_finish");
    return PIRO_OK;
}

extern "C" int piro_slab_cg_scalars(double *state, const double *pq, const double *up, piro_stream_t stream)
{
    PIRO_ARG(state && pq && up, "piro_slab_cg_scalars: null pointer");
    k_slab_cg_scalars<<<1, 32, 0, as_stream(stream)>>>(state, pq, up);
    PIRO_CHECK_LAUNCH("k_slab_cg_scalars");
    return PIRO_OK;
}

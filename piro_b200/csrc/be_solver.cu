// be_solver.cu -- backward-Euler solve (TIMESCHEME 12) on the device.
//
// System: A u = b, A = I - dt*diag(alpha)*L (CSR over all N rows, built by
// csrgeam A + beta*B).  Interior rows are unknowns, boundary rows hold u = b.
// With S = diag(alpha)^-1 A_II symmetric positive definite (L symmetric on
// the interior for the central scheme), the solve is
//   FP64 iterative refinement: r = b - A x in FP64 (x kept in FP64),
//   FP32 Jacobi-preconditioned CG on S d = diag(alpha)^-1 r, x += d,
// until ||b - A x||_2 / ||b||_2 <= rtol over the interior rows.
//
// One CG iteration is two kernels, both HBM-bound on the matrix stream:
//   k_cg_spmv:   p = z + beta*p_old (own rows; neighbours formed on the fly),
//                q = A p, partial <p, q/alpha>; the last block computes a.
//   k_cg_update: d += a p, r -= a q, z = r / A_rr, partials <r/alpha, z> and
//                <r, r>; the last block computes beta and the stop flag.
// "Last block" = the block that takes the final ticket of an atomic counter
// after publishing its partial (no spin-waits).  Scalars stay on the device;
// the host checks a pinned flag once per chunk of iterations, which are
// launched as a CUDA graph and return at once when the flag is set.
#include <cmath>
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "csr_tile.cuh"

namespace piro {

int dot_f64(int64_t n, const float *x, const float *y, double *out, void *work, size_t work_bytes, cudaStream_t s);
size_t reduce_workspace_bytes(int64_t n);

namespace {

constexpr int kChunk = 8;       // CG iterations per graph launch (even: p buffers alternate)
constexpr int kRedCap = 4096;   // max blocks of a reducing kernel

struct DevState {
    double rz;      // <s, z> of the current iterate
    double a;       // step length
    double beta;    // direction update
    double rr;      // <r, r> (FP32 residual of the correction system)
    double rr0;     // <r, r> at the start of the inner solve
    double tol2;    // inner stop: rr <= tol2 * rr0
    double rel;     // FP64 relative residual of the last refinement sweep
    double bnorm;   // ||b|| over the interior
    int done;       // inner solve finished (converged, capped or broken down)
    int iters;      // inner iterations of the current sweep
    int max_iters;  // inner cap
    int broken;     // a non-finite scalar appeared
    unsigned ticket[4];
};

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

// Publish one partial per block; returns true in the block that arrives last
// (all partials of the launch are then visible to it).
__device__ __forceinline__ bool publish_last(double *partials, int slot_stride, int nvals, const double *vals,
                                             unsigned *ticket, bool *s_last)
{
    if (threadIdx.x == 0) {
        for (int t = 0; t < nvals; ++t) partials[t * slot_stride + blockIdx.x] = vals[t];
        __threadfence();
        const unsigned k = atomicAdd(ticket, 1u);
        *s_last = k == gridDim.x - 1;
    }
    __syncthreads();
    if (*s_last) __threadfence();
    return *s_last;
}

__device__ __forceinline__ double gather_sum(const double *partials, double *s_warp)
{
    double s = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) s += ((volatile const double *)partials)[k];
    return block_sum(s, s_warp);
}

// r = b - A x in FP64 on interior rows, stored as float; z = r / A_rr;
// partials of ||r64||^2, ||b||^2, <r/alpha, z>, ||r32||^2.  The last block
// sets up the inner solve: rz, rr0, tol2, rel, done/iters reset, beta = 0.
__global__ void __launch_bounds__(kTileRows) k_residual(int nx, int ny, int nz, int64_t N,
                                                        const int32_t *__restrict__ rowptr,
                                                        const int32_t *__restrict__ col,
                                                        const float *__restrict__ val,
                                                        const float *__restrict__ alpha,
                                                        const float *__restrict__ dinv, const float *__restrict__ b,
                                                        const double *__restrict__ x, float *__restrict__ r,
                                                        float *__restrict__ z, double *__restrict__ partials,
                                                        DevState *__restrict__ st, double rtol, double inner_floor)
{
    __shared__ int32_t s_rp[kTileRows + 1];
    __shared__ int32_t s_col[kTileCap];
    __shared__ float s_val[kTileCap];
    __shared__ double s_warp[32];
    __shared__ bool s_last;
    double rr64 = 0.0, bb = 0.0, rz = 0.0, rr32 = 0.0;
    for (int64_t r0 = (int64_t)blockIdx.x * kTileRows; r0 < N; r0 += (int64_t)gridDim.x * kTileRows) {
        const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
        for (int t = threadIdx.x; t <= nrows; t += blockDim.x) s_rp[t] = rowptr[r0 + t];
        __syncthreads();
        const int64_t s = s_rp[0], e = s_rp[nrows];
        const bool staged = e - s <= kTileCap;
        if (staged) stage_tile(col, val, s, e, s_col, s_val);
        __syncthreads();
        if (threadIdx.x < nrows) {
            const int64_t row = r0 + threadIdx.x;
            if (interior(row, nx, ny, nz)) {
                double q = 0.0;
                for (int k = s_rp[threadIdx.x]; k < s_rp[threadIdx.x + 1]; ++k) {
                    const float v = staged ? s_val[k - s] : val[k];
                    const int32_t c = staged ? s_col[k - s] : col[k];
                    q += (double)v * x[c];
                }
                const double bi = (double)b[row];
                const double ri = bi - q;
                const float rf = (float)ri;
                const float zf = rf * dinv[row];
                r[row] = rf;
                z[row] = zf;
                rr64 += ri * ri;
                bb += bi * bi;
                rz += (double)rf / (double)alpha[row] * (double)zf;
                rr32 += (double)rf * (double)rf;
            } else {
                r[row] = 0.0f;
                z[row] = 0.0f;
            }
        }
        __syncthreads();
    }
    double part[4] = {block_sum(rr64, s_warp), block_sum(bb, s_warp), block_sum(rz, s_warp), block_sum(rr32, s_warp)};
    if (!publish_last(partials, kRedCap, 4, part, &st->ticket[0], &s_last)) return;
    double tot[4];
    for (int t = 0; t < 4; ++t) tot[t] = gather_sum(partials + t * kRedCap, s_warp);
    if (threadIdx.x == 0) {
        const double bn = sqrt(tot[1]) > 0.0 ? sqrt(tot[1]) : 1.0;
        const double rel = sqrt(tot[0]) / bn;
        st->rel = rel;
        st->bnorm = bn;
        st->rz = tot[2];
        st->rr = tot[3];
        st->rr0 = tot[3];
        double itol = rel > 0.0 ? 0.5 * rtol / rel : 1.0;
        itol = itol > 0.1 ? 0.1 : itol;
        itol = itol < inner_floor ? inner_floor : itol;
        st->tol2 = itol * itol;
        st->beta = 0.0;
        st->a = 0.0;
        st->iters = 0;
        st->broken = 0;
        st->done = (tot[3] == 0.0 || rel <= rtol) ? 1 : 0;
        st->ticket[0] = 0u;
    }
}

// p = z + beta*p_old (interior; 0 on boundary), q = A p, partial <p, q/alpha>.
__global__ void __launch_bounds__(kTileRows) k_cg_spmv(int nx, int ny, int nz, int64_t N,
                                                       const int32_t *__restrict__ rowptr,
                                                       const int32_t *__restrict__ col,
                                                       const float *__restrict__ val,
                                                       const float *__restrict__ alpha, const float *__restrict__ z,
                                                       const float *__restrict__ p_old, float *__restrict__ p_new,
                                                       float *__restrict__ q, double *__restrict__ partials,
                                                       DevState *__restrict__ st)
{
    __shared__ int32_t s_rp[kTileRows + 1];
    __shared__ int32_t s_col[kTileCap];
    __shared__ float s_val[kTileCap];
    __shared__ double s_warp[32];
    __shared__ bool s_last;
    __shared__ int s_done;
    __shared__ float s_beta;
    if (threadIdx.x == 0) {
        s_done = *((volatile int *)&st->done);
        s_beta = (float)st->beta;
    }
    __syncthreads();
    if (s_done) return;
    const float beta = s_beta;
    double pq = 0.0;
    for (int64_t r0 = (int64_t)blockIdx.x * kTileRows; r0 < N; r0 += (int64_t)gridDim.x * kTileRows) {
        const int nrows = (int)(N - r0 < kTileRows ? N - r0 : kTileRows);
        for (int t = threadIdx.x; t <= nrows; t += blockDim.x) s_rp[t] = rowptr[r0 + t];
        __syncthreads();
        const int64_t s = s_rp[0], e = s_rp[nrows];
        const bool staged = e - s <= kTileCap;
        if (staged) stage_tile(col, val, s, e, s_col, s_val);
        __syncthreads();
        if (threadIdx.x < nrows) {
            const int64_t row = r0 + threadIdx.x;
            if (interior(row, nx, ny, nz)) {
                float acc = 0.0f;
                for (int k = s_rp[threadIdx.x]; k < s_rp[threadIdx.x + 1]; ++k) {
                    const float v = staged ? s_val[k - s] : val[k];
                    const int32_t c = staged ? s_col[k - s] : col[k];
                    acc += v * (__ldg(z + c) + beta * __ldg(p_old + c));
                }
                const float pn = z[row] + beta * p_old[row];
                p_new[row] = pn;
                q[row] = acc;
                pq += (double)pn * (double)acc / (double)alpha[row];
            } else {
                p_new[row] = 0.0f;
                q[row] = 0.0f;
            }
        }
        __syncthreads();
    }
    double part = block_sum(pq, s_warp);
    if (!publish_last(partials, kRedCap, 1, &part, &st->ticket[1], &s_last)) return;
    const double tot = gather_sum(partials, s_warp);
    if (threadIdx.x == 0) {
        const double a = st->rz / tot;
        if (!isfinite(a) || tot <= 0.0) {
            st->broken = 1;
            st->done = 1;
            st->a = 0.0;
        } else {
            st->a = a;
        }
        st->ticket[1] = 0u;
    }
}

// d += a p, r -= a q, z = r*dinv on interior rows; partials <r/alpha, z>, <r, r>.
__global__ void __launch_bounds__(512) k_cg_update(int nx, int ny, int nz, int64_t N, const float *__restrict__ alpha,
                                                   const float *__restrict__ dinv, const float *__restrict__ p,
                                                   const float *__restrict__ q, float *__restrict__ d,
                                                   float *__restrict__ r, float *__restrict__ z,
                                                   double *__restrict__ partials, DevState *__restrict__ st)
{
    __shared__ double s_warp[32];
    __shared__ bool s_last;
    __shared__ int s_done;
    __shared__ float s_a;
    if (threadIdx.x == 0) {
        s_done = *((volatile int *)&st->done);
        s_a = (float)st->a;
    }
    __syncthreads();
    if (s_done) return;
    const float a = s_a;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const float di = dinv[i];
        if (di == 0.0f) continue;  // boundary rows carry dinv = 0
        d[i] += a * p[i];
        const float ri = r[i] - a * q[i];
        const float zi = ri * di;
        r[i] = ri;
        z[i] = zi;
        rz += (double)ri / (double)alpha[i] * (double)zi;
        rr += (double)ri * (double)ri;
    }
    double part[2] = {block_sum(rz, s_warp), block_sum(rr, s_warp)};
    if (!publish_last(partials, kRedCap, 2, part, &st->ticket[2], &s_last)) return;
    double tot[2];
    for (int t = 0; t < 2; ++t) tot[t] = gather_sum(partials + t * kRedCap, s_warp);
    if (threadIdx.x == 0) {
        const double beta = tot[0] / st->rz;
        st->beta = beta;
        st->rz = tot[0];
        st->rr = tot[1];
        const int it = st->iters + 1;
        st->iters = it;
        if (!isfinite(tot[1]) || !isfinite(beta)) {
            st->broken = 1;
            st->done = 1;
        } else if (tot[1] <= st->tol2 * st->rr0 || it >= st->max_iters) {
            st->done = 1;
        }
        st->ticket[2] = 0u;
    }
}

// Interior Jacobi scale 1/A_rr (0 on boundary rows).
__global__ void k_diag_inv(int nx, int ny, int nz, int64_t N, const int32_t *__restrict__ rowptr,
                           const int32_t *__restrict__ col, const float *__restrict__ val, float *__restrict__ dinv)
{
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        float dv = 0.0f;
        if (interior(r, nx, ny, nz)) {
            double s = 0.0;
            for (int32_t k = rowptr[r]; k < rowptr[r + 1]; ++k)
                if (col[k] == r) s += val[k];
            dv = s != 0.0 ? (float)(1.0 / s) : 0.0f;
        }
        dinv[r] = dv;
    }
}

__global__ void k_promote(int64_t N, const float *__restrict__ b, double *__restrict__ x)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = (double)b[i];
}

// x += d on interior rows, d = 0.
__global__ void k_x_update(int64_t N, const float *__restrict__ dinv, double *__restrict__ x, float *__restrict__ d)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        if (dinv[i] != 0.0f) x[i] += (double)d[i];
        d[i] = 0.0f;
    }
}

__global__ void k_demote(int64_t N, const double *__restrict__ x, float *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)x[i];
}

}  // namespace
}  // namespace piro

using namespace piro;

struct piro_be_solver {
    int nx, ny, nz;
    int64_t N;
    const int32_t *rowptr, *col;
    const float *val, *alpha;
    cudaStream_t caller;  // the stream the caller's buffers are ordered on
    cudaStream_t stream;  // the solver's own non-blocking stream (graph capture needs one)
    cudaEvent_t ev_in;
    unsigned grid_tiles, grid_elem;
    float *dinv, *r, *z, *q, *d, *p[2];
    double *x64;
    double *partials;
    DevState *st;
    DevState *h_st;  // pinned mirror
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    double inner_floor;
    // event pairs around each k_cg_spmv of the captured chunk: live kernel times
    cudaEvent_t ev0[kChunk], ev1[kChunk];
    double spmv_ms;
    long long spmv_launches;
    long long kernel_launches;  // every kernel this solver launched
};

static void be_free(piro_be_solver *s)
{
    if (!s) return;
    for (int i = 0; i < kChunk; ++i) {
        if (s->ev0[i]) cudaEventDestroy(s->ev0[i]);
        if (s->ev1[i]) cudaEventDestroy(s->ev1[i]);
    }
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->ev_in) cudaEventDestroy(s->ev_in);
    if (s->graph) cudaGraphDestroy(s->graph);
    cudaFree(s->dinv);
    cudaFree(s->x64);
    cudaFree(s->partials);
    cudaFree(s->st);
    if (s->h_st) cudaFreeHost(s->h_st);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

static int be_capture_chunk(piro_be_solver *s)
{
    // Capture kChunk iterations; p buffers alternate, so a chunk of an even
    // number of iterations starts and ends on p[0].
    for (int i = 0; i < kChunk; ++i) {
        PIRO_CUDA(cudaEventCreate(&s->ev0[i]));
        PIRO_CUDA(cudaEventCreate(&s->ev1[i]));
    }
    PIRO_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < kChunk; ++it) {
        const float *p_old = s->p[it & 1];
        float *p_new = s->p[(it + 1) & 1];
        // External: the record becomes a node of the graph, observable from the host
        cudaEventRecordWithFlags(s->ev0[it], s->stream, cudaEventRecordExternal);
        k_cg_spmv<<<s->grid_tiles, kTileRows, 0, s->stream>>>(s->nx, s->ny, s->nz, s->N, s->rowptr, s->col, s->val,
                                                              s->alpha, s->z, p_old, p_new, s->q, s->partials, s->st);
        cudaEventRecordWithFlags(s->ev1[it], s->stream, cudaEventRecordExternal);
        k_cg_update<<<s->grid_elem, 512, 0, s->stream>>>(s->nx, s->ny, s->nz, s->N, s->alpha, s->dinv, p_new, s->q,
                                                         s->d, s->r, s->z, s->partials, s->st);
    }
    cudaError_t e = cudaStreamEndCapture(s->stream, &s->graph);
    if (e != cudaSuccess) {
        piro::set_error("graph capture: %s", cudaGetErrorString(e));
        return PIRO_ERR_CUDA;
    }
    PIRO_CUDA(cudaGraphInstantiate(&s->exec, s->graph, 0));
    return PIRO_OK;
}

extern "C" int piro_be_create(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                              const float *alpha, piro_stream_t stream, piro_be_solver **out)
{
    PIRO_ARG(out && rowptr && col && val && alpha && nx >= 3 && ny >= 3 && nz >= 3, "piro_be_create: bad arguments");
    *out = nullptr;
    piro_be_solver *s = new piro_be_solver();
    s->nx = nx;
    s->ny = ny;
    s->nz = nz;
    s->N = (int64_t)nx * ny * nz;
    s->rowptr = rowptr;
    s->col = col;
    s->val = val;
    s->alpha = alpha;
    s->caller = as_stream(stream);
    s->inner_floor = 1e-6;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(s->ev_in, s->caller) != cudaSuccess || cudaStreamWaitEvent(s->stream, s->ev_in, 0) != cudaSuccess) {
        be_free(s);
        piro::set_error("piro_be_create: stream setup failed");
        return PIRO_ERR_CUDA;
    }
    const int64_t N = s->N;
    s->grid_tiles = (unsigned)std::min<int64_t>(cdiv(N, kTileRows), (int64_t)sm_count() * 6);
    s->grid_elem = (unsigned)std::min<int64_t>(cdiv(N, 512 * 4), (int64_t)sm_count() * 4);
    if (s->grid_tiles > (unsigned)kRedCap || s->grid_elem > (unsigned)kRedCap) {
        be_free(s);
        piro::set_error("piro_be_create: reduction grid exceeds %d blocks", kRedCap);
        return PIRO_ERR_ARG;
    }
    // one allocation for the seven FP32 work vectors
    float *fbuf = nullptr;
    cudaError_t e = cudaMalloc(&fbuf, sizeof(float) * (size_t)N * 7);
    if (e == cudaSuccess) e = cudaMalloc(&s->x64, sizeof(double) * (size_t)N);
    if (e == cudaSuccess) e = cudaMalloc(&s->partials, sizeof(double) * kRedCap * 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->st, sizeof(DevState));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_st, sizeof(DevState));
    if (e != cudaSuccess) {
        cudaFree(fbuf);
        be_free(s);
        piro::set_error("piro_be_create: allocation failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_NOMEM;
    }
    s->dinv = fbuf;
    s->r = fbuf + N;
    s->z = fbuf + 2 * N;
    s->q = fbuf + 3 * N;
    s->d = fbuf + 4 * N;
    s->p[0] = fbuf + 5 * N;
    s->p[1] = fbuf + 6 * N;
    if (cudaMemsetAsync(fbuf, 0, sizeof(float) * (size_t)N * 7, s->stream) != cudaSuccess ||
        cudaMemsetAsync(s->st, 0, sizeof(DevState), s->stream) != cudaSuccess) {
        be_free(s);
        piro::set_error("piro_be_create: memset failed");
        return PIRO_ERR_CUDA;
    }
    k_diag_inv<<<grid_for(N, 256, 8), 256, 0, s->stream>>>(nx, ny, nz, N, rowptr, col, val, s->dinv);
    if (cudaGetLastError() != cudaSuccess) {
        be_free(s);
        piro::set_error("k_diag_inv launch failed");
        return PIRO_ERR_CUDA;
    }
    int rc = be_capture_chunk(s);
    if (rc) {
        be_free(s);
        return rc;
    }
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
        be_free(s);
        piro::set_error("piro_be_create: setup kernels failed");
        return PIRO_ERR_CUDA;
    }
    *out = s;
    return PIRO_OK;
}

extern "C" int piro_be_solve(piro_be_solver *s, const float *b, float *x, double rtol, int max_outer, int max_inner,
                             piro_be_info *info)
{
    PIRO_ARG(s && b && x && rtol > 0.0 && max_outer > 0 && max_inner > 0, "piro_be_solve: bad arguments");
    cudaStream_t st = s->stream;
    const int64_t N = s->N;
    // b was produced on the caller's stream; x is read there after we return
    // (this call synchronizes the solver stream before returning).
    PIRO_CUDA(cudaEventRecord(s->ev_in, s->caller));
    PIRO_CUDA(cudaStreamWaitEvent(st, s->ev_in, 0));
    piro_be_info inf{};
    inf.status = PIRO_ERR_NOT_CONVERGED;
    k_promote<<<grid_for(N, 256, 8), 256, 0, st>>>(N, b, s->x64);
    PIRO_CHECK_LAUNCH("k_promote");
    s->kernel_launches += 1;
    PIRO_CUDA(cudaMemsetAsync(s->d, 0, sizeof(float) * (size_t)N, st));
    double prev_rel = INFINITY;
    for (int outer = 0; outer <= max_outer; ++outer) {
        k_residual<<<s->grid_tiles, kTileRows, 0, st>>>(s->nx, s->ny, s->nz, N, s->rowptr, s->col, s->val, s->alpha,
                                                       s->dinv, b, s->x64, s->r, s->z, s->partials, s->st, rtol,
                                                       s->inner_floor);
        PIRO_CHECK_LAUNCH("k_residual");
        s->kernel_launches += 1;
        // cap for this sweep
        int cap = max_inner - inf.inner_iterations;
        PIRO_CUDA(cudaMemcpyAsync(&s->st->max_iters, &cap, sizeof(int), cudaMemcpyHostToDevice, st));
        PIRO_CUDA(cudaMemcpyAsync(s->h_st, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
        PIRO_CUDA(cudaStreamSynchronize(st));
        const double rel = s->h_st->rel;
        inf.rel_residual = rel;
        if (!std::isfinite(rel)) {
            inf.status = PIRO_STATUS_STALLED;
            break;
        }
        if (rel <= rtol) {
            inf.status = PIRO_OK;
            break;
        }
        if (outer == max_outer || cap <= 0) break;
        if (outer > 0 && rel > 0.5 * prev_rel) {
            inf.status = PIRO_STATUS_STALLED;  // refinement no longer contracts
            break;
        }
        prev_rel = rel;
        inf.outer_iterations = outer + 1;
        // inner CG: launch graph chunks until the device flag says done
        int seen = 0;
        while (true) {
            PIRO_CUDA(cudaGraphLaunch(s->exec, st));
            s->kernel_launches += 2 * kChunk;
            PIRO_CUDA(cudaMemcpyAsync(s->h_st, s->st, sizeof(DevState), cudaMemcpyDeviceToHost, st));
            PIRO_CUDA(cudaStreamSynchronize(st));
            // kernel times of the iterations that ran in this chunk
            const int ran = std::min(kChunk, s->h_st->iters - seen);
            for (int i = 0; i < ran; ++i) {
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, s->ev0[i], s->ev1[i]) == cudaSuccess) {
                    s->spmv_ms += ms;
                    s->spmv_launches += 1;
                } else {
                    (void)cudaGetLastError();  // timing is best effort; do not leak the error
                }
            }
            seen = s->h_st->iters;
            if (s->h_st->done) break;
        }
        inf.inner_iterations += s->h_st->iters;
        if (s->h_st->broken) {
            inf.status = PIRO_STATUS_STALLED;
            break;
        }
        k_x_update<<<grid_for(N, 256, 8), 256, 0, st>>>(N, s->dinv, s->x64, s->d);
        PIRO_CHECK_LAUNCH("k_x_update");
        s->kernel_launches += 1;
    }
    k_demote<<<grid_for(N, 256, 8), 256, 0, st>>>(N, s->x64, x);
    PIRO_CHECK_LAUNCH("k_demote");
    s->kernel_launches += 1;
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (info) *info = inf;
    return inf.status == PIRO_OK ? PIRO_OK : inf.status;
}

extern "C" int piro_be_solution_f64(piro_be_solver *s, const double **x64)
{
    PIRO_ARG(s && x64, "piro_be_solution_f64: bad arguments");
    *x64 = s->x64;
    return PIRO_OK;
}

extern "C" int piro_be_kernel_stats(piro_be_solver *s, int reset, long long *spmv_launches, double *spmv_ms,
                                    long long *kernel_launches)
{
    PIRO_ARG(s, "piro_be_kernel_stats: null solver");
    if (spmv_launches) *spmv_launches = s->spmv_launches;
    if (spmv_ms) *spmv_ms = s->spmv_ms;
    if (kernel_launches) *kernel_launches = s->kernel_launches;
    if (reset) {
        s->spmv_launches = 0;
        s->spmv_ms = 0.0;
        s->kernel_launches = 0;
    }
    return PIRO_OK;
}

extern "C" int piro_be_destroy(piro_be_solver *s)
{
    be_free(s);
    return PIRO_OK;
}

// ---------------------------------------------------------------------------
// JLI, the reference's Richardson iteration, on the device.
extern "C" int piro_be_jli(int nx, int ny, int nz, const int32_t *rowptr, const int32_t *col, const float *val,
                           float dt, const float *b, float *x, float *r_work, float tol, float urf, int maxiter,
                           int *iters, piro_stream_t stream)
{
    PIRO_ARG(rowptr && col && val && b && x && r_work && maxiter > 0, "piro_be_jli: bad arguments");
    cudaStream_t st = as_stream(stream);
    const int64_t N = (int64_t)nx * ny * nz;
    size_t wb = reduce_workspace_bytes(N);
    void *work = nullptr;
    double *d_sum = nullptr, h_sum = 0.0;
    PIRO_CUDA(cudaMalloc(&work, wb + 256));
    d_sum = reinterpret_cast<double *>(static_cast<char *>(work) + wb);
    PIRO_CUDA(cudaMemcpyAsync(x, b, sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
    float res_old = 0.0f;
    int it = 0, rc = PIRO_OK;
    for (; it < maxiter; ++it) {
        if ((rc = cudaMemsetAsync(r_work, 0, sizeof(float) * N, st) != cudaSuccess ? PIRO_ERR_CUDA : PIRO_OK)) break;
        if ((rc = piro_csr_i1(nx, ny, nz, rowptr, col, val, dt, x, r_work, stream))) break;
        if ((rc = piro_vec_op(1, N, b, r_work, r_work, stream))) break;
        if ((rc = piro_vec_urf(N, x, r_work, urf, stream))) break;
        if ((rc = dot_f64(N, r_work, r_work, d_sum, work, wb, st))) break;
        if (cudaMemcpyAsync(&h_sum, d_sum, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = PIRO_ERR_CUDA;
            break;
        }
        const float res = sqrtf((float)h_sum) / sqrtf((float)N);
        const float dd = (res - res_old) * (res - res_old);
        if (dd < tol) {
            ++it;
            break;
        }
        res_old = res;
    }
    cudaFree(work);
    if (iters) *iters = it;
    return rc;
}

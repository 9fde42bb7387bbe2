// reduce.cu -- FP64-accumulated dot products and norms.
//
// The reference copies the whole residual vector to the host every iteration
// and sums squares there in float (extras.cpp:24-30, kernelprocess.cpp:195-196).
// Here a grid-stride kernel accumulates x*y in double per thread, reduces per
// warp with shuffles and per block through shared memory, and writes one
// partial per block into caller-provided workspace; the last block to finish
// (an atomic ticket, no spinning) sums the partials in block order.  The
// result is deterministic for a given device and size.
#include "common.cuh"

namespace piro {
namespace {

constexpr int kRedThreads = 512;

__device__ __forceinline__ double block_sum(double v, double *s_warp)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s_warp[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0.0;
        t = warp_sum(t);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

__global__ void __launch_bounds__(kRedThreads) k_dot(int64_t n, const float *__restrict__ x,
                                                     const float *__restrict__ y, double *__restrict__ partials,
                                                     unsigned *__restrict__ ticket, double *__restrict__ out)
{
    __shared__ double s_warp[32];
    __shared__ bool s_last;
    double acc = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i < n; i += stride) acc += (double)__ldg(x + i) * (double)__ldg(y + i);
    const double b = block_sum(acc, s_warp);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = b;
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        s_last = t == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double s = 0.0;
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) s += ((volatile double *)partials)[k];
    // fixed-order combine: per-thread strided sums, then the block tree
    s = block_sum(s, s_warp);
    if (threadIdx.x == 0) {
        *out = s;
        *ticket = 0u;  // re-arm for the next call
    }
}

unsigned dot_grid(int64_t n)
{
    const int64_t want = cdiv(n, (int64_t)kRedThreads * 4);
    const int64_t cap = (int64_t)sm_count() * 4;
    return (unsigned)(want < 1 ? 1 : want < cap ? want : cap);
}

}  // namespace

size_t reduce_workspace_bytes(int64_t n)
{
    (void)n;
    // partials for the largest grid, plus the ticket counter
    return sizeof(double) * (size_t)sm_count() * 4 + 256;
}

// Workspace layout: [ticket (256 B)] [partials].  The ticket is zeroed here
// on the stream before each launch.
int dot_f64(int64_t n, const float *x, const float *y, double *out, void *work, size_t work_bytes, cudaStream_t s)
{
    PIRO_ARG(work && work_bytes >= reduce_workspace_bytes(n), "dot: workspace too small");
    unsigned *ticket = static_cast<unsigned *>(work);
    double *partials = reinterpret_cast<double *>(static_cast<char *>(work) + 256);
    PIRO_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
    const unsigned g = dot_grid(n);
    k_dot<<<g, kRedThreads, 0, s>>>(n, x, y, partials, ticket, out);
    PIRO_CHECK_LAUNCH("k_dot");
    return PIRO_OK;
}

}  // namespace piro

using namespace piro;

extern "C" int piro_reduce_workspace(int64_t n, size_t *bytes)
{
    PIRO_ARG(bytes && n >= 0, "piro_reduce_workspace: bad arguments");
    *bytes = reduce_workspace_bytes(n);
    return PIRO_OK;
}

extern "C" int piro_dot_f64(int64_t n, const float *x, const float *y, double *out, void *work, size_t work_bytes,
                            piro_stream_t stream)
{
    PIRO_ARG(n >= 0 && x && y && out, "piro_dot_f64: null argument");
    return dot_f64(n, x, y, out, work, work_bytes, as_stream(stream));
}

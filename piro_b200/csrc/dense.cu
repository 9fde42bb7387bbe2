// dense.cu -- PIRO's DENSE format (Data 1): the N x N row-major Laplacian and
// its forward-Euler step.
//
// Piro::DENSE::stencils::laplacian_* (src/stencils.cpp:431-570) assign, per
// row l in order, A[l][l] = -6/norm and A[l][nb] = 1/norm for each existing
// neighbour x-, x+, y-, y+, z-, z+; uw/dw replace a "+"/"-" neighbour by l
// itself, so the later assignment wins on the diagonal.  No 10.0 rule here.
// The constants are int / float, i.e. float divisions.
//
// kernelsolve::DENSE::TIMESCHEME_11 (src/kernelprocess.cpp:42-66) runs
// SpMVDENSE.cl -- C[r] = dt * sum, sum += A[r][k]*u[k] for k ascending, every
// row -- then addVectors.cl, D = u + C.  The step reads N^2 floats: an HBM
// stream.  Each block takes 32 rows; warps 1-7 stream the next 32 x 256 tile
// of A (and the matching 256 entries of u) into shared memory while warp 0,
// one lane per row, adds the current tile in ascending column order, so every
// row's sum is the reference's sequential FP32 sum (multiply, then add: no
// fused multiply-add).  Padding past N adds +0, which leaves the sum as it is
// (a sum that starts at +0 never becomes -0).
#include "common.cuh"

namespace piro {
namespace {

constexpr int kDenseRows = 32, kDenseCols = 256, kDenseThreads = 256;
constexpr int kTileStride = kDenseCols + 1;  // conflict-free per-lane row reads
constexpr size_t kDenseSmem = sizeof(float) * (2 * kDenseRows * kTileStride + 2 * kDenseCols);

__global__ void k_dense_laplacian(int nx, int ny, int nz, int scheme, float vs, float vn, float *__restrict__ A)
{
    const int64_t N = (int64_t)nx * ny * nz;
    for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(l % nx), y = (int)((l / nx) % ny), z = (int)(l / ((int64_t)nx * ny));
        const int64_t sx = 1, sy = nx, sz = (int64_t)nx * ny;
        float *row = A + l * N;
        row[l] = vs;
        if (x > 0) row[scheme == 2 ? l : l - sx] = vn;
        if (x < nx - 1) row[scheme == 1 ? l : l + sx] = vn;
        if (y > 0) row[scheme == 2 ? l : l - sy] = vn;
        if (y < ny - 1) row[scheme == 1 ? l : l + sy] = vn;
        if (z > 0) row[scheme == 2 ? l : l - sz] = vn;
        if (z < nz - 1) row[scheme == 1 ? l : l + sz] = vn;
    }
}

__device__ __forceinline__ void dense_load_tile(int64_t N, const float *__restrict__ A, const float *__restrict__ u,
                                                int64_t R0, int64_t k0, float *__restrict__ sa, float *__restrict__ su)
{
    const int t = threadIdx.x - 32, nt = kDenseThreads - 32;
    for (int e = t; e < kDenseRows * kDenseCols; e += nt) {
        const int r = e / kDenseCols, c = e % kDenseCols;
        const int64_t gr = R0 + r, gc = k0 + c;
        sa[r * kTileStride + c] = (gr < N && gc < N) ? __ldcs(A + gr * N + gc) : 0.0f;
    }
    for (int c = t; c < kDenseCols; c += nt) su[c] = k0 + c < N ? __ldg(u + k0 + c) : 0.0f;
}

__global__ void __launch_bounds__(kDenseThreads) k_dense_fe(int64_t N, const float *__restrict__ A, float dt,
                                                            const float *__restrict__ u, float *__restrict__ out)
{
    extern __shared__ float sm[];
    float *sa0 = sm, *sa1 = sm + kDenseRows * kTileStride;
    float *su0 = sm + 2 * kDenseRows * kTileStride, *su1 = su0 + kDenseCols;
    const int64_t R0 = (int64_t)blockIdx.x * kDenseRows;
    const int64_t ntile = cdiv(N, kDenseCols);
    if (threadIdx.x >= 32) dense_load_tile(N, A, u, R0, 0, sa0, su0);
    __syncthreads();
    float sum = 0.0f;
    for (int64_t t = 0; t < ntile; ++t) {
        const bool odd = t & 1;
        if (threadIdx.x >= 32) {
            if (t + 1 < ntile) dense_load_tile(N, A, u, R0, (t + 1) * kDenseCols, odd ? sa0 : sa1, odd ? su0 : su1);
        } else {
            const float *a = (odd ? sa1 : sa0) + threadIdx.x * kTileStride;
            const float *uu = odd ? su1 : su0;
#pragma unroll 16
            for (int c = 0; c < kDenseCols; ++c) sum = __fadd_rn(sum, __fmul_rn(a[c], uu[c]));
        }
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        const int64_t r = R0 + threadIdx.x;
        if (r < N) out[r] = __fadd_rn(u[r], __fmul_rn(dt, sum));
    }
}

}  // namespace
}  // namespace piro

using namespace piro;

extern "C" int piro_dense_laplacian(int nx, int ny, int nz, int scheme, float norm, float *A, size_t a_bytes,
                                    piro_stream_t stream)
{
    PIRO_ARG(nx > 0 && ny > 0 && nz > 0 && A && scheme >= 1 && scheme <= 3, "piro_dense_laplacian: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(a_bytes / sizeof(float) / (size_t)N >= (size_t)N, "piro_dense_laplacian: A holds fewer than N*N floats");
    cudaStream_t st = as_stream(stream);
    PIRO_CUDA(cudaMemsetAsync(A, 0, sizeof(float) * (size_t)N * (size_t)N, st));
    const float vs = -6.0f / norm, vn = 1.0f / norm;  // stencils.cpp:439,445: int / float
    k_dense_laplacian<<<grid_for(N, 256, 8), 256, 0, st>>>(nx, ny, nz, scheme, vs, vn, A);
    PIRO_CHECK_LAUNCH("k_dense_laplacian");
    return PIRO_OK;
}

extern "C" int piro_dense_fe_step(int64_t N, const float *A, float dt, const float *u, float *out,
                                  piro_stream_t stream)
{
    PIRO_ARG(N >= 1 && A && u && out && u != out, "piro_dense_fe_step: bad arguments");
    PIRO_ARG(cdiv(N, kDenseRows) < 2147483647, "piro_dense_fe_step: N too large");
    static bool attr_set[64] = {false};
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        PIRO_CUDA(cudaFuncSetAttribute(k_dense_fe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDenseSmem));
        attr_set[dev] = true;
    }
    k_dense_fe<<<(unsigned)cdiv(N, kDenseRows), kDenseThreads, kDenseSmem, as_stream(stream)>>>(N, A, dt, u, out);
    PIRO_CHECK_LAUNCH("k_dense_fe");
    return PIRO_OK;
}

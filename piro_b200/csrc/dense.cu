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
// stream.  One thread per row keeps the reference's sequential FP32 sum
// (multiply, then add: no fused multiply-add).  A block of 256 rows streams
// its rows through shared memory 32 columns at a time, three stages deep, with
// cp.async (any N: 4-byte copies, no alignment needed; zero-filled past N), so
// that ~100 KB per block are in flight; each warp copies whole 128-byte row
// segments.  Padding adds +0, which leaves the sum as it is (a sum that starts
// at +0 never becomes -0).
#include "common.cuh"

namespace piro {
namespace {

constexpr int kDenseRows = 256, kDenseCols = 32, kDenseStages = 3, kDenseThreads = kDenseRows;
constexpr int kTileStride = kDenseCols + 1;  // conflict-free per-thread row reads
constexpr int kStageFloats = kDenseRows * kTileStride + kDenseCols;
constexpr size_t kDenseSmem = sizeof(float) * kDenseStages * kStageFloats;

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

__device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}

// Stage tile t (columns 32t .. 32t+31 of the block's rows, and u there).
__device__ __forceinline__ void dense_issue(int64_t N, const float *__restrict__ A, const float *__restrict__ u,
                                            int64_t R0, int64_t t, float *stage)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t c = t * kDenseCols + lane;
    const bool cok = c < N;
    for (int r = warp; r < kDenseRows; r += kDenseThreads / 32) {
        const int64_t row = R0 + r;
        const bool ok = cok && row < N;
        cp_async4(stage + r * kTileStride + lane, ok ? A + row * N + c : A, ok);
    }
    if (warp == 0) cp_async4(stage + kDenseRows * kTileStride + lane, cok ? u + c : u, cok);
}

// The stream when N % 4 == 0 and A, u are 16-byte aligned: per item, 32 rows
// x BC columns, each row segment (contiguous) one cp.async.bulk into a padded
// row (float4 reads conflict-free), completion on an mbarrier.  One warp per
// CTA, lane = row, persistent over row blocks; the (row block, column tile)
// items stream through S stages without a bubble at row-block boundaries.
// Measured on B200 (tail-free N): two stages and many CTAs per SM stream
// best -- 128 columns x 6 CTAs/SM 6.7 TB/s, 256 columns x 3 CTAs/SM
// 6.1 TB/s -- since each CTA's sequential row sums, not the copies, set its
// pace; the host picks the shape whose last round of row blocks wastes
// least.  Every wait is bounded.
constexpr int kBR = 32;
constexpr long long kBSpin = 1ll << 22;

template <int BC, int S>
constexpr size_t bulk_smem() { return sizeof(float) * S * (kBR * (BC + 4) + BC); }

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kBSpin; ++i)
        if (bar_try_wait(bar, parity)) return true;
    return false;
}

template <int BC, int S>
__global__ void __launch_bounds__(32) k_dense_fe_bulk(int64_t N, const float *__restrict__ A, float dt,
                                                      const float *__restrict__ u, float *__restrict__ out, int *err)
{
    constexpr int RS = BC + 4, SF = kBR * RS + BC;
    extern __shared__ __align__(128) float smb[];
    __shared__ __align__(8) uint64_t bars[S];
    const int lane = threadIdx.x;
    const int64_t nrb = cdiv(N, kBR), ntile = cdiv(N, BC);
    const int64_t my_rb = nrb > (int64_t)blockIdx.x ? cdiv(nrb - blockIdx.x, gridDim.x) : 0;
    const int64_t items = my_rb * ntile;
    if (lane == 0) {
        for (int s = 0; s < S; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[s])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    auto issue = [&](int64_t i) {
        const int s = (int)(i % S);
        const int64_t t = i % ntile, rb = blockIdx.x + (i / ntile) * gridDim.x;
        const int64_t R0 = rb * kBR, k0 = t * BC;
        const int nrows = (int)(N - R0 < kBR ? N - R0 : kBR);
        const uint32_t bytes = (uint32_t)(4 * (N - k0 < BC ? N - k0 : BC));
        float *stage = smb + s * SF;
        const uint32_t bar = smem_addr(&bars[s]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // this lane's reads of the stage first
        __syncwarp();
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"(bytes * (uint32_t)(nrows + 1))
                         : "memory");
        __syncwarp();
        if (lane < nrows)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(stage + lane * RS)),
                "l"(A + (R0 + lane) * N + k0), "r"(bytes), "r"(bar)
                : "memory");
        if (lane == 31)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(stage + kBR * RS)),
                "l"(u + k0), "r"(bytes), "r"(bar)
                : "memory");
    };
    int64_t issued = 0;
    for (; issued < S && issued < items; ++issued) issue(issued);
    float sum = 0.0f;
    int64_t i = 0;
    bool ok = true;
    for (; i < items; ++i) {
        const int s = (int)(i % S);
        if (!bar_wait(smem_addr(&bars[s]), (uint32_t)((i / S) & 1))) {
            ok = false;
            break;
        }
        const int64_t t = i % ntile, rb = blockIdx.x + (i / ntile) * gridDim.x;
        const int64_t R0 = rb * kBR, k0 = t * BC;
        const int ncols = (int)(N - k0 < BC ? N - k0 : BC);
        const float *stage = smb + s * SF;
        if (R0 + lane < N) {
            const float4 *a = reinterpret_cast<const float4 *>(stage + lane * RS);
            const float4 *uu = reinterpret_cast<const float4 *>(stage + kBR * RS);
#pragma unroll 8
            for (int c = 0; c < ncols / 4; ++c) {
                const float4 av = a[c], uv = uu[c];
                sum = __fadd_rn(sum, __fmul_rn(av.x, uv.x));
                sum = __fadd_rn(sum, __fmul_rn(av.y, uv.y));
                sum = __fadd_rn(sum, __fmul_rn(av.z, uv.z));
                sum = __fadd_rn(sum, __fmul_rn(av.w, uv.w));
            }
        }
        if (t == ntile - 1) {
            const int64_t r = R0 + lane;
            if (r < N) out[r] = __fadd_rn(u[r], __fmul_rn(dt, sum));
            sum = 0.0f;
        }
        __syncwarp();
        if (issued < items) issue(issued++);
    }
    if (!ok) {
        if (lane == 0) atomicExch(err, 1);
        for (; i < issued; ++i) (void)bar_wait(smem_addr(&bars[i % S]), (uint32_t)((i / S) & 1));
    }
}

__global__ void __launch_bounds__(kDenseThreads) k_dense_fe(int64_t N, const float *__restrict__ A, float dt,
                                                            const float *__restrict__ u, float *__restrict__ out)
{
    extern __shared__ float sm[];
    const int64_t R0 = (int64_t)blockIdx.x * kDenseRows;
    const int64_t ntile = cdiv(N, kDenseCols);
    for (int s = 0; s < kDenseStages - 1; ++s) {
        if (s < ntile) dense_issue(N, A, u, R0, s, sm + s * kStageFloats);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    float sum = 0.0f;
    for (int64_t t = 0; t < ntile; ++t) {
        const int64_t tn = t + kDenseStages - 1;
        if (tn < ntile) dense_issue(N, A, u, R0, tn, sm + (int)(tn % kDenseStages) * kStageFloats);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kDenseStages - 1) : "memory");
        __syncthreads();
        const float *st = sm + (int)(t % kDenseStages) * kStageFloats;
        const float *a = st + threadIdx.x * kTileStride, *uu = st + kDenseRows * kTileStride;
#pragma unroll
        for (int c = 0; c < kDenseCols; ++c) sum = __fadd_rn(sum, __fmul_rn(a[c], uu[c]));
        __syncthreads();  // the stage is refilled by the next iteration's issue
    }
    const int64_t r = R0 + threadIdx.x;
    if (r < N) out[r] = __fadd_rn(u[r], __fmul_rn(dt, sum));
}

// Per-device setup of the FE step: occupancy of the two bulk shapes and the
// flag a bulk-stage wait sets when it times out.
struct DenseDevice {
    int occ_a = 0, occ_b = 0;
    int *err_flag = nullptr;
};
DenseDevice dense_dev[kMaxDevices];
DeviceOnce dense_once;

int dense_setup(int dev)
{
    return device_once(dense_once, dev, [dev]() -> int {
        DenseDevice &d = dense_dev[dev];
        PIRO_CUDA(cudaFuncSetAttribute(k_dense_fe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDenseSmem));
        PIRO_CUDA(cudaFuncSetAttribute(k_dense_fe_bulk<256, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bulk_smem<256, 2>()));
        PIRO_CUDA(cudaFuncSetAttribute(k_dense_fe_bulk<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)bulk_smem<128, 2>()));
        PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_a, k_dense_fe_bulk<256, 2>, 32,
                                                                bulk_smem<256, 2>()));
        PIRO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d.occ_b, k_dense_fe_bulk<128, 2>, 32,
                                                                bulk_smem<128, 2>()));
        if (!d.err_flag) {
            PIRO_CUDA(cudaMalloc(&d.err_flag, sizeof(int)));
            PIRO_CUDA(cudaMemset(d.err_flag, 0, sizeof(int)));
        }
        return PIRO_OK;
    });
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
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    const int rc = dense_setup(dev);
    if (rc != PIRO_OK) return rc;
    const DenseDevice &d = dense_dev[dev];
    cudaStream_t st = as_stream(stream);
    const bool bulk = N % 4 == 0 && ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(u)) & 15) == 0;
    if (bulk && d.occ_a >= 1 && d.occ_b >= 1) {
        // time ~ rounds of row blocks x (CTAs per SM / measured stream rate):
        // 256 columns at up to 3 CTAs/SM ~6.1 TB/s, 128 columns at up to 6 ~6.7 TB/s
        const int64_t nrb = cdiv(N, kBR), sms = sm_count();
        const int ga = d.occ_a < 3 ? d.occ_a : 3, gb = d.occ_b < 6 ? d.occ_b : 6;
        const double ta = (double)cdiv(nrb, ga * sms) * ga / 6.1, tb = (double)cdiv(nrb, gb * sms) * gb / 6.7;
        if (ta <= tb) {
            const int64_t grid = nrb < ga * sms ? nrb : ga * sms;
            k_dense_fe_bulk<256, 2><<<(unsigned)grid, 32, bulk_smem<256, 2>(), st>>>(N, A, dt, u, out, d.err_flag);
        } else {
            const int64_t grid = nrb < gb * sms ? nrb : gb * sms;
            k_dense_fe_bulk<128, 2><<<(unsigned)grid, 32, bulk_smem<128, 2>(), st>>>(N, A, dt, u, out, d.err_flag);
        }
        PIRO_CHECK_LAUNCH("k_dense_fe_bulk");
        return PIRO_OK;
    }
    k_dense_fe<<<(unsigned)cdiv(N, kDenseRows), kDenseThreads, kDenseSmem, st>>>(N, A, dt, u, out);
    PIRO_CHECK_LAUNCH("k_dense_fe");
    return PIRO_OK;
}

extern "C" int piro_dense_check(piro_stream_t stream)
{
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    PIRO_ARG(dev >= 0 && dev < kMaxDevices, "piro_dense_check: device index");
    if (!dense_once.done[dev].load(std::memory_order_acquire)) return PIRO_OK;  // no FE step ran here
    int *flag = dense_dev[dev].err_flag;
    int h = 0;
    cudaStream_t st = as_stream(stream);
    PIRO_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (h) {
        PIRO_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
        set_error("piro_dense_fe_step: a stage wait timed out");
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

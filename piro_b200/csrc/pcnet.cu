// pcnet.cu -- the learned preconditioner network: a 3-D convolutional net
// z = M(r, f) that maps a residual r (scaled to unit RMS) and a per-cell
// feature f = log(dt * alpha / h^2) to an approximation of the error
// A^-1 r, used inside flexible CG (be_solver.cu).  Input channels: r and r*f.  PIRO has no learned
// component; this is the build's own addition to the backward-Euler solve
// (TIMESCHEME 12, src/kernelprocess.cpp:123-209).
//
// Network: four 3x3x3 convolutions, channels 2 -> 16 -> 16 -> 16 -> 1, GELU
// (tanh form) after the first three, zero padding outside the interior (boundary cells
// of the ghost-inclusive grid hold zero activations, so an interior cell's
// 27 neighbours are always inside the array).  BF16 weights and activations,
// FP32 accumulation.  Activations are stored channels-last (16 bf16 = 32 bytes
// per cell); the output is FP32.
//
// The convolutions carry no bias: with GELU(0) = 0 the network maps a zero
// residual to a zero correction, so cells where the residual has vanished get
// no spurious update (a biased network adds an r-independent term that stalls
// flexible CG once the residual is localised).  Parameters are one flat FP32
// vector (the Adam master copy): per layer W[tap][ci][co], tap =
// (dz+1)*9 + (dy+1)*3 + (dx+1).  The kernels read `wq`, the same vector
// rounded to BF16 (held as FP32 values).
//
// Training runs on the device with this file's forward and backward kernels:
// masked MSE loss against a target error, backward through the four layers
// (data gradient = the transposed convolution times GELU'; weight gradient =
// per-block partial correlations reduced in a fixed order, so gradients are
// deterministic), and Adam.  With the tensor-core engine (the default) every
// convolution of training runs on tcgen05: the forward and the data gradient
// as the implicit GEMM of conv_tc.cuh (the data gradient with the weights
// transposed and the taps reversed), the weight gradient as the GEMM over
// cells of wgrad_tc.cuh.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "conv_tc.cuh"
#include "wgrad_tc.cuh"

namespace piro {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTaps = 27;
constexpr int kLayers = 4;
constexpr int kTcZChunk = 16;  // z-planes per CTA of the tensor-core layers
constexpr int kCi[kLayers] = {2, 16, 16, 16};
constexpr int kCo[kLayers] = {16, 16, 16, 1};

struct Layout {
    int64_t w[kLayers], total;
    Layout()
    {
        int64_t o = 0;
        for (int l = 0; l < kLayers; ++l) {
            w[l] = o;
            o += (int64_t)kTaps * kCi[l] * kCo[l];
        }
        total = o;
    }
};

// GELU in its tanh form (Hendrycks & Gimpel 2016), g(x) = 0.5 x (1 + t),
// t = tanh(c (x + a x^3)), c = sqrt(2/pi), a = 0.044715, with the hardware
// tanh.approx; g'(x) = 0.5 (1 + t) + 0.5 x (1 - t^2) c (1 + 3 a x^2).
__device__ __forceinline__ float tanh_hw(float u)
{
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return t;
}
__device__ __forceinline__ float gelu(float x)
{
    return 0.5f * x * (1.0f + tanh_hw(0.7978845608028654f * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_d(float x)
{
    const float t = tanh_hw(0.7978845608028654f * (x + 0.044715f * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * x * x);
}

__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

template <int C>
__device__ __forceinline__ void load_act(const bf16 *__restrict__ p, float (&v)[C])
{
    if constexpr (C == 16) {
        const uint4 u0 = *reinterpret_cast<const uint4 *>(p);
        const uint4 u1 = *reinterpret_cast<const uint4 *>(p + 8);
        const uint32_t w[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[k]);
            const float2 f = __bfloat1622float2(h);
            v[2 * k] = f.x;
            v[2 * k + 1] = f.y;
        }
    } else if constexpr (C == 2) {
        const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p));
        v[0] = f.x;
        v[1] = f.y;
    } else {
#pragma unroll
        for (int k = 0; k < C; ++k) v[k] = __bfloat162float(p[k]);
    }
}

template <int C>
__device__ __forceinline__ void store_act(bf16 *__restrict__ p, const float (&v)[C])
{
    if constexpr (C == 16) {
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
            w[k] = *reinterpret_cast<const uint32_t *>(&h);
        }
        *reinterpret_cast<uint4 *>(p) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4 *>(p + 8) = make_uint4(w[4], w[5], w[6], w[7]);
    } else {
#pragma unroll
        for (int k = 0; k < C; ++k) p[k] = __float2bfloat16_rn(v[k]);
    }
}

template <int C>
__device__ __forceinline__ void store_zero(bf16 *__restrict__ p)
{
    if constexpr (C == 16) {
        *reinterpret_cast<uint4 *>(p) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4 *>(p + 8) = make_uint4(0, 0, 0, 0);
    } else {
#pragma unroll
        for (int k = 0; k < C; ++k) p[k] = __float2bfloat16_rn(0.0f);
    }
}

__device__ __forceinline__ int64_t tap_off(int t, int nx, int64_t nxy)
{
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    return (int64_t)dx + (int64_t)dy * nx + (int64_t)dz * nxy;
}

// x0[b][c] = (bf16(r * s_b), bf16(r * s_b * f)) on interior cells, 0
// elsewhere: the feature enters multiplied by the residual, so that both
// input channels -- and with no biases the whole network -- vanish with r.
// s_b = 1 / sqrt(rr[b] / n_int) when rr is given (device FP64 sums of r^2),
// else 1.  f may be NULL (feature 0).
__global__ void k_pack_input(GridDiv g, int64_t N, const float *__restrict__ r, const float *__restrict__ feat,
                             const double *__restrict__ rr, double n_int, bf16 *__restrict__ x0,
                             const int *__restrict__ skip)
{
    if (skip && *((volatile const int *)skip)) return;
    const int b = blockIdx.y;
    float s = 1.0f;
    if (rr) {
        const double v = rr[b];
        s = v > 0.0 ? (float)(1.0 / sqrt(v / n_int)) : 0.0f;
    }
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = (int64_t)b * N + c;
        __nv_bfloat162 h = __floats2bfloat162_rn(0.0f, 0.0f);
        if (g.interior(c)) {
            const float rs = r[o] * s;
            h = __floats2bfloat162_rn(rs, feat ? rs * feat[o] : 0.0f);
        }
        *reinterpret_cast<__nv_bfloat162 *>(x0 + 2 * o) = h;
    }
}

// One convolution layer, one interior cell per thread, all CO outputs in
// registers; the layer's weights sit in shared memory (broadcast reads).
// kMode 0: store a = bf16(GELU(bf16(acc))) (inference); 1: also store the
// pre-activation y = bf16(acc) (training); 2: CO == 1, FP32 output times
// the per-batch output scale sqrt(rr / n_int) when rr is given.  A set
// *skip (the solver's "inner solve done" flag) makes the launch return at once.
template <int CI, int CO, int kMode>
__global__ void __launch_bounds__(128) k_conv_fwd(GridDiv g, int64_t N, const bf16 *__restrict__ x,
                                                  const float *__restrict__ w, bf16 *__restrict__ y, bf16 *__restrict__ a, float *__restrict__ out,
                                                  const double *__restrict__ rr, double n_int,
                                                  const int *__restrict__ skip)
{
    if (skip && *((volatile const int *)skip)) return;
    __shared__ __align__(16) float sw[kTaps * CI * CO];
    __shared__ int64_t soff[kTaps];
    const int64_t nxy = (int64_t)g.nx * g.ny;
    for (int i = threadIdx.x; i < kTaps * CI * CO; i += blockDim.x) sw[i] = w[i];
    if (threadIdx.x < kTaps) soff[threadIdx.x] = tap_off(threadIdx.x, g.nx, nxy);
    __syncthreads();
    const int b = blockIdx.y;
    const bf16 *__restrict__ xb = x + (int64_t)b * N * CI;
    float oscale = 1.0f;
    if (kMode == 2 && rr) oscale = (float)sqrt(rr[b] / n_int);
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = (int64_t)b * N + c;
        if (!g.interior(c)) {
            if constexpr (kMode == 2) {
                out[o] = 0.0f;
            } else {
                store_zero<CO>(a + o * CO);
                if (kMode == 1) store_zero<CO>(y + o * CO);
            }
            continue;
        }
        float acc[CO];
#pragma unroll
        for (int k = 0; k < CO; ++k) acc[k] = 0.0f;
#pragma unroll 1
        for (int t = 0; t < kTaps; ++t) {
            float xv[CI];
            load_act<CI>(xb + (c + soff[t]) * CI, xv);
            const float *wt = sw + t * CI * CO;
#pragma unroll
            for (int ci = 0; ci < CI; ++ci)
#pragma unroll
                for (int k = 0; k < CO; ++k) acc[k] = fmaf(xv[ci], wt[ci * CO + k], acc[k]);
        }
        if constexpr (kMode == 2) {
            out[o] = acc[0] * oscale;
        } else {
            float yv[CO], av[CO];
#pragma unroll
            for (int k = 0; k < CO; ++k) {
                yv[k] = bfr(acc[k]);
                av[k] = gelu(yv[k]);
            }
            store_act<CO>(a + o * CO, av);
            if (kMode == 1) store_act<CO>(y + o * CO, yv);
        }
    }
}

template <int C, typename T>
__device__ __forceinline__ void load_grad(const T *__restrict__ p, float (&v)[C])
{
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int k = 0; k < C; ++k) v[k] = p[k];
    } else {
        load_act<C>(p, v);
    }
}

// Data gradient of one layer: gprev[c'][ci] = GELU'(yprev[c'][ci]) *
// sum_t sum_co W[t][ci][co] * gy[c' - off(t)][co] on interior c', 0 elsewhere.
template <int CO, int CI, typename GT>
__global__ void __launch_bounds__(128) k_conv_bwd_data(GridDiv g, int64_t N, const GT *__restrict__ gy,
                                                       const float *__restrict__ w, const bf16 *__restrict__ yprev,
                                                       bf16 *__restrict__ gprev)
{
    __shared__ __align__(16) float sw[kTaps * CI * CO];
    __shared__ int64_t soff[kTaps];
    const int64_t nxy = (int64_t)g.nx * g.ny;
    for (int i = threadIdx.x; i < kTaps * CI * CO; i += blockDim.x) sw[i] = w[i];
    if (threadIdx.x < kTaps) soff[threadIdx.x] = tap_off(threadIdx.x, g.nx, nxy);
    __syncthreads();
    const int b = blockIdx.y;
    const GT *__restrict__ gb = gy + (int64_t)b * N * CO;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = (int64_t)b * N + c;
        if (!g.interior(c)) {
            store_zero<CI>(gprev + o * CI);
            continue;
        }
        float acc[CI];
#pragma unroll
        for (int k = 0; k < CI; ++k) acc[k] = 0.0f;
#pragma unroll 1
        for (int t = 0; t < kTaps; ++t) {
            float gv[CO];
            load_grad<CO>(gb + (c - soff[t]) * CO, gv);
            const float *wt = sw + t * CI * CO;
#pragma unroll
            for (int ci = 0; ci < CI; ++ci)
#pragma unroll
                for (int k = 0; k < CO; ++k) acc[ci] = fmaf(wt[ci * CO + k], gv[k], acc[ci]);
        }
        float yp[CI];
        load_act<CI>(yprev + o * CI, yp);
#pragma unroll
        for (int k = 0; k < CI; ++k) acc[k] *= gelu_d(yp[k]);
        store_act<CI>(gprev + o * CI, acc);
    }
}

// Weight gradient partials of one layer.  A block takes chunks of
// kWChunk consecutive cells of one batch member, stages the 9 (dy, dz)-shifted
// input ranges (kWChunk + 2 cells each) and the chunk's output gradient in
// shared memory; thread (ci, co) accumulates its 27 taps in registers over all
// its chunks and writes one partial per block.
constexpr int kWChunk = 64;

template <int CI, int CO, typename GT>
__global__ void __launch_bounds__(256) k_conv_bwd_w(GridDiv g, int64_t N, int B, const bf16 *__restrict__ x,
                                                    const GT *__restrict__ gy, float *__restrict__ partials)
{
    extern __shared__ float smw[];
    float *sx = smw;                              // [9][kWChunk + 2][CI]
    float *sg = smw + 9 * (kWChunk + 2) * CI;     // [kWChunk][CO]
    constexpr int P = kTaps * CI * CO;
    const int t = threadIdx.x;
    const bool act = t < CI * CO;
    const int ci = act ? t / CO : 0, co = act ? t % CO : 0;
    const int64_t nxy = (int64_t)g.nx * g.ny;
    float acc[kTaps];
#pragma unroll
    for (int k = 0; k < kTaps; ++k) acc[k] = 0.0f;
    const int64_t chunks = cdiv(N, kWChunk);
    const int64_t total = chunks * B;
    for (int64_t k = blockIdx.x; k < total; k += gridDim.x) {
        const int b = (int)(k / chunks);
        const int64_t c0 = (k - (int64_t)b * chunks) * kWChunk;
        const bf16 *__restrict__ xb = x + (int64_t)b * N * CI;
        const GT *__restrict__ gb = gy + (int64_t)b * N * CO;
        __syncthreads();
        for (int i = t; i < 9 * (kWChunk + 2) * CI; i += blockDim.x) {
            const int ch = i % CI;
            const int j = (i / CI) % (kWChunk + 2);
            const int r = i / (CI * (kWChunk + 2));
            const int64_t cell = c0 - 1 + j + (int64_t)(r % 3 - 1) * g.nx + (int64_t)(r / 3 - 1) * nxy;
            sx[i] = (cell >= 0 && cell < N) ? __bfloat162float(xb[cell * CI + ch]) : 0.0f;
        }
        for (int i = t; i < kWChunk * CO; i += blockDim.x) {
            const int64_t cell = c0 + i / CO;
            float v = 0.0f;
            if (cell < N) {
                if constexpr (sizeof(GT) == 4)
                    v = gb[cell * CO + i % CO];
                else
                    v = __bfloat162float(gb[cell * CO + i % CO]);
            }
            sg[i] = v;
        }
        __syncthreads();
        if (act) {
#pragma unroll 4
            for (int j = 0; j < kWChunk; ++j) {
                const float gv = sg[j * CO + co];
#pragma unroll
                for (int r = 0; r < 9; ++r)
#pragma unroll
                    for (int dx = 0; dx < 3; ++dx)
                        acc[r * 3 + dx] = fmaf(sx[(r * (kWChunk + 2) + j + dx) * CI + ci], gv, acc[r * 3 + dx]);
            }
        }
    }
    if (act) {
        float *pb = partials + (int64_t)blockIdx.x * P;
#pragma unroll
        for (int k = 0; k < kTaps; ++k) pb[(k * CI + ci) * CO + co] = acc[k];
    }
}

// out[p] = sum over blocks (fixed order, FP64) of partials[block][p].
__global__ void k_reduce_partials(const float *__restrict__ partials, int nblocks, int P, float *__restrict__ out)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < nblocks; ++k) s += (double)partials[(int64_t)k * P + p];
        out[p] = (float)s;
    }
}

constexpr int kRedBlocks = 296;

// Block partials of sum(mask) into red[blockIdx.x].
__global__ void __launch_bounds__(256) k_mask_sum(int64_t n, const float *__restrict__ mask, double *__restrict__ red)
{
    __shared__ double sw[32];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += (double)mask[i];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? sw[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) red[blockIdx.x] = t;
    }
}

// Sum the kRedBlocks partials in order into red[kRedBlocks + slot].
__global__ void k_finish_sum(double *red, int slot)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kRedBlocks; ++k) s += red[k];
        red[kRedBlocks + slot] = s;
    }
}

// Masked MSE: loss = sum m (out - t)^2 / sum m; gout = 2 m (out - t) / sum m
// on interior cells (boundary outputs are constant zeros: gout = 0 there).
__global__ void __launch_bounds__(256) k_loss(GridDiv g, int64_t N, int64_t n, const float *__restrict__ out,
                                              const float *__restrict__ tgt, const float *__restrict__ mask,
                                              double *__restrict__ red, float *__restrict__ gout)
{
    __shared__ double sw[32];
    const double msum = red[kRedBlocks + 0];
    const float inv = msum > 0.0 ? (float)(1.0 / msum) : 0.0f;
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = out[i] - tgt[i];
        const float m = mask[i];
        s += (double)m * (double)d * (double)d;
        gout[i] = g.interior(i % N) ? 2.0f * m * d * inv : 0.0f;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? sw[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) red[blockIdx.x] = t * (msum > 0.0 ? 1.0 / msum : 0.0);
    }
}

__global__ void k_adam(int64_t n, float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, float *__restrict__ wq, float lr, float b1, float b2, float eps,
                       float bc1, float bc2)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        wq[i] = bfr(wi);
    }
}

__global__ void k_round_bf16(int64_t n, const float *__restrict__ w, float *__restrict__ wq)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        wq[i] = bfr(w[i]);
}

// BF16 weights of the four layers in the tensor-core operand layout: per
// layer and tap [channel group 2][co 16][8 ci] (the no-swizzle K-major core
// matrices of conv_tc.cuh), input channels beyond 2 (layer 1) and output
// channels beyond 1 (layer 4) zero.
__global__ void k_pack_wtc(const float *__restrict__ wq, Layout L, bf16 *__restrict__ wpk)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kLayers * kTaps * 256; i += gridDim.x * blockDim.x) {
        const int l = i / (kTaps * 256), rem = i % (kTaps * 256);
        const int tap = rem / 256, r2 = rem % 256;
        const int ci = (r2 / 128) * 8 + (r2 % 8), co = (r2 / 8) % 16;
        const int CI = l == 0 ? 2 : 16, CO = l == kLayers - 1 ? 1 : 16;  // kCi[l], kCo[l]
        const float v = (ci < CI && co < CO) ? wq[L.w[l] + (tap * CI + ci) * CO + co] : 0.0f;
        wpk[i] = __float2bfloat16_rn(v);
    }
}

// The data gradient of layer l as a forward convolution: input channels =
// the layer's outputs, output channels = its inputs, tap t reading the
// gradient at c + off(t) with the weights of tap 26 - t (off(26 - t) =
// -off(t)).  Per layer l = 1..3 and tap: [channel group 2][out 16][8 in] BF16,
// channels beyond the layer's zero.
__global__ void k_pack_wtc_t(const float *__restrict__ wq, Layout L, bf16 *__restrict__ wpk_t)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (kLayers - 1) * kTaps * 256; i += gridDim.x * blockDim.x) {
        const int l = 1 + i / (kTaps * 256), rem = i % (kTaps * 256);
        const int tap = rem / 256, r2 = rem % 256;
        const int gin = (r2 / 128) * 8 + (r2 % 8), gout = (r2 / 8) % 16;  // gin: the layer's co, gout: its ci
        const int CI = l == 0 ? 2 : 16, CO = l == kLayers - 1 ? 1 : 16;
        const float v = (gin < CO && gout < CI) ? wq[L.w[l] + ((kTaps - 1 - tap) * CI + gout) * CO + gin] : 0.0f;
        wpk_t[i] = __float2bfloat16_rn(v);
    }
}

// The loss gradient (FP32, one channel) as a 16-channel BF16 array: channel 0
// = bf16(gout), the rest 0 -- the input of the last layer's data gradient and
// weight gradient on the tensor cores.
__global__ void k_pack_grad16(int64_t n, const float *__restrict__ gout, bf16 *__restrict__ g16)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(gout[i], 0.0f);
        uint4 *dst = reinterpret_cast<uint4 *>(g16 + i * 16);
        dst[0] = make_uint4(*reinterpret_cast<const uint32_t *>(&h), 0, 0, 0);
        dst[1] = make_uint4(0, 0, 0, 0);
    }
}

// Tensor-core input: x16[b][c] = (r s_b, r s_b f, 0 x 14) on interior cells,
// zeros elsewhere (32 bytes per cell, the layout of the hidden activations).
__global__ void k_pack_input16(GridDiv g, int64_t N, const float *__restrict__ r, const float *__restrict__ feat,
                               const double *__restrict__ rr, double n_int, bf16 *__restrict__ x16,
                               const int *__restrict__ skip)
{
    if (skip && *((volatile const int *)skip)) return;
    const int b = blockIdx.y;
    float s = 1.0f;
    if (rr) {
        const double v = rr[b];
        s = v > 0.0 ? (float)(1.0 / sqrt(v / n_int)) : 0.0f;
    }
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = (int64_t)b * N + c;
        uint32_t w0 = 0;
        if (g.interior(c)) {
            const float rs = r[o] * s;
            const __nv_bfloat162 h = __floats2bfloat162_rn(rs, feat ? rs * feat[o] : 0.0f);
            w0 = *reinterpret_cast<const uint32_t *>(&h);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(x16 + o * 16);
        dst[0] = make_uint4(w0, 0, 0, 0);
        dst[1] = make_uint4(0, 0, 0, 0);
    }
}

// Deterministic host RNG for the initial weights (splitmix64 + Box-Muller).
struct HostRng {
    uint64_t s;
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal()
    {
        const double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

}  // namespace
}  // namespace piro

using namespace piro;

struct piro_pcnet {
    Layout L;
    float *w = nullptr, *wq = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;
    bf16 *wpk = nullptr;  // BF16 tensor-core operands of the four layers
    bf16 *wpk_t = nullptr;  // the same, transposed and tap-reversed, of layers 2-4 (data gradients)
    int *d_err = nullptr; // raised by a tensor-core launch whose bounded wait ran out
    int engine = PIRO_PCNET_TENSOR_CORES;
    float *partials = nullptr;
    double *red = nullptr;
    int64_t adam_t = 0;
    // activation workspace for cap cells (batch * N)
    int64_t cap = 0;
    bf16 *x0 = nullptr, *y[3] = {nullptr, nullptr, nullptr}, *a[3] = {nullptr, nullptr, nullptr};
    bf16 *g16[2] = {nullptr, nullptr};
    bf16 *x16 = nullptr, *go16 = nullptr;  // tensor-core training: 16-channel input and loss gradient
    float *out = nullptr, *gout = nullptr;
    long long launches = 0;
};

static void net_free_ws(piro_pcnet *n)
{
    cudaFree(n->x0);
    for (int i = 0; i < 3; ++i) {
        cudaFree(n->y[i]);
        cudaFree(n->a[i]);
    }
    cudaFree(n->g16[0]);
    cudaFree(n->g16[1]);
    cudaFree(n->x16);
    cudaFree(n->go16);
    cudaFree(n->out);
    cudaFree(n->gout);
    n->x0 = nullptr;
    for (int i = 0; i < 3; ++i) n->y[i] = n->a[i] = nullptr;
    n->g16[0] = n->g16[1] = nullptr;
    n->x16 = n->go16 = nullptr;
    n->out = n->gout = nullptr;
    n->cap = 0;
}

static int net_reserve(piro_pcnet *n, int64_t cells, bool training)
{
    if (cells <= n->cap && (!training || n->y[0])) return PIRO_OK;
    net_free_ws(n);
    const size_t c = (size_t)cells;
    cudaError_t e = cudaMalloc(&n->x0, c * 2 * sizeof(bf16));
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMalloc(&n->a[i], c * 16 * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&n->out, c * sizeof(float));
    if (training) {
        for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMalloc(&n->y[i], c * 16 * sizeof(bf16));
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&n->g16[i], c * 16 * sizeof(bf16));
        if (e == cudaSuccess) e = cudaMalloc(&n->gout, c * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&n->x16, c * 16 * sizeof(bf16));
        if (e == cudaSuccess) e = cudaMalloc(&n->go16, c * 16 * sizeof(bf16));
        // defined contents before the first pass (every layer writes all of its output)
        for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMemset(n->y[i], 0, c * 16 * sizeof(bf16));
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMemset(n->g16[i], 0, c * 16 * sizeof(bf16));
        if (e == cudaSuccess) e = cudaMemset(n->out, 0, c * sizeof(float));
    }
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMemset(n->a[i], 0, c * 16 * sizeof(bf16));
    if (e != cudaSuccess) {
        net_free_ws(n);
        set_error("piro_pcnet: workspace allocation failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_NOMEM;
    }
    n->cap = cells;
    return PIRO_OK;
}

static unsigned net_grid(int64_t N, int threads)
{
    const int64_t want = cdiv(N, threads);
    const int64_t cap = (int64_t)sm_count() * 16;
    return (unsigned)(want < cap ? want : cap);
}

// Activation buffers of one forward pass.  Training keeps every layer's
// pre-activation y and activation a; inference ping-pongs two buffers.
struct Acts {
    bf16 *x0;
    bf16 *y[3];
    bf16 *a[3];
};

// Forward pass over `batch` grids of N cells (x0 already packed); out gets
// the FP32 output (scaled by sqrt(rr / n_int) if rr is given).
static int net_forward(const float *wq, const Acts &A, int batch, const GridDiv &g, int64_t N, bool training,
                       float *out, const double *rr, double n_int, const int *skip, cudaStream_t st)
{
    const Layout L;
    const dim3 grid(net_grid(N, 128), batch);
    if (training) {
        k_conv_fwd<2, 16, 1><<<grid, 128, 0, st>>>(g, N, A.x0, wq + L.w[0], A.y[0], A.a[0], nullptr,
                                                   nullptr, 0.0, skip);
        k_conv_fwd<16, 16, 1><<<grid, 128, 0, st>>>(g, N, A.a[0], wq + L.w[1], A.y[1], A.a[1], nullptr,
                                                    nullptr, 0.0, skip);
        k_conv_fwd<16, 16, 1><<<grid, 128, 0, st>>>(g, N, A.a[1], wq + L.w[2], A.y[2], A.a[2], nullptr,
                                                    nullptr, 0.0, skip);
    } else {
        k_conv_fwd<2, 16, 0><<<grid, 128, 0, st>>>(g, N, A.x0, wq + L.w[0], nullptr, A.a[0], nullptr,
                                                   nullptr, 0.0, skip);
        k_conv_fwd<16, 16, 0><<<grid, 128, 0, st>>>(g, N, A.a[0], wq + L.w[1], nullptr, A.a[1], nullptr,
                                                    nullptr, 0.0, skip);
        k_conv_fwd<16, 16, 0><<<grid, 128, 0, st>>>(g, N, A.a[1], wq + L.w[2], nullptr, A.a[2], nullptr,
                                                    nullptr, 0.0, skip);
    }
    k_conv_fwd<16, 1, 2><<<grid, 128, 0, st>>>(g, N, A.a[2], wq + L.w[3], nullptr, nullptr, out, rr,
                                               n_int, skip);
    PIRO_CHECK_LAUNCH("k_conv_fwd");
    return PIRO_OK;
}

static Acts train_acts(piro_pcnet *n)
{
    return Acts{n->x0, {n->y[0], n->y[1], n->y[2]}, {n->a[0], n->a[1], n->a[2]}};
}

// Inference buffers inside one caller-owned block: x0 then two ping-pong
// activation buffers (layer outputs 1 and 3 share the first).
static Acts infer_acts(void *work, int64_t cells)
{
    bf16 *x0 = static_cast<bf16 *>(work);
    bf16 *b0 = x0 + cdiv(cells * 2, 128) * 128;
    bf16 *b1 = b0 + cells * 16;
    return Acts{x0, {nullptr, nullptr, nullptr}, {b0, b1, b0}};
}

// TMA descriptor of an activation array of `rows` cells (16 BF16 channels
// each) as the 3-D view (8 channels, rows at 32 bytes, 2 groups at 16 bytes)
// with box {8, box_rows, 2}: the line blocks of conv_tc.cuh (130 rows) or the
// tiles of wgrad_tc.cuh (128 rows).
static int encode_rows_map(CUtensorMap *m, const void *base, int64_t rows, int box_rows)
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
    const cuuint64_t dims[3] = {8, (cuuint64_t)rows, 2};
    const cuuint64_t strides[2] = {32, 16};
    const cuuint32_t box[3] = {8, (cuuint32_t)box_rows, 2};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(base), dims, strides, box,
                              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

// One layer on the tensor cores over `batch` grids of N cells: in (16 BF16
// channels per cell) -> out (GELU, 16 BF16 channels) or, for the last layer,
// zout (FP32 channel 0 times sqrt(rr / n_int)).  Every cell of the output is
// written, the boundary planes z = 0 and nz - 1 with zeros.
template <int kEpi>
static int conv_tc(const bf16 *in, bf16 *out, float *zout, const bf16 *wpk, const GridDiv &g, int64_t N, int batch,
                   const double *rr, double n_int, const int *skip, int *err, cudaStream_t st,
                   bf16 *yout = nullptr, const bf16 *yprev = nullptr)
{
    static DeviceOnce once;
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    int rc = device_once(once, dev, []() -> int {
        PIRO_CUDA(cudaFuncSetAttribute(tc::k_conv16_tc<kEpi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       tc::kSmemBytes));
        return PIRO_OK;
    });
    if (rc != PIRO_OK) return rc;
    CUtensorMap map;
    rc = encode_rows_map(&map, in, N * batch, tc::kLineRows);
    if (rc) return rc;
    const int64_t nxy = (int64_t)g.nx * g.ny;
    const int ncol = (int)cdiv(nxy, tc::kRows);
    const int planes = g.nz - 2;
    const int zchunk = planes < kTcZChunk ? planes : kTcZChunk;
    const int nzc = (int)cdiv(planes, zchunk);
    tc::Args a{g, N, nxy, ncol, zchunk, wpk, out, zout, rr, n_int, skip, err, yout, yprev};
    tc::k_conv16_tc<kEpi><<<dim3((unsigned)(ncol * nzc), (unsigned)batch), tc::kThreads, tc::kSmemBytes, st>>>(map, a);
    PIRO_CHECK_LAUNCH("k_conv16_tc");
    return PIRO_OK;
}

// Inference forward with all four layers on the tensor cores.  A.a[0] and
// A.a[1] ping-pong: input -> a[1], layer 1 -> a[0], 2 -> a[1], 3 -> a[0],
// layer 4 -> out.
static int net_forward_tc(const piro_pcnet *n, const Acts &A, int batch, const GridDiv &g, int64_t N,
                          const float *r, const float *feat, float *out, const double *rr, double n_int,
                          const int *skip, cudaStream_t st)
{
    bf16 *ping = A.a[0], *pong = A.a[1];
    const int64_t W = (int64_t)kTaps * 256;
    k_pack_input16<<<dim3(net_grid(N, 256), batch), 256, 0, st>>>(g, N, r, feat, rr, n_int, pong, skip);
    PIRO_CHECK_LAUNCH("k_pack_input16");
    int rc = conv_tc<0>(pong, ping, nullptr, n->wpk, g, N, batch, nullptr, 0.0, skip, n->d_err, st);
    if (!rc) rc = conv_tc<0>(ping, pong, nullptr, n->wpk + W, g, N, batch, nullptr, 0.0, skip, n->d_err, st);
    if (!rc) rc = conv_tc<0>(pong, ping, nullptr, n->wpk + 2 * W, g, N, batch, nullptr, 0.0, skip, n->d_err, st);
    if (!rc) rc = conv_tc<1>(ping, nullptr, out, n->wpk + 3 * W, g, N, batch, rr, n_int, skip, n->d_err, st);
    return rc;
}

static int net_pack(piro_pcnet *n, cudaStream_t st)
{
    k_pack_wtc<<<cdiv(kLayers * kTaps * 256, 256), 256, 0, st>>>(n->wq, n->L, n->wpk);
    PIRO_CHECK_LAUNCH("k_pack_wtc");
    k_pack_wtc_t<<<cdiv((kLayers - 1) * kTaps * 256, 256), 256, 0, st>>>(n->wq, n->L, n->wpk_t);
    PIRO_CHECK_LAUNCH("k_pack_wtc_t");
    return PIRO_OK;
}

// Weight gradient of one layer on the tensor cores (wgrad_tc.cuh): x and gy
// are 16-channel BF16 arrays of `cells` rows; the layer's dW (CI x CO kept of
// the 16 x 16 per tap) goes to grad_w through per-CTA partials reduced in a
// fixed order.
static int launch_wgrad_tc(piro_pcnet *n, const GridDiv &g, int64_t cells, const bf16 *x, const bf16 *gy, int CI,
                           int CO, float *grad_w, cudaStream_t st)
{
    static DeviceOnce once;
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    int rc = device_once(once, dev, []() -> int {
        PIRO_CUDA(cudaFuncSetAttribute(tc::k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       tc::kWgSmemBytes));
        return PIRO_OK;
    });
    if (rc != PIRO_OK) return rc;
    CUtensorMap xmap, gmap;
    rc = encode_rows_map(&xmap, x, cells, tc::kWgRows);
    if (!rc) rc = encode_rows_map(&gmap, gy, cells, tc::kWgRows);
    if (rc) return rc;
    const int64_t ntiles = cdiv(cells, tc::kWgRows);
    int64_t grid = sm_count();
    if (grid > kRedBlocks) grid = kRedBlocks;
    if (grid > ntiles) grid = ntiles;
    tc::WgArgs a{g.nx, (int64_t)g.nx * g.ny, ntiles, CI, CO, n->partials, n->d_err};
    tc::k_wgrad_tc<<<(unsigned)grid, tc::kWgThreads, tc::kWgSmemBytes, st>>>(xmap, gmap, a);
    PIRO_CHECK_LAUNCH("k_wgrad_tc");
    const int P = kTaps * CI * CO;
    k_reduce_partials<<<(P + 255) / 256, 256, 0, st>>>(n->partials, (int)grid, P, grad_w);
    PIRO_CHECK_LAUNCH("k_reduce_partials");
    n->launches += 2;
    return PIRO_OK;
}

template <int CI, int CO, typename GT>
static int launch_bwd_w(piro_pcnet *n, const GridDiv &g, int64_t N, int batch, const bf16 *x, const GT *gy,
                        float *grad_w, cudaStream_t st)
{
    const size_t smem = sizeof(float) * (9 * (kWChunk + 2) * CI + kWChunk * CO);
    static DeviceOnce once;
    int dev = 0;
    PIRO_CUDA(cudaGetDevice(&dev));
    const int rc = device_once(once, dev, [smem]() -> int {
        PIRO_CUDA(cudaFuncSetAttribute(k_conv_bwd_w<CI, CO, GT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
        return PIRO_OK;
    });
    if (rc != PIRO_OK) return rc;
    const int nblocks = kRedBlocks;
    constexpr int P = kTaps * CI * CO;
    k_conv_bwd_w<CI, CO, GT><<<nblocks, 256, smem, st>>>(g, N, batch, x, gy, n->partials);
    k_reduce_partials<<<(P + 255) / 256, 256, 0, st>>>(n->partials, nblocks, P, grad_w);
    n->launches += 2;
    PIRO_CHECK_LAUNCH("k_conv_bwd_w");
    return PIRO_OK;
}

extern "C" int piro_pcnet_num_params(int64_t *n)
{
    PIRO_ARG(n, "piro_pcnet_num_params: bad arguments");
    *n = Layout().total;
    return PIRO_OK;
}

extern "C" int piro_pcnet_create(uint64_t seed, piro_pcnet **out)
{
    PIRO_ARG(out, "piro_pcnet_create: bad arguments");
    *out = nullptr;
    piro_pcnet *n = new piro_pcnet();
    const Layout &L = n->L;
    const size_t P = (size_t)L.total;
    const int64_t pmax = (int64_t)kRedBlocks * (kTaps * 16 * 16);
    cudaError_t e = cudaMalloc(&n->w, P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->wq, P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->m, P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->v, P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->g, P * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->partials, (size_t)pmax * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->red, (kRedBlocks + 8) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&n->wpk, sizeof(bf16) * kLayers * kTaps * 256);
    if (e == cudaSuccess) e = cudaMalloc(&n->wpk_t, sizeof(bf16) * (kLayers - 1) * kTaps * 256);
    if (e == cudaSuccess) e = cudaMalloc(&n->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(n->d_err, 0, sizeof(int));
    if (e != cudaSuccess) {
        piro_pcnet_destroy(n);
        set_error("piro_pcnet_create: allocation failed: %s", cudaGetErrorString(e));
        return PIRO_ERR_NOMEM;
    }
    // He-normal initial weights for the GELU layers; the output layer starts
    // ten times smaller.
    std::vector<float> h(P, 0.0f);
    HostRng rng{seed};
    for (int l = 0; l < kLayers; ++l) {
        const double fan_in = (double)kTaps * kCi[l];
        const double sd = std::sqrt(2.0 / fan_in) * (l == kLayers - 1 ? 0.1 : 1.0);
        for (int64_t i = 0; i < (int64_t)kTaps * kCi[l] * kCo[l]; ++i) h[L.w[l] + i] = (float)(sd * rng.normal());
    }
    int rc = piro_pcnet_set_params(n, h.data(), L.total);
    if (rc) {
        piro_pcnet_destroy(n);
        return rc;
    }
    *out = n;
    return PIRO_OK;
}

extern "C" int piro_pcnet_set_params(piro_pcnet *n, const float *host, int64_t count)
{
    PIRO_ARG(n && host && count == n->L.total, "piro_pcnet_set_params: bad arguments");
    const size_t P = (size_t)count;
    PIRO_CUDA(cudaMemcpy(n->w, host, P * sizeof(float), cudaMemcpyHostToDevice));
    PIRO_CUDA(cudaMemset(n->m, 0, P * sizeof(float)));
    PIRO_CUDA(cudaMemset(n->v, 0, P * sizeof(float)));
    PIRO_CUDA(cudaMemset(n->g, 0, P * sizeof(float)));
    k_round_bf16<<<cdiv(count, 256), 256>>>(count, n->w, n->wq);
    PIRO_CHECK_LAUNCH("k_round_bf16");
    int rc = net_pack(n, 0);
    if (rc) return rc;
    PIRO_CUDA(cudaDeviceSynchronize());
    n->adam_t = 0;
    return PIRO_OK;
}

extern "C" int piro_pcnet_get_params(piro_pcnet *n, float *host, int64_t count, int rounded)
{
    PIRO_ARG(n && host && count == n->L.total, "piro_pcnet_get_params: bad arguments");
    PIRO_CUDA(cudaDeviceSynchronize());
    PIRO_CUDA(cudaMemcpy(host, rounded ? n->wq : n->w, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost));
    return PIRO_OK;
}

extern "C" int piro_pcnet_forward(piro_pcnet *n, int batch, int nx, int ny, int nz, const float *r,
                                  const float *feat, float *out, piro_stream_t stream)
{
    PIRO_ARG(n && r && out && batch >= 1 && batch <= 65535 && nx >= 3 && ny >= 3 && nz >= 3,
             "piro_pcnet_forward: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(N < ((int64_t)1 << 31), "piro_pcnet_forward: grid too large");
    cudaStream_t st = as_stream(stream);
    int rc = net_reserve(n, N * batch, false);
    if (rc) return rc;
    const GridDiv g(nx, ny, nz);
    n->launches += 5;
    const Acts A{n->x0, {nullptr, nullptr, nullptr}, {n->a[0], n->a[1], n->a[2]}};
    if (n->engine == PIRO_PCNET_TENSOR_CORES) {
        rc = net_forward_tc(n, A, batch, g, N, r, feat, out, nullptr, 1.0, nullptr, st);
        if (rc) return rc;
        int err = 0;
        PIRO_CUDA(cudaMemcpyAsync(&err, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        PIRO_CUDA(cudaStreamSynchronize(st));
        if (err) {
            set_error("piro_pcnet_forward: a tensor-core pipeline wait timed out");
            return PIRO_ERR_CUDA;
        }
        return PIRO_OK;
    }
    k_pack_input<<<dim3(net_grid(N, 256), batch), 256, 0, st>>>(g, N, r, feat, nullptr, 1.0, n->x0, nullptr);
    PIRO_CHECK_LAUNCH("k_pack_input");
    return net_forward(n->wq, A, batch, g, N, false, out, nullptr, 1.0, nullptr, st);
}

extern "C" int piro_pcnet_set_engine(piro_pcnet *n, int engine)
{
    PIRO_ARG(n && (engine == PIRO_PCNET_CUDA_CORES || engine == PIRO_PCNET_TENSOR_CORES),
             "piro_pcnet_set_engine: bad arguments");
    n->engine = engine;
    return PIRO_OK;
}

namespace piro {
// Device bytes of the caller-owned workspace of pcnet_apply for N cells.
size_t pcnet_apply_bytes(int64_t N) { return sizeof(bf16) * (size_t)(cdiv(N * 2, 128) * 128 + 2 * N * 16); }

// Tensor-core pipeline error of the network (a bounded wait ran out); clears it.
int pcnet_take_error(const piro_pcnet *n, cudaStream_t st)
{
    int err = 0;
    PIRO_CUDA(cudaMemcpyAsync(&err, n->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PIRO_CUDA(cudaStreamSynchronize(st));
    if (err) {
        PIRO_CUDA(cudaMemset(n->d_err, 0, sizeof(int)));
        set_error("learned preconditioner: a tensor-core pipeline wait timed out");
        return PIRO_ERR_CUDA;
    }
    return PIRO_OK;
}

// Preconditioner apply for the solver: z = sqrt(rr/n_int) * M(r / sqrt(rr/n_int), f),
// every launch returning at once when *skip is set.  Reads only the net's
// weight vectors (allocated once per network), so a CUDA graph that captured
// it stays valid while the network is trained or reloaded.  Five kernel
// launches; every cell of z is written (zeros on the boundary).
int pcnet_apply(const piro_pcnet *n, void *work, const GridDiv &g, int64_t N, const float *r, const float *feat,
                const double *rr, double n_int, float *z, const int *skip, cudaStream_t st)
{
    const Acts A = infer_acts(work, N);
    if (n->engine == PIRO_PCNET_TENSOR_CORES) return net_forward_tc(n, A, 1, g, N, r, feat, z, rr, n_int, skip, st);
    k_pack_input<<<dim3(net_grid(N, 256), 1), 256, 0, st>>>(g, N, r, feat, rr, n_int, A.x0, skip);
    PIRO_CHECK_LAUNCH("k_pack_input");
    return net_forward(n->wq, A, 1, g, N, false, z, rr, n_int, skip, st);
}
}  // namespace piro

extern "C" int piro_pcnet_loss_grad(piro_pcnet *n, int batch, int nx, int ny, int nz, const float *r,
                                    const float *feat, const float *target, const float *mask, double *loss,
                                    float *grad, piro_stream_t stream)
{
    PIRO_ARG(n && r && target && mask && batch >= 1 && batch <= 65535 && nx >= 3 && ny >= 3 && nz >= 3,
             "piro_pcnet_loss_grad: bad arguments");
    const int64_t N = (int64_t)nx * ny * nz;
    PIRO_ARG(N < ((int64_t)1 << 31), "piro_pcnet_loss_grad: grid too large");
    cudaStream_t st = as_stream(stream);
    int rc = net_reserve(n, N * batch, true);
    if (rc) return rc;
    const Layout &L = n->L;
    const GridDiv g(nx, ny, nz);
    const int64_t cells = N * batch;
    const bool tcore = n->engine == PIRO_PCNET_TENSOR_CORES;
    const int64_t W = (int64_t)kTaps * 256;
    if (tcore) {
        // forward on the tensor cores, keeping each hidden layer's y and a
        k_pack_input16<<<dim3(net_grid(N, 256), batch), 256, 0, st>>>(g, N, r, feat, nullptr, 1.0, n->x16, nullptr);
        PIRO_CHECK_LAUNCH("k_pack_input16");
        rc = conv_tc<2>(n->x16, n->a[0], nullptr, n->wpk, g, N, batch, nullptr, 0.0, nullptr, n->d_err, st, n->y[0]);
        if (!rc)
            rc = conv_tc<2>(n->a[0], n->a[1], nullptr, n->wpk + W, g, N, batch, nullptr, 0.0, nullptr, n->d_err, st,
                            n->y[1]);
        if (!rc)
            rc = conv_tc<2>(n->a[1], n->a[2], nullptr, n->wpk + 2 * W, g, N, batch, nullptr, 0.0, nullptr, n->d_err,
                            st, n->y[2]);
        if (!rc)
            rc = conv_tc<1>(n->a[2], nullptr, n->out, n->wpk + 3 * W, g, N, batch, nullptr, 0.0, nullptr, n->d_err, st);
    } else {
        k_pack_input<<<dim3(net_grid(N, 256), batch), 256, 0, st>>>(g, N, r, feat, nullptr, 1.0, n->x0, nullptr);
        PIRO_CHECK_LAUNCH("k_pack_input");
        rc = net_forward(n->wq, train_acts(n), batch, g, N, true, n->out, nullptr, 1.0, nullptr, st);
    }
    n->launches += 5;
    if (rc) return rc;
    k_mask_sum<<<kRedBlocks, 256, 0, st>>>(cells, mask, n->red);
    k_finish_sum<<<1, 32, 0, st>>>(n->red, 0);
    k_loss<<<kRedBlocks, 256, 0, st>>>(g, N, cells, n->out, target, mask, n->red, n->gout);
    k_finish_sum<<<1, 32, 0, st>>>(n->red, 1);
    PIRO_CHECK_LAUNCH("k_loss");
    const dim3 grid(net_grid(N, 128), batch);
    if (tcore) {
        // backward on the tensor cores: per layer the weight gradient (GEMM over
        // the cells), then the data gradient into the previous layer's
        // pre-activation (transposed, tap-reversed convolution times GELU')
        k_pack_grad16<<<net_grid(cells, 256), 256, 0, st>>>(cells, n->gout, n->go16);
        PIRO_CHECK_LAUNCH("k_pack_grad16");
        rc = launch_wgrad_tc(n, g, cells, n->a[2], n->go16, 16, 1, n->g + L.w[3], st);
        if (!rc)
            rc = conv_tc<3>(n->go16, n->g16[0], nullptr, n->wpk_t + 2 * W, g, N, batch, nullptr, 0.0, nullptr,
                            n->d_err, st, nullptr, n->y[2]);
        if (!rc) rc = launch_wgrad_tc(n, g, cells, n->a[1], n->g16[0], 16, 16, n->g + L.w[2], st);
        if (!rc)
            rc = conv_tc<3>(n->g16[0], n->g16[1], nullptr, n->wpk_t + W, g, N, batch, nullptr, 0.0, nullptr, n->d_err,
                            st, nullptr, n->y[1]);
        if (!rc) rc = launch_wgrad_tc(n, g, cells, n->a[0], n->g16[1], 16, 16, n->g + L.w[1], st);
        if (!rc)
            rc = conv_tc<3>(n->g16[1], n->g16[0], nullptr, n->wpk_t, g, N, batch, nullptr, 0.0, nullptr, n->d_err, st,
                            nullptr, n->y[0]);
        if (!rc) rc = launch_wgrad_tc(n, g, cells, n->x16, n->g16[0], 2, 16, n->g + L.w[0], st);
        if (rc) return rc;
        n->launches += 4;
        if (loss) {
            PIRO_CUDA(cudaMemcpyAsync(loss, n->red + kRedBlocks + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        if (grad) {
            PIRO_CUDA(cudaMemcpyAsync(grad, n->g, (size_t)L.total * sizeof(float), cudaMemcpyDeviceToHost, st));
        }
        if (loss || grad) return pcnet_take_error(n, st);  // synchronises the stream
        return PIRO_OK;
    }
    // layer 4 (16 -> 1): weight gradient, then the data gradient into layer 3's output
    rc = launch_bwd_w<16, 1, float>(n, g, N, batch, n->a[2], n->gout, n->g + L.w[3], st);
    if (rc) return rc;
    k_conv_bwd_data<1, 16, float><<<grid, 128, 0, st>>>(g, N, n->gout, n->wq + L.w[3], n->y[2], n->g16[0]);
    rc = launch_bwd_w<16, 16, bf16>(n, g, N, batch, n->a[1], n->g16[0], n->g + L.w[2], st);
    if (rc) return rc;
    k_conv_bwd_data<16, 16, bf16><<<grid, 128, 0, st>>>(g, N, n->g16[0], n->wq + L.w[2], n->y[1], n->g16[1]);
    rc = launch_bwd_w<16, 16, bf16>(n, g, N, batch, n->a[0], n->g16[1], n->g + L.w[1], st);
    if (rc) return rc;
    k_conv_bwd_data<16, 16, bf16><<<grid, 128, 0, st>>>(g, N, n->g16[1], n->wq + L.w[1], n->y[0], n->g16[0]);
    rc = launch_bwd_w<2, 16, bf16>(n, g, N, batch, n->x0, n->g16[0], n->g + L.w[0], st);
    if (rc) return rc;
    n->launches += 7;
    PIRO_CHECK_LAUNCH("k_conv_bwd_data");
    if (loss) {
        PIRO_CUDA(cudaMemcpyAsync(loss, n->red + kRedBlocks + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    if (grad) {
        PIRO_CUDA(cudaMemcpyAsync(grad, n->g, (size_t)L.total * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    if (loss || grad) PIRO_CUDA(cudaStreamSynchronize(st));
    return PIRO_OK;
}

extern "C" int piro_pcnet_adam_step(piro_pcnet *n, float lr, piro_stream_t stream)
{
    PIRO_ARG(n && lr > 0.0f, "piro_pcnet_adam_step: bad arguments");
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    n->adam_t += 1;
    const float bc1 = (float)(1.0 - std::pow((double)b1, (double)n->adam_t));
    const float bc2 = (float)(1.0 - std::pow((double)b2, (double)n->adam_t));
    const int64_t P = n->L.total;
    k_adam<<<cdiv(P, 256), 256, 0, as_stream(stream)>>>(P, n->w, n->m, n->v, n->g, n->wq, lr, b1, b2, eps, bc1,
                                                         bc2);
    n->launches += 2;
    PIRO_CHECK_LAUNCH("k_adam");
    return net_pack(n, as_stream(stream));
}

extern "C" int piro_pcnet_stats(piro_pcnet *n, long long *launches)
{
    PIRO_ARG(n && launches, "piro_pcnet_stats: bad arguments");
    *launches = n->launches;
    return PIRO_OK;
}

extern "C" int piro_pcnet_destroy(piro_pcnet *n)
{
    if (!n) return PIRO_OK;
    net_free_ws(n);
    cudaFree(n->w);
    cudaFree(n->wq);
    cudaFree(n->m);
    cudaFree(n->v);
    cudaFree(n->g);
    cudaFree(n->partials);
    cudaFree(n->red);
    cudaFree(n->wpk);
    cudaFree(n->wpk_t);
    cudaFree(n->d_err);
    delete n;
    return PIRO_OK;
}

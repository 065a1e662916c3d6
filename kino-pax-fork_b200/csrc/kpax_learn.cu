// kpax_learn.cu — training and inference entry points of the learned proposal network.
//
// Training runs in FP32 on the SIMT cores with hand-written kernels: a tiled SGEMM for the six
// products of the forward and backward passes, fused bias/SiLU and SiLU-gradient passes, the
// mixture-density loss and its gradient, fixed-order column and loss reductions, and Adam.
// Every reduction has a fixed order, so a training step is deterministic.  Inference for the
// planner runs on the tensor cores (kpax_mlp_tc.cuh) from a BF16 image packed here.
// The reference planner has no learned component; the network replaces nothing in it and only
// reshapes the distribution of the uniform control/duration draws.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "kpax.h"
#include "kpax_internal.h"
#include "kpax_mlp.h"
#include "kpax_mlp_tc.cuh"

using namespace kpax;
using namespace kpax::mlp;

namespace {

// ---------------------------------------------------------------------------------------------
// SIMT kernels

constexpr int kGemmBS = 256, kGT = 64, kGK = 16;

// C[M x N] = op(A) op(B) (+ C when accumulate); op(A)[m][k] = TA ? A[k*lda+m] : A[m*lda+k],
// op(B)[k][n] = TB ? B[n*ldb+k] : B[k*ldb+n].  64x64 tiles, 4x4 outputs per thread, each output
// summed over k in ascending order by one thread.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kGemmBS) k_sgemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                                   const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                                   int accumulate)
{
    __shared__ float As[kGK][kGT + 4], Bs[kGK][kGT + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * kGT, n0 = blockIdx.x * kGT;
    float acc[4][4] = {};
    for(int k0 = 0; k0 < K; k0 += kGK) {
        for(int i = threadIdx.x; i < kGT * kGK; i += kGemmBS) {
            const int mm = TA ? i % kGT : i / kGK, kk = TA ? i / kGT : i % kGK;
            const int gm = m0 + mm, gk = k0 + kk;
            As[kk][mm] = (gm < M && gk < K) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]) : 0.0f;
            const int nn = TB ? i / kGK : i % kGT, kb = TB ? i % kGK : i / kGT;
            const int gn = n0 + nn, gkb = k0 + kb;
            Bs[kb][nn] = (gn < N && gkb < K) ? (TB ? B[(size_t)gn * ldb + gkb] : B[(size_t)gkb * ldb + gn]) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for(int kk = 0; kk < kGK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for(int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i], b[i] = Bs[kk][tx * 4 + i];
#pragma unroll
            for(int i = 0; i < 4; ++i)
#pragma unroll
                for(int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for(int i = 0; i < 4; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if(m < M && n < N) {
                float* c = C + (size_t)m * ldc + n;
                *c = accumulate ? *c + acc[i][j] : acc[i][j];
            }
        }
}

__device__ __forceinline__ float sigmoid_f(float z) { return 1.0f / (1.0f + expf(-z)); }

// Z += b; A = SiLU(Z)  (rows x cols, row-major)
__global__ void k_bias_silu(float* __restrict__ Z, const float* __restrict__ b, float* __restrict__ A, uint32_t rows, int cols)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= (size_t)rows * cols) return;
    const float z = Z[i] + b[i % cols];
    Z[i] = z;
    A[i] = z * sigmoid_f(z);
}

__global__ void k_bias(float* __restrict__ Z, const float* __restrict__ b, uint32_t rows, int cols)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i < (size_t)rows * cols) Z[i] += b[i % cols];
}

// dZ = dA * SiLU'(Z), SiLU'(z) = sig(z) (1 + z (1 - sig(z)))
__global__ void k_silu_grad(const float* __restrict__ dA, const float* __restrict__ Z, float* __restrict__ dZ, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float z = Z[i], s = sigmoid_f(z);
    dZ[i] = dA[i] * (s * (1.0f + z * (1.0f - s)));
}

// Mixture-density negative log-likelihood of the logit targets y (masked dimensions only) and its
// gradient with respect to the 96 outputs, scaled by inv_n.  One thread per sample.
__global__ void k_mdn(const float* __restrict__ O, const float* __restrict__ Y, const float* __restrict__ mask, uint32_t n,
                      float inv_n, float* __restrict__ dO, float* __restrict__ loss)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float* o = O + (size_t)i * kOutPad;
    float y[kDim], m[kDim];
#pragma unroll
    for(int d = 0; d < kDim; ++d) y[d] = Y[(size_t)i * kDim + d], m[d] = mask[d];
    constexpr float kHalfLog2Pi = 0.918938533204672742f;
    float amax = o[0];
#pragma unroll
    for(int k = 1; k < kComp; ++k) amax = fmaxf(amax, o[k * kCompStride]);
    float asum = 0.0f;
#pragma unroll
    for(int k = 0; k < kComp; ++k) asum += expf(o[k * kCompStride] - amax);
    const float alse = amax + logf(asum);
    float lp[kComp];
#pragma unroll
    for(int k = 0; k < kComp; ++k) {
        float acc = o[k * kCompStride] - alse;
#pragma unroll
        for(int d = 0; d < kDim; ++d) {
            const float th = tanhf(o[k * kCompStride + 1 + kDim + d] * (1.0f / kSigHalf));
            const float s = kSigMid + kSigHalf * th, r = (y[d] - o[k * kCompStride + 1 + d]) * expf(-s);
            acc += m[d] * (-0.5f * r * r - s - kHalfLog2Pi);
        }
        lp[k] = acc;
    }
    float lmax = lp[0];
#pragma unroll
    for(int k = 1; k < kComp; ++k) lmax = fmaxf(lmax, lp[k]);
    float lsum = 0.0f;
#pragma unroll
    for(int k = 0; k < kComp; ++k) lsum += expf(lp[k] - lmax);
    const float lse = lmax + logf(lsum);
    loss[i] = -lse;
    float* g = dO + (size_t)i * kOutPad;
#pragma unroll
    for(int k = 0; k < kComp; ++k) {
        const float r = expf(lp[k] - lse), pi = expf(o[k * kCompStride] - alse);
        g[k * kCompStride] = (pi - r) * inv_n;
#pragma unroll
        for(int d = 0; d < kDim; ++d) {
            const float th = tanhf(o[k * kCompStride + 1 + kDim + d] * (1.0f / kSigHalf));
            const float s = kSigMid + kSigHalf * th, is = expf(-s);
            const float e = (y[d] - o[k * kCompStride + 1 + d]) * is;
            g[k * kCompStride + 1 + d] = -r * m[d] * e * is * inv_n;
            g[k * kCompStride + 1 + kDim + d] = -r * m[d] * (e * e - 1.0f) * (1.0f - th * th) * inv_n;
        }
    }
#pragma unroll
    for(int j = kOut; j < kOutPad; ++j) g[j] = 0.0f;
}

// db[c] = sum over rows of dZ[r][c], rows in ascending order (one thread per column).
__global__ void k_colsum(const float* __restrict__ dZ, uint32_t rows, int cols, float* __restrict__ db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= cols) return;
    float acc = 0.0f;
    for(uint32_t r = 0; r < rows; ++r) acc += dZ[(size_t)r * cols + c];
    db[c] = acc;
}

// Sum of n values: 1024 strided partial sums, then a fixed halving tree (one block).
__global__ void __launch_bounds__(1024) k_sum(const float* __restrict__ v, uint32_t n, float* __restrict__ out)
{
    __shared__ float s[1024];
    float acc = 0.0f;
    for(uint32_t i = threadIdx.x; i < n; i += 1024) acc += v[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for(int h = 512; h > 0; h >>= 1) {
        if((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if(threadIdx.x == 0) *out = s[0];
}

// Adam with bias corrections folded into c1 = lr / (1 - b1^t) and c2 = 1 / (1 - b2^t).
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v, size_t n,
                       float b1, float b2, float c1, float c2, float eps)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi, v[i] = vi;
    w[i] -= c1 * mi / (sqrtf(vi * c2) + eps);
}

__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ Y, const uint32_t* __restrict__ idx, uint32_t n,
                         float* __restrict__ Xb, float* __restrict__ Yb)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n * (kInPad + kDim)) return;
    const uint32_t r = i / (kInPad + kDim), c = i % (kInPad + kDim), src = idx[r];
    if(c < (uint32_t)kInPad) Xb[(size_t)r * kInPad + c] = X[(size_t)src * kInPad + c];
    else Yb[(size_t)r * kDim + c - kInPad] = Y[(size_t)src * kDim + c - kInPad];
}

// FP32 master -> BF16 image in the MMA's shared-memory layout, plus the FP32 biases.
__global__ void k_pack(const float* __restrict__ w, uint8_t* __restrict__ img)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n1 = kH * kInPad, n2 = kH * kH, n3 = kOutPad * kH, nb = kH + kH + kOutPad;
    if(i < n1) {
        const uint32_t r = i / kInPad, k = i % kInPad;
        *reinterpret_cast<__nv_bfloat16*>(img + kImgW1 + swz(r, k)) = __float2bfloat16_rn(w[kOffW1 + i]);
    } else if(i < n1 + n2) {
        const uint32_t j = i - n1, r = j / kH, k = j % kH;
        *reinterpret_cast<__nv_bfloat16*>(img + kImgW2 + (k >> 6) * kH * kSlabRowBytes + swz(r, k & 63)) =
          __float2bfloat16_rn(w[kOffW2 + j]);
    } else if(i < n1 + n2 + n3) {
        const uint32_t j = i - n1 - n2, r = j / kH, k = j % kH;
        *reinterpret_cast<__nv_bfloat16*>(img + kImgW3 + (k >> 6) * kOutPad * kSlabRowBytes + swz(r, k & 63)) =
          __float2bfloat16_rn(w[kOffW3 + j]);
    } else if(i < n1 + n2 + n3 + nb) {
        const uint32_t j = i - n1 - n2 - n3;
        const float b = j < (uint32_t)kH ? w[kOffB1 + j] : j < 2u * kH ? w[kOffB2 + j - kH] : w[kOffB3 + j - 2 * kH];
        reinterpret_cast<float*>(img + kImgBias)[j] = b;
    }
}

__global__ void k_features(const KParams p, const uint32_t* __restrict__ occ, const float* __restrict__ states, uint32_t stride,
                           const float* __restrict__ goals, uint32_t n, float* __restrict__ X)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    float s[12], g[3], x[kInPad];
#pragma unroll
    for(int d = 0; d < 12; ++d) s[d] = states[(size_t)i * stride + d];
#pragma unroll
    for(int d = 0; d < 3; ++d) g[d] = goals[(size_t)i * 3 + d];
    features(p, occ, s, g, x);
#pragma unroll
    for(int c = 0; c < kInPad; ++c) X[(size_t)i * kInPad + c] = x[c];
}

// Rows given as arrays of states and goals (tests and offline use of the tensor-core pass).
struct ArraySrc {
    static constexpr bool kDebug = true;
    KParams p;
    const uint32_t* occ;
    const float* states;
    const float* goals;
    uint32_t stride, n;
    float* mix;
    float* out;
    uint16_t* h1;
    uint16_t* h2;
    uint32_t row0;  // first row of the current tile
    __device__ uint32_t tiles() const { return (n + tc::kRows - 1) / tc::kRows; }
    __device__ void seek(uint32_t tile) { row0 = tile * tc::kRows; }
    __device__ uint32_t rows() const { return min((uint32_t)tc::kRows, n - row0); }
    __device__ float* records() const { return mix + (size_t)row0 * kMixFloats; }
    __device__ void row_features(uint32_t r, float x[kInPad]) const
    {
        const uint32_t row = row0 + r;
        float s[12], g[3];
        for(int d = 0; d < 12; ++d) s[d] = states[(size_t)row * stride + d];
        for(int d = 0; d < 3; ++d) g[d] = goals[(size_t)row * 3 + d];
        features(p, occ, s, g, x);
    }
    __device__ void dump_h(int layer, uint32_t r, uint32_t col0, const uint4 bits[2]) const
    {
        uint16_t* dst = layer == 1 ? h1 : h2;
        if(!dst) return;
        uint4* d = reinterpret_cast<uint4*>(dst + (size_t)(row0 + r) * kH + col0);
        d[0] = bits[0], d[1] = bits[1];
    }
    __device__ void dump_out(uint32_t r, uint32_t col, float v) const
    {
        if(out) out[(size_t)(row0 + r) * kOutPad + col] = v;
    }
};

__global__ void __launch_bounds__(tc::kThreads, 1) k_forward_tc(const ArraySrc src, const uint8_t* __restrict__ img, uint32_t* err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    ArraySrc s = src;  // per-thread cursor
    tc::forward(s, img, smem, err);
}

// One warp per R1 workspace cell: the cell is blocked when at least half of the 4x4x4 lattice
// of points at offsets (i + 1/2) / 4 lies inside an obstacle (closed boxes).  `words` must be
// zeroed by the caller.
__global__ void k_occupancy(const KParams p, const Grid g, uint32_t* __restrict__ words)
{
    const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    const int ncell = p.W1 * p.W1 * p.W1;
    if(warp >= ncell) return;
    const int c[3] = {warp % p.W1, (warp / p.W1) % p.W1, warp / (p.W1 * p.W1)};
    uint32_t inside = 0;
#pragma unroll
    for(int h = 0; h < 2; ++h) {
        const int j = lane + 32 * h, i3[3] = {j & 3, (j >> 2) & 3, j >> 4};
        float q[3];
#pragma unroll
        for(int d = 0; d < 3; ++d)
            q[d] = __fadd_rn(p.wmin, __fmul_rn(__fadd_rn((float)c[d], 0.125f * (float)(2 * i3[d] + 1)), p.w1size));
        const int gc = grid_coord(g, q[0]) + g.dim * (grid_coord(g, q[1]) + g.dim * grid_coord(g, q[2]));
        bool in = false;
        for(uint32_t k = __ldg(g.off + gc), e = __ldg(g.off + gc + 1); k < e && !in; ++k) {
            const uint32_t o = __ldg(g.ent + k);
            const float4 a = __ldg(g.obs + 2 * o), m = __ldg(g.obs + 2 * o + 1);
            in = a.x <= q[0] && q[0] <= m.x && a.y <= q[1] && q[1] <= m.y && a.z <= q[2] && q[2] <= m.z;
        }
        inside += __popc(__ballot_sync(0xffffffffu, in));
    }
    if(lane == 0 && inside >= 32) atomicOr(words + (warp >> 5), 1u << (warp & 31));
}

inline uint32_t blocks(size_t n, int bs) { return (uint32_t)((n + bs - 1) / bs); }

}  // namespace

struct kpax_mlp {
    uint32_t max_batch = 0;
    float* w = nullptr;     // FP32 master parameters
    float* g = nullptr;     // gradients
    float* m = nullptr;     // Adam moments
    float* v = nullptr;
    uint8_t* img = nullptr; // BF16 image
    uint32_t* err = nullptr;
    float* mask = nullptr;  // 5 loss-dimension weights
    float* loss = nullptr;  // scalar
    float* h_loss = nullptr;  // pinned scalar
    // activations of a batch
    float *xb = nullptr, *yb = nullptr, *z1 = nullptr, *a1 = nullptr, *z2 = nullptr, *a2 = nullptr, *o = nullptr;
    float *d_o = nullptr, *d_a = nullptr, *d_z = nullptr, *ls = nullptr;
    uint64_t step = 0;
    bool packed = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the last tensor-core pass
    float last_ms = 0.0f;
};

namespace kpax {

// Forward pass of a batch already in (x, n) into the activation buffers.
static kpax_status mlp_forward_f32(kpax_mlp* n, const float* x, uint32_t rows, cudaStream_t st)
{
    const dim3 g1(blocks(kH, kGT), blocks(rows, kGT)), g3(blocks(kOutPad, kGT), blocks(rows, kGT));
    k_sgemm<false, true><<<g1, kGemmBS, 0, st>>>(rows, kH, kInPad, x, kInPad, n->w + kOffW1, kInPad, n->z1, kH, 0);
    k_bias_silu<<<blocks((size_t)rows * kH, 256), 256, 0, st>>>(n->z1, n->w + kOffB1, n->a1, rows, kH);
    k_sgemm<false, true><<<g1, kGemmBS, 0, st>>>(rows, kH, kH, n->a1, kH, n->w + kOffW2, kH, n->z2, kH, 0);
    k_bias_silu<<<blocks((size_t)rows * kH, 256), 256, 0, st>>>(n->z2, n->w + kOffB2, n->a2, rows, kH);
    k_sgemm<false, true><<<g3, kGemmBS, 0, st>>>(rows, kOutPad, kH, n->a2, kH, n->w + kOffW3, kH, n->o, kOutPad, 0);
    k_bias<<<blocks((size_t)rows * kOutPad, 256), 256, 0, st>>>(n->o, n->w + kOffB3, rows, kOutPad);
    count_launch(6);
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

// Loss and gradients (into n->g) of the batch (x, y); the loss sum lands in n->loss.
static kpax_status mlp_backward_f32(kpax_mlp* n, const float* x, const float* y, uint32_t rows, cudaStream_t st)
{
    k_mdn<<<blocks(rows, 128), 128, 0, st>>>(n->o, y, n->mask, rows, 1.0f / (float)rows, n->d_o, n->ls);
    k_sum<<<1, 1024, 0, st>>>(n->ls, rows, n->loss);
    const dim3 gw3(blocks(kH, kGT), blocks(kOutPad, kGT)), gw2(blocks(kH, kGT), blocks(kH, kGT)), gw1(blocks(kInPad, kGT), blocks(kH, kGT));
    const dim3 ga(blocks(kH, kGT), blocks(rows, kGT));
    // layer 3: dW3 = dO^T A2, db3 = colsum(dO), dA2 = dO W3
    k_sgemm<true, false><<<gw3, kGemmBS, 0, st>>>(kOutPad, kH, rows, n->d_o, kOutPad, n->a2, kH, n->g + kOffW3, kH, 0);
    k_colsum<<<1, 128, 0, st>>>(n->d_o, rows, kOutPad, n->g + kOffB3);
    k_sgemm<false, false><<<ga, kGemmBS, 0, st>>>(rows, kH, kOutPad, n->d_o, kOutPad, n->w + kOffW3, kH, n->d_a, kH, 0);
    k_silu_grad<<<blocks((size_t)rows * kH, 256), 256, 0, st>>>(n->d_a, n->z2, n->d_z, (size_t)rows * kH);
    // layer 2
    k_sgemm<true, false><<<gw2, kGemmBS, 0, st>>>(kH, kH, rows, n->d_z, kH, n->a1, kH, n->g + kOffW2, kH, 0);
    k_colsum<<<blocks(kH, 128), 128, 0, st>>>(n->d_z, rows, kH, n->g + kOffB2);
    k_sgemm<false, false><<<ga, kGemmBS, 0, st>>>(rows, kH, kH, n->d_z, kH, n->w + kOffW2, kH, n->d_a, kH, 0);
    k_silu_grad<<<blocks((size_t)rows * kH, 256), 256, 0, st>>>(n->d_a, n->z1, n->d_z, (size_t)rows * kH);
    // layer 1
    k_sgemm<true, false><<<gw1, kGemmBS, 0, st>>>(kH, kInPad, rows, n->d_z, kH, x, kInPad, n->g + kOffW1, kInPad, 0);
    k_colsum<<<blocks(kH, 128), 128, 0, st>>>(n->d_z, rows, kH, n->g + kOffB1);
    count_launch(12);
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

kpax_status launch_occupancy(const KParams& p, const Grid& g, uint32_t* d_words, cudaStream_t st)
{
    const uint32_t cells = (uint32_t)(p.W1 * p.W1 * p.W1);
    KPAX_CUDA(cudaMemsetAsync(d_words, 0, sizeof(uint32_t) * ((cells + 31) / 32), st));
    k_occupancy<<<blocks((size_t)cells * 32, 256), 256, 0, st>>>(p, g, d_words);
    count_launch();
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

const uint8_t* mlp_image(const kpax_mlp* n) { return n && n->packed ? n->img : nullptr; }

}  // namespace kpax

static kpax_status env_occupancy(kpax_env* e, cudaStream_t st)
{
    if(e->d_occ) return KPAX_OK;
    const uint32_t words = (uint32_t)((e->params.W1 * e->params.W1 * e->params.W1 + 31) / 32);
    KPAX_CUDA(cudaMalloc(&e->d_occ, sizeof(uint32_t) * words));
    return launch_occupancy(e->params, e->env.view(), e->d_occ, st);
}

static kpax_status check_learned_env(const kpax_env* e, const char* fn)
{
    if(!e) return set_error("%s: null env", fn), KPAX_EINVAL;
    if(e->params.model != KPAX_MODEL_QUADROTOR) return set_error("%s: the proposal network is defined for the quadrotor", fn), KPAX_EINVAL;
    return KPAX_OK;
}

extern "C" {

kpax_status kpax_mlp_create(uint32_t max_batch, kpax_mlp** out)
{
    if(!out || max_batch == 0 || max_batch > (1u << 22)) return set_error("kpax_mlp_create: bad arguments"), KPAX_EINVAL;
    *out = nullptr;
    kpax_mlp* n = new(std::nothrow) kpax_mlp();
    if(!n) return set_error("kpax_mlp_create: host allocation failed"), KPAX_ENOMEM;
    n->max_batch = max_batch;
    const size_t P = kNumParams, B = max_batch;
    auto fail = [&](kpax_status st) {
        kpax_mlp_destroy(n);
        return st;
    };
#define KPAX_MLP_ALLOC(ptr, bytes)                                                          \
    do {                                                                                    \
        cudaError_t e_ = cudaMalloc(&(ptr), (bytes));                                       \
        if(e_ != cudaSuccess) {                                                             \
            set_error("kpax_mlp_create: %s", cudaGetErrorString(e_));                       \
            return fail(e_ == cudaErrorMemoryAllocation ? KPAX_ENOMEM : KPAX_ECUDA);        \
        }                                                                                   \
    } while(0)
    KPAX_MLP_ALLOC(n->w, P * 4);
    KPAX_MLP_ALLOC(n->g, P * 4);
    KPAX_MLP_ALLOC(n->m, P * 4);
    KPAX_MLP_ALLOC(n->v, P * 4);
    KPAX_MLP_ALLOC(n->img, kImgBytes);
    KPAX_MLP_ALLOC(n->err, 4);
    KPAX_MLP_ALLOC(n->mask, kDim * 4);
    KPAX_MLP_ALLOC(n->loss, 4);
    KPAX_MLP_ALLOC(n->xb, B * kInPad * 4);
    KPAX_MLP_ALLOC(n->yb, B * kDim * 4);
    KPAX_MLP_ALLOC(n->z1, B * kH * 4);
    KPAX_MLP_ALLOC(n->a1, B * kH * 4);
    KPAX_MLP_ALLOC(n->z2, B * kH * 4);
    KPAX_MLP_ALLOC(n->a2, B * kH * 4);
    KPAX_MLP_ALLOC(n->o, B * kOutPad * 4);
    KPAX_MLP_ALLOC(n->d_o, B * kOutPad * 4);
    KPAX_MLP_ALLOC(n->d_a, B * kH * 4);
    KPAX_MLP_ALLOC(n->d_z, B * kH * 4);
    KPAX_MLP_ALLOC(n->ls, B * 4);
#undef KPAX_MLP_ALLOC
    if(cudaMallocHost(&n->h_loss, 4) != cudaSuccess) return set_error("kpax_mlp_create: pinned alloc"), fail(KPAX_ENOMEM);
    if(cudaEventCreate(&n->ev0) != cudaSuccess || cudaEventCreate(&n->ev1) != cudaSuccess)
        return set_error("kpax_mlp_create: event creation failed"), fail(KPAX_ECUDA);
    if(cudaMemset(n->w, 0, P * 4) != cudaSuccess || cudaMemset(n->m, 0, P * 4) != cudaSuccess ||
       cudaMemset(n->v, 0, P * 4) != cudaSuccess || cudaMemset(n->err, 0, 4) != cudaSuccess ||
       cudaMemset(n->img, 0, kImgBytes) != cudaSuccess)
        return set_error("kpax_mlp_create: memset failed"), fail(KPAX_ECUDA);
    const float ones[kDim] = {1, 1, 1, 1, 1};
    if(cudaMemcpy(n->mask, ones, sizeof(ones), cudaMemcpyHostToDevice) != cudaSuccess)
        return set_error("kpax_mlp_create: copy failed"), fail(KPAX_ECUDA);
    *out = n;
    return KPAX_OK;
}

kpax_status kpax_mlp_destroy(kpax_mlp* n)
{
    if(!n) return KPAX_OK;
    void* dev[] = {n->w, n->g, n->m, n->v, n->img, n->err, n->mask, n->loss, n->xb, n->yb, n->z1, n->a1, n->z2, n->a2, n->o, n->d_o, n->d_a, n->d_z, n->ls};
    for(void* p : dev)
        if(p) cudaFree(p);
    if(n->h_loss) cudaFreeHost(n->h_loss);
    if(n->ev0) cudaEventDestroy(n->ev0);
    if(n->ev1) cudaEventDestroy(n->ev1);
    delete n;
    return KPAX_OK;
}

uint32_t kpax_mlp_num_params(void) { return (uint32_t)kNumParams; }

float kpax_mlp_last_propose_ms(const kpax_mlp* n) { return n ? n->last_ms : 0.0f; }

kpax_status kpax_mlp_set_params(kpax_mlp* n, const float* h_params, void* stream)
{
    if(!n || !h_params) return set_error("kpax_mlp_set_params: null argument"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    KPAX_CUDA(cudaMemcpyAsync(n->w, h_params, kNumParams * 4, cudaMemcpyHostToDevice, st));
    KPAX_CUDA(cudaMemsetAsync(n->m, 0, kNumParams * 4, st));
    KPAX_CUDA(cudaMemsetAsync(n->v, 0, kNumParams * 4, st));
    KPAX_CUDA(cudaStreamSynchronize(st));
    n->step = 0;
    return kpax_mlp_pack(n, stream);
}

kpax_status kpax_mlp_get_params(kpax_mlp* n, float* h_params, void* stream)
{
    if(!n || !h_params) return set_error("kpax_mlp_get_params: null argument"), KPAX_EINVAL;
    KPAX_CUDA(cudaMemcpyAsync(h_params, n->w, kNumParams * 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    KPAX_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return KPAX_OK;
}

kpax_status kpax_mlp_set_loss_mask(kpax_mlp* n, const float* h_mask5, void* stream)
{
    if(!n || !h_mask5) return set_error("kpax_mlp_set_loss_mask: null argument"), KPAX_EINVAL;
    KPAX_CUDA(cudaMemcpyAsync(n->mask, h_mask5, kDim * 4, cudaMemcpyHostToDevice, (cudaStream_t)stream));
    KPAX_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return KPAX_OK;
}

kpax_status kpax_mlp_pack(kpax_mlp* n, void* stream)
{
    if(!n) return set_error("kpax_mlp_pack: null network"), KPAX_EINVAL;
    const uint32_t total = kH * kInPad + kH * kH + kOutPad * kH + kH + kH + kOutPad;
    k_pack<<<blocks(total, 256), 256, 0, (cudaStream_t)stream>>>(n->w, n->img);
    count_launch();
    KPAX_CHECK_LAUNCH();
    n->packed = true;
    return KPAX_OK;
}

kpax_status kpax_mlp_forward(kpax_mlp* n, const float* d_x, uint32_t rows, float* d_out, void* stream)
{
    if(!n || !d_x || !d_out || rows > n->max_batch) return set_error("kpax_mlp_forward: bad arguments"), KPAX_EINVAL;
    if(!rows) return KPAX_OK;
    cudaStream_t st = (cudaStream_t)stream;
    kpax_status s = mlp_forward_f32(n, d_x, rows, st);
    if(s != KPAX_OK) return s;
    KPAX_CUDA(cudaMemcpyAsync(d_out, n->o, (size_t)rows * kOutPad * 4, cudaMemcpyDeviceToDevice, st));
    return KPAX_OK;
}

kpax_status kpax_mlp_loss_grad(kpax_mlp* n, const float* d_x, const float* d_y, uint32_t rows, float* h_loss, float* d_grad,
                               void* stream)
{
    if(!n || !d_x || !d_y || !rows || rows > n->max_batch) return set_error("kpax_mlp_loss_grad: bad arguments"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    kpax_status s = mlp_forward_f32(n, d_x, rows, st);
    if(s == KPAX_OK) s = mlp_backward_f32(n, d_x, d_y, rows, st);
    if(s != KPAX_OK) return s;
    if(d_grad) KPAX_CUDA(cudaMemcpyAsync(d_grad, n->g, kNumParams * 4, cudaMemcpyDeviceToDevice, st));
    if(h_loss) {
        KPAX_CUDA(cudaMemcpyAsync(n->h_loss, n->loss, 4, cudaMemcpyDeviceToHost, st));
        KPAX_CUDA(cudaStreamSynchronize(st));
        *h_loss = *n->h_loss / (float)rows;
    }
    return KPAX_OK;
}

kpax_status kpax_mlp_train_step(kpax_mlp* n, const float* d_x, const float* d_y, const uint32_t* d_idx, uint32_t batch, float lr,
                                float* h_loss, void* stream)
{
    if(!n || !d_x || !d_y || !d_idx || !batch || batch > n->max_batch || !(lr > 0.0f))
        return set_error("kpax_mlp_train_step: bad arguments"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    k_gather<<<blocks((size_t)batch * (kInPad + kDim), 256), 256, 0, st>>>(d_x, d_y, d_idx, batch, n->xb, n->yb);
    count_launch();
    kpax_status s = mlp_forward_f32(n, n->xb, batch, st);
    if(s == KPAX_OK) s = mlp_backward_f32(n, n->xb, n->yb, batch, st);
    if(s != KPAX_OK) return s;
    n->step += 1;
    const double b1 = 0.9, b2 = 0.999;
    const float c1 = (float)(lr / (1.0 - pow(b1, (double)n->step))), c2 = (float)(1.0 / (1.0 - pow(b2, (double)n->step)));
    k_adam<<<blocks(kNumParams, 256), 256, 0, st>>>(n->w, n->g, n->m, n->v, kNumParams, (float)b1, (float)b2, c1, c2, 1e-8f);
    count_launch();
    KPAX_CHECK_LAUNCH();
    n->packed = false;
    if(h_loss) {
        KPAX_CUDA(cudaMemcpyAsync(n->h_loss, n->loss, 4, cudaMemcpyDeviceToHost, st));
        KPAX_CUDA(cudaStreamSynchronize(st));
        *h_loss = *n->h_loss / (float)batch;
    }
    return KPAX_OK;
}

kpax_status kpax_mlp_adam_state(kpax_mlp* n, float* h_m, float* h_v, uint64_t* step, void* stream)
{
    if(!n) return set_error("kpax_mlp_adam_state: null network"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    if(h_m) KPAX_CUDA(cudaMemcpyAsync(h_m, n->m, kNumParams * 4, cudaMemcpyDeviceToHost, st));
    if(h_v) KPAX_CUDA(cudaMemcpyAsync(h_v, n->v, kNumParams * 4, cudaMemcpyDeviceToHost, st));
    KPAX_CUDA(cudaStreamSynchronize(st));
    if(step) *step = n->step;
    return KPAX_OK;
}

kpax_status kpax_env_occupancy(kpax_env* e, uint32_t* d_words, void* stream)
{
    kpax_status s = check_learned_env(e, "kpax_env_occupancy");
    if(s != KPAX_OK) return s;
    if(!d_words) return set_error("kpax_env_occupancy: null output"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    s = env_occupancy(e, st);
    if(s != KPAX_OK) return s;
    const uint32_t words = (uint32_t)((e->params.W1 * e->params.W1 * e->params.W1 + 31) / 32);
    KPAX_CUDA(cudaMemcpyAsync(d_words, e->d_occ, sizeof(uint32_t) * words, cudaMemcpyDeviceToDevice, st));
    return KPAX_OK;
}

kpax_status kpax_mlp_features(kpax_env* e, const float* d_states, uint32_t stride, const float* d_goals, uint32_t n,
                              float* d_x, void* stream)
{
    kpax_status s = check_learned_env(e, "kpax_mlp_features");
    if(s != KPAX_OK) return s;
    if(!n) return KPAX_OK;
    if(!d_states || !d_goals || !d_x || stride < 12) return set_error("kpax_mlp_features: bad arguments"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    s = env_occupancy(e, st);
    if(s != KPAX_OK) return s;
    k_features<<<blocks(n, 128), 128, 0, st>>>(e->params, e->d_occ, d_states, stride, d_goals, n, d_x);
    count_launch();
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

kpax_status kpax_mlp_propose(kpax_mlp* net, kpax_env* e, const float* d_states, uint32_t stride, const float* d_goals, uint32_t n,
                             float* d_mix, float* d_out, uint16_t* d_h1, uint16_t* d_h2, void* stream)
{
    kpax_status s = check_learned_env(e, "kpax_mlp_propose");
    if(s != KPAX_OK) return s;
    if(!net || !net->packed) return set_error("kpax_mlp_propose: network not packed"), KPAX_EINVAL;
    if(!n) return KPAX_OK;
    if(!d_states || !d_goals || !d_mix || stride < 12) return set_error("kpax_mlp_propose: bad arguments"), KPAX_EINVAL;
    cudaStream_t st = (cudaStream_t)stream;
    s = env_occupancy(e, st);
    if(s != KPAX_OK) return s;
    KPAX_CUDA(cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::kSmemBytes));
    int dev = 0, sms = 0;
    KPAX_CUDA(cudaGetDevice(&dev));
    KPAX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t tiles = (n + tc::kRows - 1) / tc::kRows;
    ArraySrc src{e->params, e->d_occ, d_states, d_goals, stride, n, d_mix, d_out, d_h1, d_h2};
    KPAX_CUDA(cudaMemsetAsync(net->err, 0, 4, st));
    KPAX_CUDA(cudaEventRecord(net->ev0, st));
    k_forward_tc<<<std::min<uint32_t>(tiles, (uint32_t)sms), tc::kThreads, tc::kSmemBytes, st>>>(src, net->img, net->err);
    count_launch();
    KPAX_CHECK_LAUNCH();
    KPAX_CUDA(cudaEventRecord(net->ev1, st));
    uint32_t h_err = 0;
    KPAX_CUDA(cudaMemcpyAsync(&h_err, net->err, 4, cudaMemcpyDeviceToHost, st));
    KPAX_CUDA(cudaStreamSynchronize(st));
    KPAX_CUDA(cudaEventElapsedTime(&net->last_ms, net->ev0, net->ev1));
    if(h_err) return set_error("kpax_mlp_propose: a tensor-core pipeline wait expired (code %u)", h_err), KPAX_ETIMEOUT;
    return KPAX_OK;
}

}  // extern "C"

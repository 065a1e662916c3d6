// kpax_mlp_tc.cuh — device side of the learned proposal: input features, the mixture record,
// the mixture sampler, and the BF16 tensor-core forward pass (tcgen05, FP32 accumulators in
// tensor memory).
//
// Forward pass: one CTA of 20 warps per SM, persistent over tiles of 128 rows, with roles:
//   warp 0      issues the MMAs (one thread) and owns the tensor-memory allocation
//   warp 1      streams the weights from the global image through a 3-slot ring of 32 KB
//               shared-memory buffers by bulk copies (no tensor map, no multicast)
//   warps 2-3   build the input features of the next tiles into a double-buffered X slab
//   warps 4-19  epilogues: TMEM -> bias + SiLU -> BF16 H slabs, and the mixture records
// Per tile: D1[128x256] = X W1^T (TMEM columns 0..255), H = SiLU(D1 + b1); D2 = H W2^T (columns
// 256..511), H = SiLU(D2 + b2); D3[128x96] = H W3^T (columns 0..95) -> records.  The MMAs of
// K-slab j of layers 2 and 3 start as soon as the epilogue has written H slab j, so epilogues
// overlap the tensor cores.  Operands are K-major with the 128-byte swizzle; every handoff is an
// mbarrier, and every wait is bounded in time: on expiry the kernel records an error bit, lets
// its copies and MMAs drain (bounded), frees its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "kpax_device.cuh"
#include "kpax_mlp.h"

namespace kpax {
namespace mlp {

// ---------------------------------------------------------------------------------------------
// Features, occupancy and mixture sampling (shared by the SIMT and tensor-core paths)

// R1 workspace cell of coordinate x (the expression of region_r1), clamped into the grid.
__device__ __forceinline__ int w1_cell(const KParams& p, float x)
{
    return clampi(f2i(__fdiv_rn(__fmul_rn((float)p.W1, __fsub_rn(x, p.wmin)), p.wspan)), 0, p.W1 - 1);
}

// Occupancy bit of R1 workspace cell (cx, cy, cz); cells outside the grid count as blocked.
__device__ __forceinline__ float occ_bit(const KParams& p, const uint32_t* __restrict__ occ, int cx, int cy, int cz)
{
    if(cx < 0 || cy < 0 || cz < 0 || cx >= p.W1 || cy >= p.W1 || cz >= p.W1) return 1.0f;
    const uint32_t c = (uint32_t)((cz * p.W1 + cy) * p.W1 + cx);
    return (__ldg(occ + (c >> 5)) >> (c & 31)) & 1u ? 1.0f : 0.0f;
}

// x[0..11] = scaled state, x[12..23] = scaled (goal - state) with the goal's non-position
// components zero, x[24..50] = occupancy of the 3x3x3 cells around the state (dx fastest),
// x[51..63] = 0.
__device__ __forceinline__ void features(const KParams& p, const uint32_t* __restrict__ occ, const float s[12],
                                         const float g[3], float x[kInPad])
{
#pragma unroll
    for(int i = 0; i < 12; ++i) {
        x[i] = __fmul_rn(s[i], input_scale(i));
        x[12 + i] = __fmul_rn(__fsub_rn(i < 3 ? g[i] : 0.0f, s[i]), input_scale(i));
    }
    const int cx = w1_cell(p, s[0]), cy = w1_cell(p, s[1]), cz = w1_cell(p, s[2]);
#pragma unroll
    for(int j = 0; j < 27; ++j) x[24 + j] = occ_bit(p, occ, cx + j % 3 - 1, cy + (j / 3) % 3 - 1, cz + j / 9 - 1);
#pragma unroll
    for(int i = kIn; i < kInPad; ++i) x[i] = 0.0f;
}

// Draws of child `index` from the mixture record (network outputs) of its entry.  u[] holds the
// plain uniform draws on entry; they are kept when the Philox stream-3 uniform is <= eps
// (probability eps), else u[0..4] are replaced by sigmoid(mu + sigma * n): the component is the
// first whose cumulative softmax weight reaches a stream-3 uniform (the last one if none), sigma
// = exp(kSigMid + kSigHalf * tanh(raw / kSigHalf)), and n are Box-Muller normals from streams 3
// and 4.  Only the drawn component's sigmas are evaluated.  u[5] (frontier acceptance) is never
// changed.
__device__ __forceinline__ void mixture_draws(const KParams& p, const float* __restrict__ rec, float eps, uint32_t stream,
                                              uint32_t iter, uint32_t index, float u[6])
{
    const U4 a = philox(index, iter, 3u, stream, p.seed_lo, p.seed_hi);
    if(u01(a.x) <= eps) return;
    const U4 b = philox(index, iter, 4u, stream, p.seed_lo, p.seed_hi);
    float lg[kComp], mx = -INFINITY;
#pragma unroll
    for(int j = 0; j < kComp; ++j) lg[j] = __ldg(rec + j * kCompStride), mx = fmaxf(mx, lg[j]);
    float e[kComp], tot = 0.0f;
#pragma unroll
    for(int j = 0; j < kComp; ++j) e[j] = expf(lg[j] - mx), tot += e[j];
    const float target = u01(a.y) * tot;  // component: first with cumulative weight sum >= target
    float acc = 0.0f;
    int k = kComp - 1;
    for(int j = 0; j < kComp - 1; ++j) {
        acc += e[j];
        if(acc >= target) {
            k = j;
            break;
        }
    }
    const uint32_t bm[6] = {a.z, a.w, b.x, b.y, b.z, b.w};
    float n[6];
#pragma unroll
    for(int i = 0; i < 3; ++i) {
        const float r = sqrtf(-2.0f * logf(u01(bm[2 * i])));
        float sn, cs;
        sincospif(2.0f * u01(bm[2 * i + 1]), &sn, &cs);
        n[2 * i] = r * cs, n[2 * i + 1] = r * sn;
    }
    const float* c = rec + k * kCompStride;
#pragma unroll
    for(int d = 0; d < kDim; ++d) {
        // fused multiply-adds written out: the same draws in every kernel this is inlined into
        const float sg = expf(__fmaf_rn(kSigHalf, tanhf(__fmul_rn(__ldg(c + 1 + kDim + d), 1.0f / kSigHalf)), kSigMid));
        const float z = __fmaf_rn(sg, n[d], __ldg(c + 1 + d));
        const float v = 1.0f / (1.0f + expf(-z));
        u[d] = fminf(fmaxf(v, 5.9604645e-8f), 1.0f);
    }
}

// ---------------------------------------------------------------------------------------------
// tcgen05 forward pass

namespace tc {

constexpr int kThreads = 640, kRows = 128, kStages = 3, kEpiThreads = 512, kFeatThreads = 64;
constexpr uint32_t kRingBytes = 32768, kSlabBytes = kRows * kSlabRowBytes;  // 16 KB: 128 rows x 64 BF16
constexpr uint32_t kSmX = 0, kSmH = kSmX + 2 * kSlabBytes, kSmRing = kSmH + 4 * kSlabBytes;
constexpr uint32_t kSmBias = kSmRing + kStages * kRingBytes;
constexpr uint32_t kRecStride = kMixFloats + 1;  // staging row stride (odd: conflict-free)
// mbarriers: ring full / empty, X full / empty, layer accumulators, H slabs of layers 1 and 2,
// tensor memory free (end of a tile's record epilogue), drain
constexpr int kBarRF = 0, kBarRE = 3, kBarXF = 6, kBarXE = 8, kBarD1 = 10, kBarD2 = 11, kBarD3 = 12, kBarHF = 13, kBarGF = 17,
              kBarTF = 21, kBarFin = 22, kNumBars = 23;
constexpr uint32_t kSmBar = kSmBias + (kH + kH + kOutPad) * 4, kSmTmem = kSmBar + kNumBars * 8, kSmUsed = kSmTmem + 16;
constexpr uint32_t kSmemBytes = kSmUsed + 1024;  // slack for the 1024-byte alignment of the slabs
constexpr int kChunks = 9;                       // W1, 4 slabs of W2, 4 slabs of W3
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr uint32_t kErrWait = 4u;
static_assert(kRows * kRecStride * 4 <= 4 * kSlabBytes, "record staging must fit in the H slabs");

__host__ __device__ constexpr uint32_t chunk_src(int c)
{
    return c == 0 ? kImgW1 : c <= 4 ? kImgW2 + (uint32_t)(c - 1) * kH * kSlabRowBytes : kImgW3 + (uint32_t)(c - 5) * kOutPad * kSlabRowBytes;
}
__host__ __device__ constexpr uint32_t chunk_bytes(int c) { return c <= 4 ? kH * kSlabRowBytes : kOutPad * kSlabRowBytes; }

// Instruction descriptor of kind::f16: FP32 accumulate, BF16 A and B, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc(uint32_t n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row atoms 1024 bytes apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
           ((uint64_t)2 << 61);
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
    return ok != 0u;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    if(mbar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while(!mbar_try(bar, parity))
        if(now_ns() - t0 > kWaitNs) return false;
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst), "l"(src),
                 "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc)
{
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
    for(int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tmem_ld1(uint32_t taddr)
{
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// SiLU of two values: x * sigmoid(x) = h + h * tanh(h) with h = x / 2, the tanh of both halves
// in one MUFU operation (tanh.approx.bf16x2: h rounded to BF16, tanh returned in BF16), so
// |error| < 2^-8 |x| before the result is rounded to BF16.
__device__ __forceinline__ void silu2(float& x0, float& x1)
{
    const float h0 = 0.5f * x0, h1 = 0.5f * x1;
    const __nv_bfloat162 hb = __floats2bfloat162_rn(h0, h1);
    uint32_t tin = *reinterpret_cast<const uint32_t*>(&hb), tout;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(tout) : "r"(tin));
    const __nv_bfloat162 tb = *reinterpret_cast<const __nv_bfloat162*>(&tout);
    x0 = fmaf(h0, __low2float(tb), h0);
    x1 = fmaf(h1, __high2float(tb), h1);
}

// Named barrier of the 512 epilogue threads; the OR form returns a value uniform across them.
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 512;" ::: "memory"); }
__device__ __forceinline__ bool epi_sync_or(bool v)
{
    uint32_t r;
    asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.or.pred p, 1, 512, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(r)
      : "r"((uint32_t)v)
      : "memory");
    return r != 0u;
}

// Stores 16 consecutive columns (col0 a multiple of 16) of row r into the swizzled slabs at base.
__device__ __forceinline__ void store_row16(uint8_t* base, uint32_t r, uint32_t col0, const float v[16], uint4* packed = nullptr)
{
    uint8_t* slab = base + (col0 >> 6) * kSlabBytes;
    const uint32_t k = col0 & 63u;
    const uint4 lo = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    const uint4 hi = make_uint4(pack_bf16(v[8], v[9]), pack_bf16(v[10], v[11]), pack_bf16(v[12], v[13]), pack_bf16(v[14], v[15]));
    *reinterpret_cast<uint4*>(slab + swz(r, k)) = lo;
    *reinterpret_cast<uint4*>(slab + swz(r, k + 8)) = hi;
    if(packed) packed[0] = lo, packed[1] = hi;
}

// Source of rows, a tile of kRows rows at a time (each thread keeps its own copy):
// `uint32_t tiles()` (tiles in all), `void seek(uint32_t tile)` (a thread visits its tiles in
// increasing order), and for the current tile `uint32_t rows()` (1..kRows valid rows),
// `void row_features(uint32_t r, float x[64])` (row r of the tile), `float* records()` (the
// tile's rows() records of kMixFloats floats); for debug dumps `kDebug` with
// `dump_h(layer, r, col0, const uint4 bits[2])` (16 BF16 values) and `dump_out(r, col, v)`.
// CTA b takes tiles b, b + gridDim.x, ...
// Returns false in every thread of a CTA whose pipeline gave up a wait (err has kErrWait set).
template <class Src>
__device__ bool forward(Src& src, const uint8_t* __restrict__ img, uint8_t* smem_raw, uint32_t* __restrict__ err)
{
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t ntiles = src.tiles();
    if(blockIdx.x >= ntiles) return true;
    const uint32_t my_tiles = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    uint8_t* sm = smem_raw + pad;
    const uint32_t sb = raw + pad;
    const float* bias = reinterpret_cast<const float*>(sm + kSmBias);
    auto bar = [&](int i) { return sb + kSmBar + 8u * (uint32_t)i; };
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kSmTmem);
    volatile uint32_t* s_err = s_tmem + 1;

    if(warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sb + kSmTmem), "r"(512u) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if(tid == 32) {
        for(int s = 0; s < kStages; ++s) mbar_init(bar(kBarRF + s), 1), mbar_init(bar(kBarRE + s), 1);
        for(int b = 0; b < 2; ++b) mbar_init(bar(kBarXF + b), kFeatThreads), mbar_init(bar(kBarXE + b), 1);
        mbar_init(bar(kBarD1), 1), mbar_init(bar(kBarD2), 1), mbar_init(bar(kBarD3), 1);
        for(int j = 0; j < 4; ++j) mbar_init(bar(kBarHF + j), 128), mbar_init(bar(kBarGF + j), 128);
        mbar_init(bar(kBarTF), kEpiThreads), mbar_init(bar(kBarFin), 1);
        *s_err = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for(uint32_t i = tid; i < (uint32_t)(kH + kH + kOutPad); i += blockDim.x)
        reinterpret_cast<float*>(sm + kSmBias)[i] = __ldg(reinterpret_cast<const float*>(img + kImgBias) + i);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_tmem;
    auto fail = [&]() {
        atomicOr(err, kErrWait);
        *s_err = 1u;
    };

    if(warp == 0) {
        // ---------------------------------------------------------------- MMA issuer
        if(lane == 0) {
            uint32_t g = 0;  // chunk sequence number
            auto chunk = [&](uint32_t a_addr, uint32_t d_col, uint32_t nn, bool acc) -> bool {
                const uint32_t s = g % kStages;
                if(!mbar_wait(bar(kBarRF + s), (g / kStages) & 1u)) return false;
                fence_after();
                const uint32_t b_addr = sb + kSmRing + s * kRingBytes;
#pragma unroll
                for(uint32_t kk = 0; kk < 4; ++kk)
                    mma(tmem + d_col, sdesc(a_addr + 32u * kk), sdesc(b_addr + 32u * kk), idesc(nn), (acc || kk) ? 1u : 0u);
                commit(bar(kBarRE + s));
                ++g;
                return true;
            };
            for(uint32_t i = 0; i < my_tiles && !*s_err; ++i) {
                const uint32_t b = i & 1u;
                bool ok = mbar_wait(bar(kBarXF + b), (i >> 1) & 1u);
                if(ok && i > 0) ok = mbar_wait(bar(kBarTF), (i - 1) & 1u);  // tile i-1 done with TMEM
                if(ok) ok = chunk(sb + kSmX + b * kSlabBytes, 0u, kH, false);
                if(!ok) {
                    fail();
                    break;
                }
                commit(bar(kBarXE + b));
                commit(bar(kBarD1));
                for(uint32_t j = 0; j < 4 && ok; ++j) {
                    ok = mbar_wait(bar(kBarHF + j), i & 1u);
                    if(ok) fence_after(), ok = chunk(sb + kSmH + j * kSlabBytes, 256u, kH, j > 0);
                }
                if(ok) commit(bar(kBarD2));
                for(uint32_t j = 0; j < 4 && ok; ++j) {
                    ok = mbar_wait(bar(kBarGF + j), i & 1u);
                    if(ok) fence_after(), ok = chunk(sb + kSmH + j * kSlabBytes, 0u, kOutPad, j > 0);
                }
                if(!ok) {
                    fail();
                    break;
                }
                commit(bar(kBarD3));
            }
            commit(bar(kBarFin));  // arrives once every MMA issued above has completed
            mbar_wait(bar(kBarFin), 0u);
        }
        __syncwarp();
    } else if(warp == 1) {
        // ---------------------------------------------------------------- weight producer
        if(lane == 0) {
            const uint32_t total = my_tiles * kChunks;
            uint32_t g = 0;
            for(; g < total && !*s_err; ++g) {
                const uint32_t s = g % kStages;
                if(g >= (uint32_t)kStages && !mbar_wait(bar(kBarRE + s), (g / kStages - 1) & 1u)) {
                    fail();
                    break;
                }
                const int c = (int)(g % kChunks);
                bulk_load(sb + kSmRing + s * kRingBytes, img + chunk_src(c), chunk_bytes(c), bar(kBarRF + s));
            }
            for(uint32_t h = g > (uint32_t)kStages ? g - kStages : 0u; h < g; ++h)  // drain copies in flight
                mbar_wait(bar(kBarRF + h % kStages), (h / kStages) & 1u);
        }
        __syncwarp();
    } else if(warp < 4) {
        // ---------------------------------------------------------------- features
        const uint32_t ft = tid - 64u;
        for(uint32_t i = 0; i < my_tiles && !*s_err; ++i) {
            const uint32_t b = i & 1u, tile = blockIdx.x + i * gridDim.x;
            if(i >= 2 && !mbar_wait(bar(kBarXE + b), ((i >> 1) - 1) & 1u)) {
                fail();
                break;
            }
            src.seek(tile);
            const uint32_t nr = src.rows();
            for(uint32_t r = ft; r < (uint32_t)kRows; r += kFeatThreads) {
                float x[kInPad];
                if(r < nr) src.row_features(r, x);
                else
#pragma unroll
                    for(int c = 0; c < kInPad; ++c) x[c] = 0.0f;
#pragma unroll
                for(int c = 0; c < kInPad; c += 16) store_row16(sm + kSmX + b * kSlabBytes, r, (uint32_t)c, x + c);
            }
            fence_async_smem();
            mbar_arrive(bar(kBarXF + b));
        }
    } else {
        // ---------------------------------------------------------------- epilogues
        const uint32_t q = warp & 3u, cg = (warp - 4u) >> 2, r = 32u * q + lane;
        const uint32_t t_lane = tmem + ((32u * q) << 16);
        float* stg = reinterpret_cast<float*>(sm + kSmH);
        for(uint32_t i = 0; i < my_tiles; ++i) {
            src.seek(blockIdx.x + i * gridDim.x);
            const uint32_t nr = src.rows();
            // hidden layers: D (columns d_col..) -> SiLU -> H slab cg; arrive `ready`
            auto hidden = [&](int layer, int bar_d, uint32_t d_col, const float* b, int bar_ready) -> bool {
                const bool ok = mbar_wait(bar(bar_d), i & 1u);
                if(epi_sync_or(!ok || *s_err)) return false;
                fence_after();
#pragma unroll
                for(int half = 0; half < 2; ++half) {
                    float v[2][16];
#pragma unroll
                    for(int cc = 0; cc < 2; ++cc) tmem_ld16(t_lane + d_col + cg * 64u + 32u * half + 16u * cc, v[cc]);
                    tmem_wait_ld();
#pragma unroll
                    for(int cc = 0; cc < 2; ++cc) {
                        const uint32_t col0 = cg * 64u + 32u * half + 16u * cc;
#pragma unroll
                        for(int k = 0; k < 16; k += 2) {
                            v[cc][k] += b[col0 + k], v[cc][k + 1] += b[col0 + k + 1];
                            silu2(v[cc][k], v[cc][k + 1]);
                        }
                        uint4 bits[2];
                        store_row16(sm + kSmH, r, col0, v[cc], bits);
                        if constexpr(Src::kDebug) {
                            if(r < nr) src.dump_h(layer, r, col0, bits);
                        }
                    }
                }
                fence_async_smem();
                fence_before();
                mbar_arrive(bar(bar_ready + (int)cg));
                return true;
            };
            if(!hidden(1, kBarD1, 0u, bias, kBarHF)) break;
            if(!hidden(2, kBarD2, 256u, bias + kH, kBarGF)) break;
            // records: the outputs plus biases; warp group cg stages columns 22cg .. 22cg + 21
            const bool ok = mbar_wait(bar(kBarD3), i & 1u);
            if(epi_sync_or(!ok || *s_err)) break;
            fence_after();
            constexpr int kCols = kOut / 4;
            float o[kCols];
#pragma unroll
            for(int c = 0; c < kCols; ++c) o[c] = tmem_ld1(t_lane + cg * (uint32_t)kCols + (uint32_t)c);
            tmem_wait_ld();
            fence_before();
            mbar_arrive(bar(kBarTF));
            const float* b3 = bias + 2 * kH + cg * kCols;
            float* rec = stg + r * kRecStride + cg * kCols;
#pragma unroll
            for(int c = 0; c < kCols; ++c) rec[c] = o[c] + b3[c];
            if constexpr(Src::kDebug) {
                if(r < nr)
                    for(int c = 0; c < kCols; ++c) src.dump_out(r, cg * (uint32_t)kCols + (uint32_t)c, o[c] + b3[c]);
            }
            epi_sync();
            // coalesced copy of the tile's records (contiguous rows) to global memory
            float* dst = src.records();
            for(uint32_t f = tid - 128u; f < nr * (uint32_t)kMixFloats; f += (uint32_t)kEpiThreads)
                dst[f] = stg[(f / kMixFloats) * kRecStride + f % kMixFloats];
            epi_sync();  // staging read before the next tile's epilogue rewrites H
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if(warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    return *s_err == 0u;
}

}  // namespace tc
}  // namespace mlp
}  // namespace kpax

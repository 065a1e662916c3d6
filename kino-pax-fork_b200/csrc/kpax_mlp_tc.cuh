// kpax_mlp_tc.cuh — device side of the learned proposal: input features, obstacle occupancy of
// the R1 workspace cells, the mixture record, the mixture sampler, and the BF16 tensor-core
// forward pass (tcgen05, FP32 accumulators in tensor memory).
//
// Forward pass, one CTA of 512 threads per SM, persistent over tiles of 128 rows:
//   features   threads 0..127 build one row each and store it as BF16 into the swizzled X slab
//   layer 1    D1[128x256] = X W1^T           (4 MMAs of K=16, N=256; TMEM columns 0..255)
//   epilogue   H = SiLU(D1 + b1) as BF16 into four swizzled slabs (16 warps, 64 columns each)
//   layer 2    D2[128x256] = H W2^T           (16 MMAs; TMEM columns 256..511)
//   epilogue   H = SiLU(D2 + b2)
//   layer 3    D3[128x96]  = H W3^T           (16 MMAs, N=96; TMEM columns 0..95)
//   epilogue   threads 0..127 turn their row's 88 outputs (+ b3) into a mixture record
// Weights stream from the global image through a two-slot ring of 32 KB shared-memory buffers
// by bulk copies (no tensor map, no multicast); one thread issues the copies and the MMAs and
// tracks both with mbarriers.  Every wait is bounded in time: on expiry the kernel records an
// error bit, waits (bounded) for its copies and MMAs, frees its tensor memory and returns.
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

// Mixture record from the 88 network outputs (biases included): cumulative component weights
// (softmax in component order, last entry exactly 1), means, sigmas = exp(s) with
// s = kSigMid + kSigHalf * tanh(raw * (1 / kSigHalf)).
__device__ __forceinline__ void mixture_record(const float* o, float* __restrict__ rec)
{
    float mx = o[0];
#pragma unroll
    for(int k = 1; k < kComp; ++k) mx = fmaxf(mx, o[k * kCompStride]);
    float e[kComp], tot = 0.0f;
#pragma unroll
    for(int k = 0; k < kComp; ++k) e[k] = expf(o[k * kCompStride] - mx), tot += e[k];
    float acc = 0.0f;
#pragma unroll
    for(int k = 0; k < kComp; ++k) {
        acc += e[k];
        rec[kMixCdf + k] = k == kComp - 1 ? 1.0f : acc / tot;
    }
#pragma unroll
    for(int k = 0; k < kComp; ++k)
#pragma unroll
        for(int d = 0; d < kDim; ++d) {
            rec[kMixMu + k * kDim + d] = o[k * kCompStride + 1 + d];
            const float s = kSigMid + kSigHalf * tanhf(o[k * kCompStride + 1 + kDim + d] * (1.0f / kSigHalf));
            rec[kMixSigma + k * kDim + d] = expf(s);
        }
}

// Draws of child `index` from the mixture record of its entry.  u[] holds the plain uniform
// draws on entry; they are kept when the Philox stream-3 uniform is <= eps (probability eps), else u[0..4] are
// replaced by sigmoid(mu + sigma * n) of a component picked by the cumulative weights, with
// Box-Muller normals from Philox streams 3 and 4.  u[5] (frontier acceptance) is never changed.
__device__ __forceinline__ void mixture_draws(const KParams& p, const float* __restrict__ rec, float eps, uint32_t stream,
                                              uint32_t iter, uint32_t index, float u[6])
{
    const U4 a = philox(index, iter, 3u, stream, p.seed_lo, p.seed_hi);
    if(u01(a.x) <= eps) return;
    const U4 b = philox(index, iter, 4u, stream, p.seed_lo, p.seed_hi);
    const float uc = u01(a.y);
    int k = 0;
#pragma unroll
    for(int j = 0; j < kComp - 1; ++j) k += __ldg(rec + kMixCdf + j) < uc ? 1 : 0;
    const uint32_t bm[6] = {a.z, a.w, b.x, b.y, b.z, b.w};
    float n[6];
#pragma unroll
    for(int i = 0; i < 3; ++i) {
        const float r = sqrtf(-2.0f * logf(u01(bm[2 * i])));
        float sn, cs;
        sincospif(2.0f * u01(bm[2 * i + 1]), &sn, &cs);
        n[2 * i] = r * cs, n[2 * i + 1] = r * sn;
    }
#pragma unroll
    for(int d = 0; d < kDim; ++d) {
        const float z = __ldg(rec + kMixMu + k * kDim + d) + __ldg(rec + kMixSigma + k * kDim + d) * n[d];
        const float v = 1.0f / (1.0f + expf(-z));
        u[d] = fminf(fmaxf(v, 5.9604645e-8f), 1.0f);
    }
}

// ---------------------------------------------------------------------------------------------
// tcgen05 forward pass

namespace tc {

constexpr int kThreads = 512, kRows = 128;
constexpr uint32_t kRingBytes = 32768;
constexpr uint32_t kSmX = 0, kSmH = 16384, kSmRing = kSmH + 65536, kSmBias = kSmRing + 2 * kRingBytes;
constexpr uint32_t kSmBar = kSmBias + (kH + kH + kOutPad) * 4, kSmTmem = kSmBar + 8 * 8, kSmUsed = kSmTmem + 16;
constexpr uint32_t kSmemBytes = kSmUsed + 1024;  // slack for the 1024-byte alignment of the slabs
constexpr int kChunks = 9;                       // W1, 4 slabs of W2, 4 slabs of W3
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr uint32_t kErrWait = 4u;

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

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ float silu(float x) { return __fdividef(x, 1.0f + __expf(-x)); }

// Stores 16 consecutive columns (col0 a multiple of 16) of row r into the swizzled slabs at base.
__device__ __forceinline__ void store_row16(uint8_t* base, uint32_t r, uint32_t col0, const float v[16])
{
    uint8_t* slab = base + (col0 >> 6) * (kRows * kSlabRowBytes);
    const uint32_t k = col0 & 63u;
    const uint4 lo = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    const uint4 hi = make_uint4(pack_bf16(v[8], v[9]), pack_bf16(v[10], v[11]), pack_bf16(v[12], v[13]), pack_bf16(v[14], v[15]));
    *reinterpret_cast<uint4*>(slab + swz(r, k)) = lo;
    *reinterpret_cast<uint4*>(slab + swz(r, k + 8)) = hi;
}

// Source of rows: `uint32_t count()`, `void row_features(uint32_t row, float x[64])`,
// `void store(uint32_t row, const float o[96])`, and for debug dumps `kDebug` with
// `dump_h(layer, row, const uint8_t* slabs, uint32_t r)`.
template <class Src>
__device__ void forward(Src& src, const uint8_t* __restrict__ img, uint8_t* smem_raw, uint32_t* __restrict__ err)
{
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t n = src.count();
    const uint32_t ntiles = (n + kRows - 1) / kRows;
    if(blockIdx.x >= ntiles) return;
    const uint32_t my_tiles = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
    const uint32_t total = my_tiles * kChunks;
    const uint32_t raw = (uint32_t)__cvta_generic_to_shared(smem_raw);
    const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
    uint8_t* sm = smem_raw + pad;
    const uint32_t sbase = raw + pad;
    const float* bias = reinterpret_cast<const float*>(sm + kSmBias);
    const uint32_t bar_full = sbase + kSmBar, bar_empty = bar_full + 16, bar_done = bar_full + 32;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kSmTmem);
    volatile uint32_t* s_err = s_tmem + 1;

    if(warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kSmTmem), "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if(tid == 0) {
        for(int i = 0; i < 2; ++i) mbar_init(bar_full + 8 * i, 1), mbar_init(bar_empty + 8 * i, 1);
        mbar_init(bar_done, 1);
        *s_err = 0u;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for(uint32_t i = tid; i < (uint32_t)(kH + kH + kOutPad); i += blockDim.x)
        reinterpret_cast<float*>(sm + kSmBias)[i] = __ldg(reinterpret_cast<const float*>(img + kImgBias) + i);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *s_tmem;

    // chunk g of this CTA's sequence lands in ring slot g & 1; its phases have parity (g >> 1) & 1
    uint32_t issued = 0, consumed = 0, done_cnt = 0;
    auto issue = [&]() {
        const uint32_t slot = issued & 1u;
        const int c = (int)(issued % kChunks);
        bulk_load(sbase + kSmRing + slot * kRingBytes, img + chunk_src(c), chunk_bytes(c), bar_full + 8 * slot);
        ++issued;
    };
    auto fail = [&]() { atomicOr(err, kErrWait), *s_err = 1u; };
    if(tid == 0)
        while(issued < total && issued < 2) issue();

    // MMAs of one chunk: A = the K slab at a_addr (K = 64), B = the ring slot; accumulate after
    // the first K step when `acc`.  Issued by thread 0 only.
    auto run_chunk = [&](uint32_t a_addr, uint32_t d_col, uint32_t nn, bool acc, bool last) -> bool {
        const uint32_t slot = consumed & 1u, par = (consumed >> 1) & 1u;
        if(!mbar_wait(bar_full + 8 * slot, par)) return false;
        fence_after();
        const uint32_t b_addr = sbase + kSmRing + slot * kRingBytes;
#pragma unroll
        for(uint32_t kk = 0; kk < 4; ++kk)
            mma(tmem + d_col, sdesc(a_addr + 32u * kk), sdesc(b_addr + 32u * kk), idesc(nn), (acc || kk) ? 1u : 0u);
        commit(bar_empty + 8 * slot);
        if(last) commit(bar_done);
        ++consumed;
        if(!mbar_wait(bar_empty + 8 * slot, par)) return false;  // slot free: refill it
        if(issued < total) issue();
        return true;
    };
    // Epilogue of layers 1 and 2: 16 warps, warp w reads TMEM lanes 32*(w%4).. and 64 columns.
    auto hidden_epilogue = [&](uint32_t d_col, const float* b) {
        const uint32_t q = warp & 3u, cg = warp >> 2, r = 32u * q + lane;
        float v[4][16];
#pragma unroll
        for(int cc = 0; cc < 4; ++cc) tmem_ld16(tmem + ((32u * q) << 16) + d_col + cg * 64u + 16u * cc, v[cc]);
        tmem_wait_ld();
#pragma unroll
        for(int cc = 0; cc < 4; ++cc) {
            const uint32_t col0 = cg * 64u + 16u * cc;
#pragma unroll
            for(int i = 0; i < 16; ++i) v[cc][i] = silu(v[cc][i] + b[col0 + i]);
            store_row16(sm + kSmH, r, col0, v[cc]);
        }
    };
    // All threads wait for the layer's MMAs; returns a CTA-uniform verdict so that the warp-wide
    // TMEM loads that follow are executed by whole warps or not at all.
    auto layer_sync = [&]() -> bool {
        bool ok = true;
        if(!*s_err) ok = mbar_wait(bar_done, done_cnt & 1u);
        ++done_cnt;
        fence_after();
        const bool bad = __syncthreads_or(!ok || *s_err) != 0;
        if(bad && tid == 0) fail();
        return !bad;
    };
    auto publish_smem = [&]() {  // generic-proxy writes -> visible to the MMA; TMEM reads ordered
        fence_async_smem();
        fence_before();
        __syncthreads();
    };

    for(uint32_t t = 0; t < my_tiles; ++t) {
        const uint32_t tile = blockIdx.x + t * gridDim.x;
        if(tid < (uint32_t)kRows) {
            const uint32_t row = tile * kRows + tid;
            float x[kInPad];
            if(row < n) src.row_features(row, x);
            else
#pragma unroll
                for(int i = 0; i < kInPad; ++i) x[i] = 0.0f;
#pragma unroll
            for(int c = 0; c < kInPad; c += 16) store_row16(sm + kSmX, tid, (uint32_t)c, x + c);
        }
        publish_smem();
        if(tid == 0) {
            fence_after();
            if(!run_chunk(sbase + kSmX, 0u, kH, false, true)) fail();
        }
        if(!layer_sync()) break;
        hidden_epilogue(0u, bias);
        publish_smem();
        if constexpr(Src::kDebug) {
            if(tid < (uint32_t)kRows && tile * kRows + tid < n) src.dump_h(1, tile * kRows + tid, sm + kSmH, tid);
        }
        if(tid == 0) {
            fence_after();
            for(uint32_t j = 0; j < 4; ++j)
                if(!run_chunk(sbase + kSmH + j * (kRows * kSlabRowBytes), 256u, kH, j > 0, j == 3)) {
                    fail();
                    break;
                }
        }
        if(!layer_sync()) break;
        // H is rewritten only after every layer-2 MMA has completed (bar_done)
        hidden_epilogue(256u, bias + kH);
        publish_smem();
        if constexpr(Src::kDebug) {
            if(tid < (uint32_t)kRows && tile * kRows + tid < n) src.dump_h(2, tile * kRows + tid, sm + kSmH, tid);
        }
        if(tid == 0) {
            fence_after();
            for(uint32_t j = 0; j < 4; ++j)
                if(!run_chunk(sbase + kSmH + j * (kRows * kSlabRowBytes), 0u, kOutPad, j > 0, j == 3)) {
                    fail();
                    break;
                }
        }
        if(!layer_sync()) break;
        if(warp < 4) {
            const uint32_t r = 32u * warp + lane, row = tile * kRows + r;
            float o[kOutPad];
#pragma unroll
            for(int cc = 0; cc < kOutPad / 16; ++cc) tmem_ld16(tmem + ((32u * warp) << 16) + 16u * cc, o + 16 * cc);
            tmem_wait_ld();
            if(row < n) {
#pragma unroll
                for(int i = 0; i < kOutPad; ++i) o[i] += bias[2 * kH + i];
                src.store(row, o);
            }
        }
        fence_before();
        __syncthreads();
    }
    // teardown: on an error, let copies and MMAs in flight finish (bounded) before freeing TMEM
    if(tid == 0 && *s_err) {
        for(uint32_t g = consumed; g < issued; ++g) mbar_wait(bar_full + 8 * (g & 1u), (g >> 1) & 1u);
        commit(bar_empty);  // arrives on slot 0 once every MMA issued so far is complete
        mbar_wait(bar_empty, ((consumed + 1u) >> 1) & 1u);
    }
    fence_before();
    __syncthreads();
    fence_after();
    if(warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
}

}  // namespace tc
}  // namespace mlp
}  // namespace kpax

// kpax_env.cu — obstacle grid build and the kernel-level batch entry points.
//
// The reference keeps a fixed 16-slot list per 5 m cell and rebuilds it with atomics every
// iteration (spatialHash.cu:9-67, KPAX.cu:306), silently dropping entries past 16 in nondeterministic order.  Here
// the grid is compressed sparse rows (count -> scan -> fill), holds every (cell, obstacle)
// pair and is built once per plan.  Query verdicts equal the brute-force isMotionValid
// (collisionCheck.cu:49-62) for every box: the cell map is monotone, so any strictly
// overlapping obstacle shares at least one cell with the box.
#include <stdio.h>
#include <limits.h>
#include <algorithm>
#include <string.h>

#include <mutex>
#include <new>

#include "kpax_internal.h"

namespace kpax {

std::atomic<uint64_t> g_launches{0};

namespace {

__device__ __forceinline__ void obstacle_cells(const Grid& g, const float4& lo, const float4& hi, int c0[3], int c1[3])
{
    c0[0] = grid_coord(g, lo.x), c0[1] = grid_coord(g, lo.y), c0[2] = grid_coord(g, lo.z);
    c1[0] = grid_coord(g, hi.x), c1[1] = grid_coord(g, hi.y), c1[2] = grid_coord(g, hi.z);
}

// Cell (x, y, z) of the k-th cell of an obstacle's cell box [c0, c1].
__device__ __forceinline__ int box_cell(const Grid& g, const int c0[3], const int c1[3], int k)
{
    const int nx = c1[0] - c0[0] + 1, ny = c1[1] - c0[1] + 1;
    const int x = c0[0] + k % nx, y = c0[1] + (k / nx) % ny, z = c0[2] + k / (nx * ny);
    return x + g.dim * (y + g.dim * z);
}

__device__ __forceinline__ int box_cells(const int c0[3], const int c1[3])
{
    return (c1[0] - c0[0] + 1) * (c1[1] - c0[1] + 1) * (c1[2] - c0[2] + 1);
}

// One warp per obstacle: pack n x 6 floats into float4 pairs and count (cell, obstacle) pairs.
__global__ void k_env_count(Grid g, const float* __restrict__ obs, uint32_t n, float4* __restrict__ packed,
                            uint32_t* __restrict__ counts)
{
    const uint32_t o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if(o >= n) return;
    const float* b = obs + (size_t)6 * o;
    const float4 lo = make_float4(b[0], b[1], b[2], 0.0f), hi = make_float4(b[3], b[4], b[5], 0.0f);
    if(lane == 0) packed[2 * o] = lo, packed[2 * o + 1] = hi;
    int c0[3], c1[3];
    obstacle_cells(g, lo, hi, c0, c1);
    const int total = box_cells(c0, c1);
    for(int k = lane; k < total; k += 32) atomicAdd(counts + box_cell(g, c0, c1, k), 1u);
}

// Exclusive scan of counts[0, n) in place (single CTA of 1024 threads; each thread scans 8
// consecutive counts per pass, read and written as two 16-byte vectors where the pass is full and
// both arrays start 16-byte aligned, one count at a time otherwise); counts[n] = total; cursor
// gets a copy of the offsets.
constexpr int kEnvScanItems = 8;
__global__ void __launch_bounds__(1024) k_env_scan(uint32_t* __restrict__ counts, uint32_t n, uint32_t* __restrict__ cursor)
{
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool vec = ((reinterpret_cast<uintptr_t>(counts) | reinterpret_cast<uintptr_t>(cursor)) & 15u) == 0;
    if(threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for(uint32_t base = 0; base < n; base += 1024 * kEnvScanItems) {
        const uint32_t i0 = base + threadIdx.x * kEnvScanItems;
        const bool full = vec && i0 + kEnvScanItems <= n;
        uint32_t v[kEnvScanItems], sum = 0;
        if(full) {
            const uint4 a = *reinterpret_cast<const uint4*>(counts + i0), b = *reinterpret_cast<const uint4*>(counts + i0 + 4);
            v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
        } else {
#pragma unroll
            for(int j = 0; j < kEnvScanItems; ++j) v[j] = i0 + j < n ? counts[i0 + j] : 0u;
        }
#pragma unroll
        for(int j = 0; j < kEnvScanItems; ++j) sum += v[j];
        uint32_t x = sum;
#pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += y;
        }
        if(lane == 31) s_warp[warp] = x;
        __syncthreads();
        if(warp == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for(int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
                if(lane >= d) w += y;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        uint32_t e[kEnvScanItems], acc = s_carry + (warp ? s_warp[warp - 1] : 0u) + x - sum;
#pragma unroll
        for(int j = 0; j < kEnvScanItems; ++j) e[j] = acc, acc += v[j];
        if(full) {
            const uint4 a = make_uint4(e[0], e[1], e[2], e[3]), b = make_uint4(e[4], e[5], e[6], e[7]);
            *reinterpret_cast<uint4*>(counts + i0) = a, *reinterpret_cast<uint4*>(counts + i0 + 4) = b;
            *reinterpret_cast<uint4*>(cursor + i0) = a, *reinterpret_cast<uint4*>(cursor + i0 + 4) = b;
        } else {
#pragma unroll
            for(int j = 0; j < kEnvScanItems; ++j)
                if(i0 + j < n) counts[i0 + j] = e[j], cursor[i0 + j] = e[j];
        }
        __syncthreads();
        if(threadIdx.x == 0) s_carry += s_warp[31];
        __syncthreads();
    }
    if(threadIdx.x == 0) counts[n] = s_carry;
}

__global__ void k_env_fill(Grid g, const float4* __restrict__ packed, uint32_t n, uint32_t* __restrict__ cursor,
                           uint32_t* __restrict__ ent)
{
    const uint32_t o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if(o >= n) return;
    int c0[3], c1[3];
    obstacle_cells(g, packed[2 * o], packed[2 * o + 1], c0, c1);
    const int total = box_cells(c0, c1);
    for(int k = lane; k < total; k += 32) ent[atomicAdd(cursor + box_cell(g, c0, c1, k), 1u)] = o;
}

inline uint32_t warp_blocks(uint32_t n) { return (uint32_t)(((uint64_t)n * 32 + 255) / 256); }

// ---------------------------------------------------------------- batch kernels

template <int M>
__global__ void __launch_bounds__(256, 4) k_propagate_batch(KParams p, Grid g, const float* __restrict__ parents,
                                                         const float* __restrict__ draws, uint32_t stream_id, uint32_t n,
                                                         float* __restrict__ rows, uint8_t* __restrict__ valid,
                                                         int32_t* __restrict__ steps_out)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD, S = SD + CD + 1;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    float s[SD], u[6], c[4], rc[4];
#pragma unroll
    for(int k = 0; k < SD; ++k) s[k] = __ldg(parents + (size_t)i * SD + k);
    if(draws) {
#pragma unroll
        for(int k = 0; k < 5; ++k) u[k] = __ldg(draws + (size_t)i * 5 + k);
        u[5] = 0.0f;
    } else {
        child_draws(p, stream_id, 0u, i, u);
    }
    const int steps = draw_controls(p, u, c);
    int done = 0;
    const bool ok = propagate<M>(p, g, s, c, steps, done);
    row_controls<M>(c, rc);
    float* dst = rows + (size_t)i * S;
#pragma unroll
    for(int k = 0; k < SD; ++k) dst[k] = s[k];
#pragma unroll
    for(int k = 0; k < CD; ++k) dst[SD + k] = rc[k];
    dst[SD + CD] = __fmul_rn(p.h, (float)steps);  // STEP_SIZE * propagationDuration
    valid[i] = ok ? 1 : 0;
    if(steps_out) steps_out[i] = done;
}

// Large batches run in phases so that lanes do not idle behind their warp's longest segment: the
// head runs every segment for its first kHeadSteps steps and finishes the segments that end there
// (a fifth of them fail in their first steps); the others are appended, state and controls, to a
// compact list.  A middle phase carries that list to 3/5 of the longest segment (mid_steps),
// finishes the segments that end by then and appends the rest to a second list, which the tail
// carries to the end, each with full warps.  Every phase runs the same per-step code in the same
// order, so rows, verdicts and step counts equal the one-pass kernel's.  Dubins microbench, 2^22
// segments of 20 steps: 2.15 G valid segments/s in two phases; 2.15 / 2.18 / 2.19 G/s with the
// middle phase ending after step 6 / 8 / 12.
constexpr int kHeadSteps = 2;
inline int mid_steps(const KParams& p) { return std::max(kHeadSteps + 1, (p.nsteps + 1) * 3 / 5); }
constexpr uint32_t kPhasedMin = 1u << 18;   // segments; below this the one-pass kernel is used
// Segments per round of the three phases (bounds the survivor lists' scratch).  Each round pays the
// latency of its longest segment in every phase, so rounds are as large as the scratch allows:
// rounds of 2^19 segments (lists resident in L2 between the phases) measured 1.73 G segments/s
// on the Dubins microbench against 2.18 G/s in one round of 2^22.
constexpr uint32_t kPhaseChunk = 1u << 24;

struct LiveList {
    uint32_t* count;
    uint32_t* idx;
    int32_t* steps;  // unused (null) for fixed-step models
    float* ctl;      // CD per entry
    float* state;    // SD per entry
};

template <int M>
__device__ __forceinline__ void write_segment(const KParams& p, uint32_t i, const float* s, const float* c, int steps, bool ok,
                                              int done, float* __restrict__ rows, uint8_t* __restrict__ valid,
                                              int32_t* __restrict__ steps_out)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD, S = SD + CD + 1;
    float rc[4];
    row_controls<M>(c, rc);
    float* dst = rows + (size_t)i * S;
#pragma unroll
    for(int k = 0; k < SD; ++k) dst[k] = s[k];
#pragma unroll
    for(int k = 0; k < CD; ++k) dst[SD + k] = rc[k];
    dst[SD + CD] = __fmul_rn(p.h, (float)steps);
    valid[i] = ok ? 1 : 0;
    if(steps_out) steps_out[i] = done;
}

// Appends the warp's live segments to `live` (one atomic per warp); called by all 32 lanes.
template <int SD, int CD>
__device__ __forceinline__ void append_live(const LiveList& live, bool alive, int lane, uint32_t i, int steps, const float* c,
                                            const float* s)
{
    const uint32_t m = __ballot_sync(0xffffffffu, alive);
    if(!m) return;
    const int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if(lane == leader) base = atomicAdd(live.count, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    if(alive) {
        const uint32_t j = base + __popc(m & ((1u << lane) - 1u));
        live.idx[j] = i;
        if(live.steps) live.steps[j] = steps;
#pragma unroll
        for(int k = 0; k < CD; ++k) live.ctl[(size_t)j * CD + k] = c[k];
#pragma unroll
        for(int k = 0; k < SD; ++k) live.state[(size_t)j * SD + k] = s[k];
    }
}

// Segments i of one round (pointers offset to the round's first segment; i0 = that segment's index
// in the batch, which keys its draws).
template <int M>
__global__ void __launch_bounds__(256, 4) k_propagate_head(KParams p, Grid g, const float* __restrict__ parents,
                                                        const float* __restrict__ draws, uint32_t stream_id, uint32_t n,
                                                        uint32_t i0, float* __restrict__ rows, uint8_t* __restrict__ valid,
                                                        int32_t* __restrict__ steps_out, LiveList live)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool alive = false;
    float s[SD], c[4];
    int steps = 0;
    if(i < n) {
        float u[6];
#pragma unroll
        for(int k = 0; k < SD; ++k) s[k] = __ldg(parents + (size_t)i * SD + k);
        if(draws) {
#pragma unroll
            for(int k = 0; k < 5; ++k) u[k] = __ldg(draws + (size_t)i * 5 + k);
            u[5] = 0.0f;
        } else {
            child_draws(p, stream_id, 0u, i0 + i, u);
        }
        steps = draw_controls(p, u, c);
        const auto k = segment_consts<M>(p, c);
        const StepParams sp = step_params(p);
        bool ok = true;
        int done = 0;
        while(done < steps && done < kHeadSteps) {
            ok = model_step<M>(sp, g, s, c, k);
            ++done;
            if(!ok) break;
        }
        alive = ok && done < steps;
        if(!alive) write_segment<M>(p, i, s, c, steps, ok, done, rows, valid, steps_out);
    }
    append_live<SD, CD>(live, alive, lane, i, steps, c, s);
}

template <int M>
__global__ void __launch_bounds__(256, 4) k_propagate_tail(KParams p, Grid g, float* __restrict__ rows,
                                                        uint8_t* __restrict__ valid, int32_t* __restrict__ steps_out,
                                                        LiveList live, int from, int until, LiveList next)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD;
    const uint32_t count = *live.count;
    if(blockIdx.x * blockDim.x >= count) return;  // whole block past the list: the ballot below needs full warps
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool alive = false;
    uint32_t i = 0;
    int steps = 0;
    float s[SD], c[4];
    if(j < count) {
        i = live.idx[j];
        steps = live.steps ? live.steps[j] : p.nsteps;
#pragma unroll
        for(int k = 0; k < 4; ++k) c[k] = k < CD ? live.ctl[(size_t)j * CD + k] : 0.0f;
#pragma unroll
        for(int k = 0; k < SD; ++k) s[k] = live.state[(size_t)j * SD + k];
        const auto kc = segment_consts<M>(p, c);
        const StepParams sp = step_params(p);
        bool ok = true;
        int done = from;
        while(done < steps && done < until) {
            ok = model_step<M>(sp, g, s, c, kc);
            ++done;
            if(!ok) break;
        }
        alive = next.count && ok && done < steps;
        if(!alive) write_segment<M>(p, i, s, c, steps, ok, done, rows, valid, steps_out);
    }
    if(next.count) append_live<SD, CD>(next, alive, lane, i, steps, c, s);
}

// The three phases over rounds of kPhaseChunk segments; `counts` (two words, 128 bytes apart) are
// cleared before every round.
template <int M>
void launch_phases(const KParams& p, const Grid& g, const float* parents, const float* draws, uint32_t stream_id, uint32_t n,
                   float* rows, uint8_t* valid, int32_t* steps_out, const LiveList& first, const LiveList& second,
                   const LiveList& none, void* counts, cudaStream_t s)
{
    const int SD = p.sd, S = p.S, mid = mid_steps(p);
    for(uint32_t o = 0; o < n; o += kPhaseChunk) {
        const uint32_t m = std::min(kPhaseChunk, n - o), blocks = (m + 255) / 256;
        float* r = rows + (size_t)o * S;
        uint8_t* v = valid + o;
        int32_t* st = steps_out ? steps_out + o : nullptr;
        cudaMemsetAsync(counts, 0, 256, s);
        k_propagate_head<M><<<blocks, 256, 0, s>>>(p, g, parents + (size_t)o * SD, draws ? draws + (size_t)o * 5 : nullptr,
                                                   stream_id, m, o, r, v, st, first);
        k_propagate_tail<M><<<blocks, 256, 0, s>>>(p, g, r, v, st, first, kHeadSteps, mid, second);
        k_propagate_tail<M><<<blocks, 256, 0, s>>>(p, g, r, v, st, second, mid, INT_MAX, none);
        count_launch(3);
    }
}

__global__ void k_collide_batch(Grid g, const float* __restrict__ bbmin, const float* __restrict__ bbmax, uint32_t n,
                                uint8_t* __restrict__ free_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float lo[3] = {bbmin[3 * i], bbmin[3 * i + 1], bbmin[3 * i + 2]};
    const float hi[3] = {bbmax[3 * i], bbmax[3 * i + 1], bbmax[3 * i + 2]};
    free_out[i] = box_free(g, lo, hi) ? 1 : 0;
}

__global__ void k_region_batch(KParams p, const float* __restrict__ states, uint32_t n, int32_t* __restrict__ r1,
                               int32_t* __restrict__ r2)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    float s[12];
    for(int k = 0; k < p.sd; ++k) s[k] = states[(size_t)i * p.sd + k];
    const int a = region_r1<12>(p, s);
    r1[i] = a;
    if(r2) r2[i] = region_r2<12>(p, s, a);
}

__global__ void k_sincos_pair(const float* __restrict__ x, uint32_t n, float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    float s, c, s2, c2;
    sincos_checked(x[i], &s, &c);
    sincosf(x[i], &s2, &c2);
    out[4 * i] = s, out[4 * i + 1] = c, out[4 * i + 2] = s2, out[4 * i + 3] = c2;
}

}  // namespace

kpax_status Env::build(const KParams& p, const float* d_obstacles, uint32_t n, cudaStream_t stream)
{
    cell = p.cell;
    wmin = p.wmin;
    dim = p.gdim;
    const uint32_t cells = (uint32_t)dim * dim * dim;
    if(cells != n_cells) {
        if(d_off) cudaFree(d_off), d_off = nullptr;
        if(d_cursor) cudaFree(d_cursor), d_cursor = nullptr;
        KPAX_CUDA(cudaMalloc(&d_off, sizeof(uint32_t) * (cells + 1)));
        KPAX_CUDA(cudaMalloc(&d_cursor, sizeof(uint32_t) * cells));
        n_cells = cells;
    }
    if(!h_total) KPAX_CUDA(cudaMallocHost(&h_total, sizeof(uint32_t)));
    if(n > obs_cap) {
        if(d_obs) cudaFree(d_obs), d_obs = nullptr;
        KPAX_CUDA(cudaMalloc(&d_obs, sizeof(float4) * 2 * n));
        obs_cap = n;
    }
    n_obs = n;
    KPAX_CUDA(cudaMemsetAsync(d_off, 0, sizeof(uint32_t) * (cells + 1), stream));
    const Grid g0 = view();
    if(n) {
        k_env_count<<<warp_blocks(n), 256, 0, stream>>>(g0, d_obstacles, n, d_obs, d_off);
        KPAX_CHECK_LAUNCH();
        k_env_scan<<<1, 1024, 0, stream>>>(d_off, cells, d_cursor);
        KPAX_CHECK_LAUNCH();
        count_launch(2);
        KPAX_CUDA(cudaMemcpyAsync(h_total, d_off + cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        n_ent = *h_total;
        if(n_ent > ent_cap) {
            if(d_ent) cudaFree(d_ent), d_ent = nullptr;
            const uint32_t want = n_ent + n_ent / 4 + 1024;
            KPAX_CUDA(cudaMalloc(&d_ent, sizeof(uint32_t) * want));
            ent_cap = want;
        }
        k_env_fill<<<warp_blocks(n), 256, 0, stream>>>(view(), d_obs, n, d_cursor, d_ent);
        KPAX_CHECK_LAUNCH();
        count_launch(1);
    } else {
        n_ent = 0;
        if(!d_ent) {
            KPAX_CUDA(cudaMalloc(&d_ent, sizeof(uint32_t) * 1024));
            ent_cap = 1024;
        }
        if(!d_obs) {
            KPAX_CUDA(cudaMalloc(&d_obs, sizeof(float4) * 2));
            obs_cap = 1;
        }
    }
    return KPAX_OK;
}

void Env::release()
{
    if(d_obs) cudaFree(d_obs);
    if(d_off) cudaFree(d_off);
    if(d_cursor) cudaFree(d_cursor);
    if(d_ent) cudaFree(d_ent);
    if(d_live) cudaFree(d_live), d_live = nullptr, live_cap = 0;
    if(h_total) cudaFreeHost(h_total);
    d_obs = nullptr, d_off = d_cursor = d_ent = h_total = nullptr;
    obs_cap = ent_cap = n_cells = n_ent = n_obs = 0;
}

kpax_status launch_propagate(const KParams& p, const Grid& g, const float* parents, const float* draws, uint32_t stream_id,
                             uint32_t n, float* rows, uint8_t* valid, int32_t* steps, cudaStream_t stream)
{
    if(!n) return KPAX_OK;
    const uint32_t blocks = (n + 255) / 256;
    switch(p.model) {
        case KPAX_MODEL_DOUBLE_INTEGRATOR:
            k_propagate_batch<KPAX_MODEL_DOUBLE_INTEGRATOR><<<blocks, 256, 0, stream>>>(p, g, parents, draws, stream_id, n, rows, valid, steps);
            break;
        case KPAX_MODEL_DUBINS_AIRPLANE:
            k_propagate_batch<KPAX_MODEL_DUBINS_AIRPLANE><<<blocks, 256, 0, stream>>>(p, g, parents, draws, stream_id, n, rows, valid, steps);
            break;
        default:
            k_propagate_batch<KPAX_MODEL_QUADROTOR><<<blocks, 256, 0, stream>>>(p, g, parents, draws, stream_id, n, rows, valid, steps);
            break;
    }
    KPAX_CHECK_LAUNCH();
    count_launch();
    return KPAX_OK;
}

}  // namespace kpax

using namespace kpax;

extern "C" {

uint64_t kpax_kernel_launches(void) { return g_launches.load(); }

kpax_status kpax_test_sincos(const float* d_x, uint32_t n, float* d_out, void* stream)
{
    if(n && (!d_x || !d_out)) return set_error("kpax_test_sincos: null argument"), KPAX_EINVAL;
    if(!n) return KPAX_OK;
    k_sincos_pair<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_x, n, d_out);
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

// FP32 issue-rate microkernel: every thread advances kChains independent FMA chains `iters` times
// (2 FLOP per FMA); the values stay bounded (|a| < 1) and are folded into one store the compiler
// cannot drop.  The measured rate is the denominator of the propagation kernels' roofline.
constexpr int kFmaChains = 8;
__global__ void __launch_bounds__(512) k_fma_peak(float* __restrict__ out, uint32_t iters, float a, float b)
{
    float x[kFmaChains];
#pragma unroll
    for(int j = 0; j < kFmaChains; ++j) x[j] = (float)(threadIdx.x + j) * 1e-3f;
    for(uint32_t i = 0; i < iters; i += 16) {
#pragma unroll
        for(int u = 0; u < 16; ++u)
#pragma unroll
            for(int j = 0; j < kFmaChains; ++j) x[j] = fmaf(x[j], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for(int j = 0; j < kFmaChains; ++j) s += x[j];
    if(s == -1.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true; keeps the chains live
}

kpax_status kpax_fp32_peak(uint32_t iters, double* h_tflops, double* h_ms, void* stream)
{
    if(!h_tflops || iters < 16) return set_error("kpax_fp32_peak: need h_tflops and iters >= 16"), KPAX_EINVAL;
    iters = iters / 16 * 16;
    int dev = 0, sms = 0;
    KPAX_CUDA(cudaGetDevice(&dev));
    KPAX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t blocks = (uint32_t)sms * 4u, threads = 512;  // 2048 threads per SM
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    KPAX_CUDA(cudaEventCreate(&e0));
    KPAX_CUDA(cudaEventCreate(&e1));
    float ms = 0.0f;
    for(int rep = 0; rep < 2; ++rep) {  // the first launch warms up
        cudaEventRecord(e0, s);
        k_fma_peak<<<blocks, threads, 0, s>>>(nullptr, iters, 0.99999f, 1e-6f);
        cudaEventRecord(e1, s);
        count_launch();
    }
    cudaError_t err = cudaEventSynchronize(e1);
    if(err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if(err != cudaSuccess) return set_error("kpax_fp32_peak: %s", cudaGetErrorString(err)), KPAX_ECUDA;
    const double flop = 2.0 * kFmaChains * (double)iters * blocks * threads;
    *h_tflops = ms > 0.0f ? flop / (ms * 1e-3) / 1e12 : 0.0;
    if(h_ms) *h_ms = ms;
    return KPAX_OK;
}

kpax_status kpax_env_create(const kpax_config* cfg, const float* d_obstacles, uint32_t n_obs, void* stream, kpax_env** out)
{
    NvtxRange range("kpax_env_create");
    if(!cfg || !out || (n_obs && !d_obstacles)) return set_error("kpax_env_create: null argument"), KPAX_EINVAL;
    *out = nullptr;
    kpax_env* e = new(std::nothrow) kpax_env();
    if(!e) return set_error("kpax_env_create: host allocation failed"), KPAX_ENOMEM;
    kpax_status st = derive_params(*cfg, &e->params);
    if(st == KPAX_OK) st = e->env.build(e->params, d_obstacles, n_obs, (cudaStream_t)stream);
    if(st == KPAX_OK) {
        cudaError_t err = cudaStreamSynchronize((cudaStream_t)stream);
        if(err != cudaSuccess) set_error("kpax_env_create: %s", cudaGetErrorString(err)), st = KPAX_ECUDA;
    }
    if(st != KPAX_OK) {
        e->env.release();
        delete e;
        return st;
    }
    *out = e;
    return KPAX_OK;
}

kpax_status kpax_env_destroy(kpax_env* e)
{
    if(!e) return KPAX_OK;
    e->env.release();
    if(e->d_occ) cudaFree(e->d_occ);
    delete e;
    return KPAX_OK;
}

kpax_status kpax_env_stats(kpax_env* e, uint32_t* n_cells, uint32_t* n_entries)
{
    if(!e) return set_error("kpax_env_stats: null env"), KPAX_EINVAL;
    if(n_cells) *n_cells = e->env.n_cells;
    if(n_entries) *n_entries = e->env.n_ent;
    return KPAX_OK;
}

kpax_status kpax_propagate_batch(const kpax_config* cfg, kpax_env* env, const float* d_parents, const float* d_draws,
                                 uint32_t draw_stream, uint32_t n, float* d_rows, uint8_t* d_valid, int32_t* d_steps,
                                 void* stream)
{
    NvtxRange range("kpax_propagate_batch");
    if(!cfg || !env || (n && (!d_parents || !d_rows || !d_valid)))
        return set_error("kpax_propagate_batch: null argument"), KPAX_EINVAL;
    KParams p;
    kpax_status st = derive_params(*cfg, &p);
    if(st != KPAX_OK) return st;
    if(p.gdim != env->env.dim || p.cell != env->env.cell || p.wmin != env->env.wmin)
        return set_error("kpax_propagate_batch: env was built for another workspace grid"), KPAX_EINVAL;
    if(n < kPhasedMin)
        return launch_propagate(p, env->env.view(), d_parents, d_draws, draw_stream, n, d_rows, d_valid, d_steps,
                                (cudaStream_t)stream);
    // phases: the two live lists of a round live in the env's scratch, grown on demand (counts at
    // bytes 0 and 128, then each list's index, step-count (drawn durations only), control and state
    // arrays)
    Env& e = env->env;
    auto align = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t m = std::min(n, kPhaseChunk);
    const size_t l_idx = 0, l_steps = align(4ull * m), l_ctl = l_steps + (p.fixed_steps ? 0 : align(4ull * m)),
                 l_state = l_ctl + align(4ull * p.cd * m), l_bytes = l_state + align(4ull * p.sd * m), bytes = 256 + 2 * l_bytes;
    if(bytes > e.live_cap) {
        if(e.d_live) cudaFree(e.d_live), e.d_live = nullptr, e.live_cap = 0;
        KPAX_CUDA(cudaMalloc(&e.d_live, bytes));
        e.live_cap = bytes;
    }
    char* base = static_cast<char*>(e.d_live);
    auto list = [&](int k) {
        char* l = base + 256 + (size_t)k * l_bytes;
        return LiveList{reinterpret_cast<uint32_t*>(base + 128 * k), reinterpret_cast<uint32_t*>(l + l_idx),
                        p.fixed_steps ? nullptr : reinterpret_cast<int32_t*>(l + l_steps), reinterpret_cast<float*>(l + l_ctl),
                        reinterpret_cast<float*>(l + l_state)};
    };
    const LiveList first = list(0), second = list(1), none{};
    cudaStream_t s = (cudaStream_t)stream;
    const Grid g = e.view();
    switch(p.model) {
        case KPAX_MODEL_DOUBLE_INTEGRATOR:
            launch_phases<KPAX_MODEL_DOUBLE_INTEGRATOR>(p, g, d_parents, d_draws, draw_stream, n, d_rows, d_valid, d_steps, first,
                                                       second, none, base, s);
            break;
        case KPAX_MODEL_DUBINS_AIRPLANE:
            launch_phases<KPAX_MODEL_DUBINS_AIRPLANE>(p, g, d_parents, d_draws, draw_stream, n, d_rows, d_valid, d_steps, first,
                                                     second, none, base, s);
            break;
        default:
            launch_phases<KPAX_MODEL_QUADROTOR>(p, g, d_parents, d_draws, draw_stream, n, d_rows, d_valid, d_steps, first, second,
                                               none, base, s);
            break;
    }
    KPAX_CHECK_LAUNCH();
    return KPAX_OK;
}

kpax_status kpax_collide_batch(kpax_env* env, const float* d_bbmin, const float* d_bbmax, uint32_t n, uint8_t* d_free,
                               void* stream)
{
    if(!env || (n && (!d_bbmin || !d_bbmax || !d_free))) return set_error("kpax_collide_batch: null argument"), KPAX_EINVAL;
    if(!n) return KPAX_OK;
    k_collide_batch<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(env->env.view(), d_bbmin, d_bbmax, n, d_free);
    KPAX_CHECK_LAUNCH();
    count_launch();
    return KPAX_OK;
}

kpax_status kpax_region_batch(const kpax_config* cfg, const float* d_states, uint32_t n, int32_t* d_r1, int32_t* d_r2,
                              void* stream)
{
    if(!cfg || (n && (!d_states || !d_r1))) return set_error("kpax_region_batch: null argument"), KPAX_EINVAL;
    KParams p;
    kpax_status st = derive_params(*cfg, &p);
    if(st != KPAX_OK) return st;
    if(!n) return KPAX_OK;
    k_region_batch<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p, d_states, n, d_r1, d_r2);
    KPAX_CHECK_LAUNCH();
    count_launch();
    return KPAX_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free propagation
// kpax_propagate_batch_noalloc builds the obstacle grid in a fixed device array instead of
// memory from cudaMalloc, for callers that must not allocate device memory while they run: a
// planner called from a robot's real-time control cycle (cudaMalloc can synchronise the device
// and take unbounded time) or a host application that reserves all device memory up front for
// its own pool.  The array below lives in every GPU that loads this library, until exit.
namespace {

constexpr uint32_t kNoAllocMaxObstacles = 4096;
constexpr uint32_t kNoAllocMaxCells = 1u << 17;    // e.g. a 50^3 grid
constexpr uint32_t kNoAllocMaxEntries = 1u << 18;  // (cell, obstacle) pairs

struct NoAllocScratch {
    float4 obs[2 * kNoAllocMaxObstacles];
    uint32_t off[kNoAllocMaxCells + 4];  // cells + 1, padded so that cursor starts 16-byte aligned
    uint32_t cursor[kNoAllocMaxCells];
    uint32_t ent[kNoAllocMaxEntries];
};

// In host code this name is only a stand-in for the device array; kernels get the address
// from cudaGetSymbolAddress below.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per device.
kpax_status noalloc_scratch(NoAllocScratch** out)
{
    int dev = 0;
    KPAX_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= kNoAllocMaxDevices) return set_error("device ordinal %d not supported", dev), KPAX_EINVAL;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if(!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess || !p)
            return set_error("cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e)), KPAX_ECUDA;
        g_noalloc_addr[dev] = (NoAllocScratch*)p;
    }
    *out = g_noalloc_addr[dev];
    return KPAX_OK;
}

}  // namespace

extern "C" kpax_status kpax_propagate_batch_noalloc(const kpax_config* cfg, const float* d_obstacles, uint32_t n_obs,
                                                    const float* d_parents, const float* d_draws, uint32_t draw_stream,
                                                    uint32_t n, float* d_rows, uint8_t* d_valid, int32_t* d_steps,
                                                    void* stream)
{
    if(!cfg || (n_obs && !d_obstacles) || (n && (!d_parents || !d_rows || !d_valid)))
        return set_error("kpax_propagate_batch_noalloc: null argument"), KPAX_EINVAL;
    KParams p;
    kpax_status st = derive_params(*cfg, &p);
    if(st != KPAX_OK) return st;
    const uint32_t cells = (uint32_t)p.gdim * p.gdim * p.gdim;
    if(n_obs > kNoAllocMaxObstacles)
        return set_error("kpax_propagate_batch_noalloc: %u obstacles exceed the limit of %u", n_obs, kNoAllocMaxObstacles),
               KPAX_ECAPACITY;
    if(cells > kNoAllocMaxCells)
        return set_error("kpax_propagate_batch_noalloc: %u grid cells exceed the limit of %u", cells, kNoAllocMaxCells),
               KPAX_ECAPACITY;
    NoAllocScratch* s = nullptr;
    if((st = noalloc_scratch(&s)) != KPAX_OK) return st;
    cudaStream_t cs = (cudaStream_t)stream;
    const Grid g{s->obs, s->off, s->ent, p.wmin, 1.0f / p.cell, p.gdim};
    // the array keeps the previous call's grid: the counts must start from zero
    KPAX_CUDA(cudaMemsetAsync(s->off, 0, sizeof(uint32_t) * (cells + 1), cs));
    if(n_obs) {
        k_env_count<<<warp_blocks(n_obs), 256, 0, cs>>>(g, d_obstacles, n_obs, s->obs, s->off);
        KPAX_CHECK_LAUNCH();
        k_env_scan<<<1, 1024, 0, cs>>>(s->off, cells, s->cursor);
        KPAX_CHECK_LAUNCH();
        count_launch(2);
        uint32_t total = 0;
        KPAX_CUDA(cudaMemcpyAsync(&total, s->off + cells, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
        KPAX_CUDA(cudaStreamSynchronize(cs));
        if(total > kNoAllocMaxEntries)
            return set_error("kpax_propagate_batch_noalloc: %u (cell, obstacle) pairs exceed the limit of %u", total,
                             kNoAllocMaxEntries),
                   KPAX_ECAPACITY;
        k_env_fill<<<warp_blocks(n_obs), 256, 0, cs>>>(g, s->obs, n_obs, s->cursor, s->ent);
        KPAX_CHECK_LAUNCH();
        count_launch(1);
    }
    return launch_propagate(p, g, d_parents, d_draws, draw_stream, n, d_rows, d_valid, d_steps, cs);
}

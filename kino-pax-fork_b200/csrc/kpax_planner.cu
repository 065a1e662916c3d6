// kpax_planner.cu — the plan loop: per-iteration kernels, CUDA-graph capture and the C ABI.
//
// One iteration of the reference (KPAX.cu:94-105) is propagateFrontier (303-351),
// Graph::updateVertices (Graph.cu:207-227) and updateFrontier (520-543), with thrust scans over
// the full tree capacity and ~6 host synchronisations.  Here it is three kernels with all sizes
// kept on the device, captured `unroll` iterations at a time in a CUDA graph:
//   k_frontier  re-activation of the previous iteration (KPAX.cu:505-517), repeat counts of new
//               nodes (476-479) and an order-preserving scan of the frontier into the entry
//               list (Planner.cu:52-80) — one pass over the live tree, decoupled look-back;
//   k_expand    per child: draw, RK4 + per-step collision, R1/R2 ids, counters, frontier mark
//               (KPAX.cu:381-396) and the stable append of accepted children to the tree with
//               cost and goal test (458-502) — one kernel, decoupled look-back for the slots;
//   k_scores    R2 snapshot update, region scores and their normalisation (Graph.cu:233-358)
//               in one CTA, then the iteration bookkeeping (tree size, fAccept, stop flags).
// Deterministic replacements for the reference's races are listed in oracle/kpax_oracle.h.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "kpax_internal.h"

namespace kpax {
namespace {

constexpr uint8_t kPending = 255;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kFrontierBS = 256, kItems = 4, kTile = kFrontierBS * kItems;
constexpr int kExpandBS = 448;  // 2^16 children over 148 SMs: one 14-warp block per SM
constexpr int kFrontierCTAs = 2 * 148;
constexpr int kScoreBS = 256, kScoreCTAs = 128, kPartials = 1024;
constexpr uint32_t kSpinLimit = 1u << 22;  // ~4 s of polling before a wait gives up
constexpr uint32_t kErrTimeout = 1u, kErrCapacity = 2u;

struct TreeDev {
    float4* s[3];  // state planes: floats 4k..4k+3 of every node
    float4* ctl;   // controls as stored in the row
    float* dur;
    int32_t* parent;
    float* cost;
    int32_t* r1;
    uint8_t* rep;  // frontier repeat count; 0 = not in frontier; kPending = added last iteration
};

struct RegDev {
    int32_t* counter;
    int32_t* valid;
    float* score;
    uint32_t* cur;  // R2 activation bits as of the start of the iteration
    uint32_t* nxt;  // R2 activation bits including this iteration
};

struct CaptureDev {
    float* rows;
    uint8_t* valid;
    int32_t* r1;
    int32_t* r2;
    uint8_t* next;
    int32_t* parent;
};

struct alignas(16) Ctl {
    uint32_t tree, tree_old, iter, R, k, E, n, appended;
    uint32_t goal_idx, done, full, error;
    uint32_t plan_idx, max_iters, stop_at_goal, epoch;
    uint32_t ticket1, ticket2, iters_done, path_len;
    float faccept, goal[3];
    float score_total;      // sum of raw region scores of the last score pass
    uint32_t scores_ready;  // 0 until the first score pass of a plan (scores read as 0, KPAX.cu:69)
    unsigned long long n_exp, n_valid, n_steps;
    double path_cost;
};

// ---------------------------------------------------------------- look-back helpers
// Status word: [epoch:30 | flag:2 | value:32]; flag 1 = block aggregate, 2 = inclusive prefix.
__device__ __forceinline__ void lb_publish(unsigned long long* slot, uint32_t epoch, uint32_t flag, uint32_t value)
{
    const unsigned long long w = ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | ((unsigned long long)flag << 32) | value;
    __threadfence();
    atomicExch(slot, w);
}

// Exclusive prefix of tile b, computed by the 32 lanes of one warp: each probe reads the status
// of 32 predecessors at once and stops at the nearest inclusive prefix.  Returns false when a
// predecessor never published (bounded wait, ~4 s).
__device__ __forceinline__ bool lb_exclusive(unsigned long long* lb, uint32_t b, uint32_t epoch, uint32_t& excl)
{
    const uint32_t tag = epoch & 0x3FFFFFFFu;
    const int lane = threadIdx.x & 31;
    uint32_t acc = 0, spins = 0;
    int top = (int)b - 1;
    while(top >= 0) {
        const int j = top - lane;  // lane 0 probes the nearest predecessor
        uint32_t flag = 2u, val = 0u;  // past tile 0: an inclusive prefix of zero
        if(j >= 0) {
            const unsigned long long w = atomicAdd(lb + j, 0ull);
            flag = (uint32_t)(w >> 34) == tag ? (uint32_t)(w >> 32) & 3u : 0u;
            val = (uint32_t)w;
        }
        const uint32_t ready = __ballot_sync(0xffffffffu, flag != 0u), incl = __ballot_sync(0xffffffffu, flag == 2u);
        const int first = incl ? __ffs(incl) - 1 : 31;
        const uint32_t need = first == 31 ? 0xffffffffu : ((2u << first) - 1u);
        if((ready & need) != need) {
            if(++spins > kSpinLimit) {
                excl = acc;
                return false;
            }
            if(spins > 32) __nanosleep(100);
            continue;
        }
        uint32_t v = lane <= first ? val : 0u;
#pragma unroll
        for(int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        acc += v;
        if(incl) break;
        top -= 32;
    }
    excl = acc;
    return true;
}

__device__ __forceinline__ uint32_t popcount_range(const uint32_t* __restrict__ bits, uint64_t lo, uint64_t hi)
{
    uint32_t n = 0;
    const uint64_t w0 = lo >> 5, w1 = (hi - 1) >> 5;
    for(uint64_t w = w0; w <= w1; ++w) {
        uint32_t m = bits[w];
        if(w == w0) m &= ~0u << (lo & 31);
        if(w == w1) {
            const uint32_t top = (uint32_t)((hi - 1) & 31);
            m &= top == 31 ? ~0u : ((1u << (top + 1)) - 1u);
        }
        n += __popc(m);
    }
    return n;
}

// Normalised score of a region (Graph.cu:297-304, 349-357) from its stored raw score.
__device__ __forceinline__ float region_score(float raw, float total, uint32_t ready, float eps)
{
    if(!ready) return 0.0f;
    return raw < 0.0f ? 1.0f : __fadd_rn(eps, __fdiv_rn(raw, total));
}

template <int SD>
__device__ __forceinline__ void load_state(const TreeDev& t, uint32_t i, float* s)
{
    const float4 a = t.s[0][i], b = t.s[1][i];
    s[0] = a.x, s[1] = a.y, s[2] = a.z, s[3] = a.w, s[4] = b.x, s[5] = b.y;
    if constexpr(SD == 12) {
        const float4 c = t.s[2][i];
        s[6] = b.z, s[7] = b.w, s[8] = c.x, s[9] = c.y, s[10] = c.z, s[11] = c.w;
    }
}

template <int SD>
__device__ __forceinline__ void store_state(const TreeDev& t, uint32_t i, const float* s)
{
    if constexpr(SD == 12) {
        t.s[0][i] = make_float4(s[0], s[1], s[2], s[3]);
        t.s[1][i] = make_float4(s[4], s[5], s[6], s[7]);
        t.s[2][i] = make_float4(s[8], s[9], s[10], s[11]);
    } else {
        t.s[0][i] = make_float4(s[0], s[1], s[2], s[3]);
        t.s[1][i] = make_float4(s[4], s[5], 0.0f, 0.0f);
    }
}

__device__ __forceinline__ float goal_distance(const float* s, const float* g)
{
    const float dx = __fsub_rn(s[0], g[0]), dy = __fsub_rn(s[1], g[1]), dz = __fsub_rn(s[2], g[2]);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

// ---------------------------------------------------------------- kernels

__global__ void k_begin(KParams p, TreeDev t, Ctl* ctl, const float* __restrict__ init_goal, uint32_t plan_idx,
                        uint32_t max_iters, uint32_t stop_at_goal)
{
    if(threadIdx.x != 0 || blockIdx.x != 0) return;
    float s[12] = {0};
    for(int k = 0; k < p.sd; ++k) s[k] = init_goal[k];
    if(p.sd == 12) store_state<12>(t, 0, s);
    else store_state<6>(t, 0, s);
    float c[4] = {0, 0, 0, 0};
    for(int k = 0; k < p.cd; ++k) c[k] = init_goal[p.sd + k];
    t.ctl[0] = make_float4(c[0], c[1], c[2], c[3]);
    t.dur[0] = init_goal[p.S - 1];
    t.parent[0] = -1;
    t.cost[0] = 0.0f;
    t.r1[0] = region_r1(p, s);
    t.rep[0] = (uint8_t)p.root_repeat;
    const uint32_t epoch = ctl->epoch + 1;
    Ctl z;
    memset(&z, 0, sizeof(z));
    z.tree = 1, z.tree_old = 0, z.iter = 1, z.goal_idx = kNone;
    z.plan_idx = plan_idx, z.max_iters = max_iters, z.stop_at_goal = stop_at_goal, z.epoch = epoch;
    z.goal[0] = init_goal[p.S], z.goal[1] = init_goal[p.S + 1], z.goal[2] = init_goal[p.S + 2];
    *ctl = z;
}

// Frontier pass 1: resolve every live node's repeat count (re-activation of the previous
// iteration, KPAX.cu:505-517; repeat of nodes added last iteration, KPAX.cu:476-479) and write
// one sum per tile of kTile nodes.  The last CTA to finish scans the tile sums, giving the total
// entry count R, and sets this iteration's budget (KPAX.cu:323-350).
__device__ __forceinline__ uint32_t resolve_repeat(const KParams& p, const TreeDev& t, const RegDev& rg, uint32_t i,
                                                   uint32_t tree_old, uint32_t iter, uint32_t plan, float fa, float total,
                                                   uint32_t ready)
{
    const uint32_t r0 = t.rep[i];
    uint32_t r = r0;
    if(r == 0u) {
        if(i < tree_old) {
            const float sc = region_score(rg.score[t.r1[i]], total, ready, p.eps);
            if(reactivate_draw(p, plan, iter - 1u, i) <= __fadd_rn(sc, fa)) r = 1u;
        }
    } else if(r == kPending) {
        r = rg.valid[t.r1[i]] < p.sparse_thr ? p.sparse_repeat : 1u;
    }
    if(r != r0) t.rep[i] = (uint8_t)r;
    return r;
}

__global__ void __launch_bounds__(kFrontierBS) k_frontier_count(KParams p, TreeDev t, RegDev rg, Ctl* ctl,
                                                                uint32_t* __restrict__ tile_sums, uint32_t* __restrict__ arrivals)
{
    __shared__ uint32_t s_done, s_last, s_carry;
    __shared__ uint32_t s_warp[kFrontierBS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(threadIdx.x == 0) s_done = ctl->done;
    __syncthreads();
    if(s_done) return;
    const uint32_t tree = ctl->tree, tree_old = ctl->tree_old, iter = ctl->iter, plan = ctl->plan_idx;
    const uint32_t ready = ctl->scores_ready;
    const float fa = ctl->faccept, total = ctl->score_total;
    const uint32_t ntiles = (tree + kTile - 1) / kTile;
    for(uint32_t b = blockIdx.x; b < ntiles; b += gridDim.x) {
        uint32_t sum = 0;
#pragma unroll
        for(int j = 0; j < kItems; ++j) {
            const uint32_t i = b * kTile + j * kFrontierBS + threadIdx.x;  // coalesced
            if(i < tree) sum += resolve_repeat(p, t, rg, i, tree_old, iter, plan, fa, total, ready);
        }
#pragma unroll
        for(int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
        if(lane == 0) s_warp[warp] = sum;
        __syncthreads();
        if(threadIdx.x == 0) {
            uint32_t acc = 0;
            for(int w = 0; w < kFrontierBS / 32; ++w) acc += s_warp[w];
            tile_sums[b] = acc;
        }
        __syncthreads();
    }
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) s_last = atomicAdd(arrivals, 1u) == gridDim.x - 1u;
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    // exclusive scan of the tile sums in place (kFrontierBS at a time), total R
    if(threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    volatile uint32_t* ts = tile_sums;
    for(uint32_t base = 0; base < ntiles; base += kFrontierBS) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < ntiles ? ts[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += y;
        }
        if(lane == 31) s_warp[warp] = x;
        __syncthreads();
        uint32_t wex = 0;
        for(int w = 0; w < warp; ++w) wex += s_warp[w];
        const uint32_t excl = s_carry + wex + x - v;
        if(i < ntiles) ts[i] = excl;
        __syncthreads();
        if(threadIdx.x == kFrontierBS - 1) s_carry = excl + v;
        __syncthreads();
    }
    if(threadIdx.x == 0) {
        *arrivals = 0u;
        const uint64_t R = s_carry;
        const uint32_t B = min(p.budget, p.cap - tree);
        uint32_t k = p.per_entry, E = 0, n = 0;
        if(B == 0) {
            ctl->full = 1u;
            ctl->done = 1u;
        } else if(R) {
            if(R * k > B) {
                k = (uint32_t)(B / R);
                if(k == 0) k = 1;
            }
            E = (uint32_t)(R < (uint64_t)(B / k) ? R : (uint64_t)(B / k));
            n = E * k;
        }
        ctl->R = (uint32_t)R;
        ctl->k = k, ctl->E = E, ctl->n = n;
    }
}

// Frontier pass 2: node i owns virtual entries [a, a + rep) with a from the tile scan.  Entry j
// of the E taken is virtual entry floor(j*R/E), i.e. node i writes entries ceil(a*E/R) ..
// ceil((a+rep)*E/R) - 1 (all of its entries when E == R).  Nodes with an entry taken leave the
// frontier (KPAX.cu:372).
__global__ void __launch_bounds__(kFrontierBS) k_frontier_write(KParams p, TreeDev t, Ctl* ctl,
                                                                const uint32_t* __restrict__ tile_pre,
                                                                uint32_t* __restrict__ entries)
{
    __shared__ uint32_t s_done;
    __shared__ uint32_t s_warp[kFrontierBS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(threadIdx.x == 0) s_done = ctl->done;
    __syncthreads();
    if(s_done) return;
    const uint32_t tree = ctl->tree, E = ctl->E;
    const uint64_t R = ctl->R;
    if(E == 0) return;
    const uint32_t ntiles = (tree + kTile - 1) / kTile;
    for(uint32_t b = blockIdx.x; b < ntiles; b += gridDim.x) {
        // kItems consecutive nodes per thread so the in-tile prefix is a plain block scan
        const uint32_t i0 = b * kTile + threadIdx.x * kItems;
        uint32_t cnt[kItems], sum = 0;
#pragma unroll
        for(int j = 0; j < kItems; ++j) {
            const uint32_t i = i0 + j;
            cnt[j] = i < tree ? (uint32_t)t.rep[i] : 0u;
            sum += cnt[j];
        }
        uint32_t x = sum;
#pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += y;
        }
        if(lane == 31) s_warp[warp] = x;
        __syncthreads();
        uint32_t wex = 0;
        for(int w = 0; w < warp; ++w) wex += s_warp[w];
        uint64_t a = (uint64_t)tile_pre[b] + wex + x - sum;
#pragma unroll
        for(int j = 0; j < kItems; ++j) {
            if(!cnt[j]) continue;
            const uint64_t bnd = a + cnt[j];
            const uint64_t lo = (a * E + R - 1) / R, hi = (bnd * E + R - 1) / R;
            for(uint64_t e = lo; e < hi; ++e) entries[e] = i0 + j;
            if(lo < hi) t.rep[i0 + j] = 0;
            a = bnd;
        }
        __syncthreads();
    }
}

template <int M>
__global__ void __launch_bounds__(kExpandBS) k_expand(KParams p, Grid g, TreeDev t, RegDev rg, Ctl* ctl,
                                                      const uint32_t* __restrict__ entries, unsigned long long* __restrict__ lb,
                                                      CaptureDev cap)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD, S = SD + CD + 1;
    constexpr int NW = kExpandBS / 32;
    __shared__ uint32_t s_b, s_done, s_excl, s_ok;
    __shared__ uint32_t s_wn[NW], s_wv[NW], s_ws[NW];
    if(threadIdx.x == 0) {
        s_done = ctl->done;
        s_b = s_done ? 0u : atomicAdd(&ctl->ticket2, 1u);
    }
    __syncthreads();
    if(s_done) return;
    const uint32_t n = ctl->n, k = ctl->k, tree = ctl->tree, iter = ctl->iter, plan = ctl->plan_idx, epoch = ctl->epoch;
    const uint32_t ready = ctl->scores_ready;
    const float total = ctl->score_total;
    const uint32_t nblk = n ? (n + kExpandBS - 1) / kExpandBS : 1u, b = s_b;
    if(b >= nblk) return;
    const uint32_t c = b * kExpandBS + threadIdx.x;
    const bool active = c < n;
    bool valid = false, next = false;
    float s[SD], cc[4], rc[4], u[6];
    uint32_t parent = 0;
    int r1v = 0, r2v = 0, steps = 0, steps_done = 0;
    if(active) {
        const uint32_t e = c / k;
        parent = entries[e];
        load_state<SD>(t, parent, s);
        child_draws(p, plan, iter, c, u);
        steps = draw_controls(p, u, cc);
        valid = propagate<M>(p, g, s, cc, steps, steps_done);
        r1v = region_r1(p, s);
        r2v = region_r2(p, s, r1v);
        atomicAdd(rg.counter + r1v, 1);
        if(valid) {
            atomicAdd(rg.valid + r1v, 1);
            const uint32_t word = (uint32_t)r2v >> 5, bit = 1u << (r2v & 31);
            const bool seen = (__ldg(rg.cur + word) & bit) != 0u;
            next = (u[5] < region_score(__ldg(rg.score + r1v), total, ready, p.eps)) || !seen;
            atomicOr(rg.nxt + word, bit);
        }
        row_controls<M>(cc, rc);
        if(cap.rows) {
            float* dst = cap.rows + (size_t)c * S;
            for(int q = 0; q < SD; ++q) dst[q] = s[q];
            for(int q = 0; q < CD; ++q) dst[SD + q] = rc[q];
            dst[SD + CD] = __fmul_rn(p.h, (float)steps);
            cap.valid[c] = valid, cap.r1[c] = r1v, cap.r2[c] = r2v, cap.next[c] = next, cap.parent[c] = (int32_t)parent;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t mn = __ballot_sync(0xffffffffu, next), mv = __ballot_sync(0xffffffffu, valid);
    const uint32_t rank = __popc(mn & ((1u << lane) - 1u));
    uint32_t wsteps = active ? (uint32_t)steps_done : 0u;  // RK4 steps executed (algorithmic work)
#pragma unroll
    for(int d = 16; d > 0; d >>= 1) wsteps += __shfl_xor_sync(0xffffffffu, wsteps, d);
    if(lane == 0) s_wn[warp] = __popc(mn), s_wv[warp] = __popc(mv), s_ws[warp] = wsteps;
    __syncthreads();
    if(warp == 0) {
        uint32_t acc = 0, nv = 0;
        unsigned long long ns = 0;
        for(int w = 0; w < NW; ++w) acc += s_wn[w], nv += s_wv[w], ns += s_ws[w];
        uint32_t excl = 0;
        bool ok = true;
        if(b == 0) {
            if(lane == 0) lb_publish(lb, epoch, 2u, acc);
        } else {
            if(lane == 0) lb_publish(lb + b, epoch, 1u, acc);
            ok = lb_exclusive(lb, b, epoch, excl);
            if(ok && lane == 0) lb_publish(lb + b, epoch, 2u, excl + acc);
        }
        if(lane == 0) {
            if(nv) atomicAdd(&ctl->n_valid, (unsigned long long)nv);
            if(ns) atomicAdd(&ctl->n_steps, ns);
            if(!ok) {
                atomicOr(&ctl->error, kErrTimeout);
                ctl->done = 1u;
            }
            if(ok && b == nblk - 1) ctl->appended = excl + acc;
            s_excl = excl;
            s_ok = ok;
        }
    }
    __syncthreads();
    if(!next || !s_ok) return;
    uint32_t wex = 0;  // accepted children of the lower warps of this block
    for(int w = 0; w < warp; ++w) wex += s_wn[w];
    const uint32_t slot = tree + s_excl + wex + rank;
    if(slot >= p.cap) {
        atomicOr(&ctl->error, kErrCapacity);
        return;
    }
    store_state<SD>(t, slot, s);
    t.ctl[slot] = make_float4(rc[0], rc[1], rc[2], rc[3]);
    t.dur[slot] = __fmul_rn(p.h, (float)steps);
    t.parent[slot] = (int32_t)parent;
    const float d = goal_distance(s, ctl->goal);
    t.cost[slot] = d;
    t.r1[slot] = r1v;
    t.rep[slot] = kPending;
    if(d < p.goal_thresh) atomicMin(&ctl->goal_idx, slot);
}

// Region scores (Graph.cu:233-358) over kScoreCTAs CTAs, one warp per partial sum j: lane m
// scores region j + 1024*m and the warp adds them in ascending region order; the last CTA to
// finish adds the 1024 partials with a fixed halving tree, so the total (and every normalised
// score) is bit-identical to the oracle's.  Scores are stored raw (negative = no valid sample) and
// normalised where they are read (region_score).
__global__ void __launch_bounds__(kScoreBS) k_scores(KParams p, RegDev rg, Ctl* ctl, float* __restrict__ partials,
                                                     uint32_t* __restrict__ arrivals)
{
    __shared__ float s_part[kPartials];
    __shared__ uint32_t s_done, s_last;
    const int tid = threadIdx.x, lane = tid & 31;
    if(tid == 0) s_done = ctl->done;
    __syncthreads();
    if(s_done) return;
    const uint32_t gtid = blockIdx.x * blockDim.x + tid, gsize = gridDim.x * blockDim.x;
    for(uint32_t w = gtid; w < p.r2_words; w += gsize) rg.cur[w] = rg.nxt[w];
    const int nwarps = gridDim.x * (kScoreBS / 32);
    for(int j = blockIdx.x * (kScoreBS / 32) + (tid >> 5); j < kPartials; j += nwarps) {
        float part = 0.0f;
        for(int m0 = 0; j + kPartials * m0 < p.num_r1; m0 += 32) {
            const int r = j + kPartials * (m0 + lane);
            float contrib = 0.0f;
            if(r < p.num_r1) {
                const int nv = rg.valid[r];
                float stored = -1.0f;  // region without valid samples: score 1
                if(nv > 0) {           // Graph.cu:241-256, coverage from an exact R2 popcount
                    const int cnt = rg.counter[r];
                    const uint32_t pc = popcount_range(rg.nxt, (uint64_t)r * p.P, (uint64_t)(r + 1) * p.P);
                    const float cov = __fdiv_rn((float)pc, (float)p.P);
                    const float fnv = __fadd_rn(p.eps, (float)nv);
                    const float fv = __fmul_rn(__fdiv_rn(fnv, __fadd_rn(fnv, (float)(cnt - nv))), p.vol);
                    const float fv2 = __fmul_rn(fv, fv), fv4 = __fmul_rn(fv2, fv2), cf = (float)cnt;
                    stored = contrib = __fdiv_rn(fv4, __fmul_rn(__fadd_rn(1.0f, cov), __fadd_rn(1.0f, __fmul_rn(cf, cf))));
                }
                rg.score[r] = stored;
            }
            for(int q = 0; q < 32; ++q) {
                const float v = __shfl_sync(0xffffffffu, contrib, q);
                if(j + kPartials * (m0 + q) < p.num_r1) part = __fadd_rn(part, v);
            }
        }
        if(lane == 0) partials[j] = part;
    }
    __threadfence();
    __syncthreads();
    if(tid == 0) s_last = atomicAdd(arrivals, 1u) == gridDim.x - 1u;
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    for(int j = tid; j < kPartials; j += kScoreBS) s_part[j] = ((volatile float*)partials)[j];
    __syncthreads();
    for(int s = kPartials / 2; s > 0; s >>= 1) {
        for(int j = tid; j < s; j += kScoreBS) s_part[j] = __fadd_rn(s_part[j], s_part[j + s]);
        __syncthreads();
    }
    if(tid == 0) {
        *arrivals = 0u;
        ctl->score_total = s_part[0];
        ctl->scores_ready = 1u;
        const uint32_t iter = ctl->iter, tree_old = ctl->tree, tree_new = tree_old + ctl->appended;
        ctl->tree_old = tree_old;
        ctl->tree = tree_new;
        const float a = __fsub_rn(1.0f, __fdiv_rn((float)tree_new, (float)p.cap));  // KPAX.cu:527-528
        const float a2 = __fmul_rn(a, a), a4 = __fmul_rn(a2, a2), a5 = __fmul_rn(a4, a);
        ctl->faccept = __fmul_rn(__fmul_rn((float)iter, p.eps), a5);
        ctl->n_exp += ctl->n;
        ctl->iters_done = iter;
        if(ctl->goal_idx != kNone && ctl->stop_at_goal) ctl->done = 1u;
        if(iter >= ctl->max_iters) ctl->done = 1u;
        ctl->iter = iter + 1u;
        ctl->epoch = ctl->epoch + 1u;
        ctl->ticket1 = 0u;
        ctl->ticket2 = 0u;
    }
}

// Re-activation of the last iteration without a scan (makes exported frontier flags final).
__global__ void k_reactivate(KParams p, TreeDev t, RegDev rg, const Ctl* ctl)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tree_old = ctl->tree_old;
    if(i >= tree_old || ctl->iters_done == 0u) return;
    const float sc = region_score(rg.score[t.r1[i]], ctl->score_total, ctl->scores_ready, p.eps);
    if(t.rep[i] == 0 && reactivate_draw(p, ctl->plan_idx, ctl->iter - 1u, i) <= __fadd_rn(sc, ctl->faccept)) t.rep[i] = 1;
}

// Goal-to-root walk (KPAX.cu:482-501), goal row first, root row last.
__global__ void k_path(KParams p, TreeDev t, Ctl* ctl, float* __restrict__ path, uint32_t max_rows)
{
    if(threadIdx.x != 0 || blockIdx.x != 0) return;
    int32_t node = ctl->goal_idx == kNone ? -1 : (int32_t)ctl->goal_idx;
    uint32_t len = 0;
    double cost = 0.0;
    while(node >= 0 && len < max_rows) {
        float s[12] = {0};
        if(p.sd == 12) load_state<12>(t, (uint32_t)node, s);
        else load_state<6>(t, (uint32_t)node, s);
        const float4 c = t.ctl[node];
        const float cv[4] = {c.x, c.y, c.z, c.w};
        float* dst = path + (size_t)len * p.S;
        for(int k = 0; k < p.sd; ++k) dst[k] = s[k];
        for(int k = 0; k < p.cd; ++k) dst[p.sd + k] = cv[k];
        dst[p.S - 1] = t.dur[node];
        const int32_t par = t.parent[node];
        if(par >= 0) cost += (double)t.dur[node];
        ++len;
        node = par;
    }
    ctl->path_len = len;
    ctl->path_cost = cost;
}

template <class T>
kpax_status dalloc(T** p, size_t n)
{
    *p = nullptr;
    if(!n) n = 1;
    KPAX_CUDA(cudaMalloc((void**)p, sizeof(T) * n));
    return KPAX_OK;
}

}  // namespace
}  // namespace kpax

using namespace kpax;

struct kpax_planner {
    kpax_config cfg{};
    KParams p{};
    cudaStream_t stream = nullptr;
    Env env;
    TreeDev tree{};
    RegDev reg{};
    CaptureDev cap{};
    bool capture_on = false;
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl = nullptr;
    float* d_init = nullptr;  // init row, then goal row
    float* d_obs_host = nullptr;
    uint32_t obs_host_cap = 0;
    uint32_t* d_entries = nullptr;
    uint32_t* d_tiles = nullptr;
    uint32_t* d_farrivals = nullptr;
    float* d_partials = nullptr;
    uint32_t* d_arrivals = nullptr;
    unsigned long long *d_lb1 = nullptr, *d_lb2 = nullptr;
    uint32_t nblk1 = 0, nblk2 = 0;
    float* d_path = nullptr;
    float* h_path = nullptr;
    uint32_t path_rows = 0;
    cudaGraphExec_t graph = nullptr;
    const void* graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
    int unroll = 8;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t plans = 0;
    bool begun = false;
    kpax_result last{};
    std::vector<void*> allocs;

    template <class T>
    kpax_status alloc(T** ptr, size_t n)
    {
        kpax_status st = dalloc(ptr, n);
        if(st == KPAX_OK) allocs.push_back((void*)*ptr);
        return st;
    }

    kpax_status init(const kpax_config& c)
    {
        cfg = c;
        kpax_status st = derive_params(c, &p);
        if(st != KPAX_OK) return st;
        unroll = c.unroll_iters > 0 ? c.unroll_iters : 8;
        KPAX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        KPAX_CUDA(cudaEventCreate(&ev0));
        KPAX_CUDA(cudaEventCreate(&ev1));
        const size_t cap_n = p.cap;
        const int planes = p.sd == 12 ? 3 : 2;
        for(int k = 0; k < 3; ++k) tree.s[k] = nullptr;
        for(int k = 0; k < planes; ++k)
            if((st = alloc(&tree.s[k], cap_n)) != KPAX_OK) return st;
        if(planes == 2) tree.s[2] = tree.s[1];
        if((st = alloc(&tree.ctl, cap_n)) || (st = alloc(&tree.dur, cap_n)) || (st = alloc(&tree.parent, cap_n)) ||
           (st = alloc(&tree.cost, cap_n)) || (st = alloc(&tree.r1, cap_n)) || (st = alloc(&tree.rep, cap_n)))
            return st;
        if((st = alloc(&reg.counter, p.num_r1)) || (st = alloc(&reg.valid, p.num_r1)) || (st = alloc(&reg.score, p.num_r1)) ||
           (st = alloc(&reg.cur, p.r2_words)) || (st = alloc(&reg.nxt, p.r2_words)))
            return st;
        nblk1 = (p.cap + kTile - 1) / kTile;
        nblk2 = (p.budget + kExpandBS - 1) / kExpandBS;
        if((st = alloc(&d_partials, kPartials)) || (st = alloc(&d_arrivals, 1)) || (st = alloc(&d_farrivals, 1)) ||
           (st = alloc(&d_tiles, (p.cap + kTile - 1) / kTile + 1)))
            return st;
        KPAX_CUDA(cudaMemsetAsync(d_arrivals, 0, sizeof(uint32_t), stream));
        KPAX_CUDA(cudaMemsetAsync(d_farrivals, 0, sizeof(uint32_t), stream));
        if((st = alloc(&d_entries, p.budget)) || (st = alloc(&d_lb1, nblk1)) || (st = alloc(&d_lb2, nblk2)) ||
           (st = alloc(&d_ctl, 1)) || (st = alloc(&d_init, 2 * (size_t)p.S)))
            return st;
        KPAX_CUDA(cudaMemsetAsync(d_lb1, 0, sizeof(unsigned long long) * nblk1, stream));
        KPAX_CUDA(cudaMemsetAsync(d_lb2, 0, sizeof(unsigned long long) * nblk2, stream));
        KPAX_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(Ctl), stream));
        KPAX_CUDA(cudaMemsetAsync(tree.rep, 0, cap_n, stream));
        path_rows = c.max_iter + 2;
        if((st = alloc(&d_path, (size_t)path_rows * p.S)) != KPAX_OK) return st;
        KPAX_CUDA(cudaMallocHost(&h_path, sizeof(float) * path_rows * p.S));
        KPAX_CUDA(cudaMallocHost(&h_ctl, sizeof(Ctl)));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        return KPAX_OK;
    }

    void release()
    {
        if(stream) cudaStreamSynchronize(stream);
        if(graph) cudaGraphExecDestroy(graph);
        for(void* a : allocs) cudaFree(a);
        allocs.clear();
        release_capture();
        env.release();
        if(h_path) cudaFreeHost(h_path);
        if(h_ctl) cudaFreeHost(h_ctl);
        for(cudaEvent_t e : tev) cudaEventDestroy(e);
        tev.clear();
        if(d_flush) cudaFree(d_flush), d_flush = nullptr;
        if(ev0) cudaEventDestroy(ev0);
        if(ev1) cudaEventDestroy(ev1);
        if(stream) cudaStreamDestroy(stream);
        graph = nullptr, h_path = nullptr, h_ctl = nullptr, stream = nullptr;
    }

    void release_capture()
    {
        void* bufs[6] = {cap.rows, cap.valid, cap.r1, cap.r2, cap.next, cap.parent};
        for(void* b : bufs)
            if(b) cudaFree(b);
        cap = CaptureDev{};
    }

    kpax_status set_capture(bool on)
    {
        if(on == capture_on) return KPAX_OK;
        if(graph) cudaGraphExecDestroy(graph), graph = nullptr;
        release_capture();
        capture_on = on;
        if(on) {
            kpax_status st;
            const size_t n = p.budget;
            if((st = dalloc(&cap.rows, n * p.S)) || (st = dalloc(&cap.valid, n)) || (st = dalloc(&cap.r1, n)) ||
               (st = dalloc(&cap.r2, n)) || (st = dalloc(&cap.next, n)) || (st = dalloc(&cap.parent, n)))
                return st;
        }
        return KPAX_OK;
    }

    // ev (optional): four events recorded before k_frontier, k_expand, k_scores and after k_scores.
    void launch_iteration(cudaEvent_t* ev = nullptr)
    {
        if(ev) cudaEventRecord(ev[0], stream);
        const uint32_t fgrid = std::min<uint32_t>(nblk1, kFrontierCTAs);
        k_frontier_count<<<fgrid, kFrontierBS, 0, stream>>>(p, tree, reg, d_ctl, d_tiles, d_farrivals);
        k_frontier_write<<<fgrid, kFrontierBS, 0, stream>>>(p, tree, d_ctl, d_tiles, d_entries);
        if(ev) cudaEventRecord(ev[1], stream);
        const Grid g = env.view();
        switch(p.model) {
            case KPAX_MODEL_DOUBLE_INTEGRATOR:
                k_expand<KPAX_MODEL_DOUBLE_INTEGRATOR><<<nblk2, kExpandBS, 0, stream>>>(p, g, tree, reg, d_ctl, d_entries, d_lb2, cap);
                break;
            case KPAX_MODEL_DUBINS_AIRPLANE:
                k_expand<KPAX_MODEL_DUBINS_AIRPLANE><<<nblk2, kExpandBS, 0, stream>>>(p, g, tree, reg, d_ctl, d_entries, d_lb2, cap);
                break;
            default:
                k_expand<KPAX_MODEL_QUADROTOR><<<nblk2, kExpandBS, 0, stream>>>(p, g, tree, reg, d_ctl, d_entries, d_lb2, cap);
                break;
        }
        if(ev) cudaEventRecord(ev[2], stream);
        k_scores<<<kScoreCTAs, kScoreBS, 0, stream>>>(p, reg, d_ctl, d_partials, d_arrivals);
        if(ev) cudaEventRecord(ev[3], stream);
    }

    void* d_flush = nullptr;
    uint64_t flush_cap = 0;
    std::vector<cudaEvent_t> tev;

    // Benchmark iterations: each optionally preceded (outside its events) by a write of
    // flush_bytes, which evicts the 126 MB L2, then the three kernels bracketed by events.
    kpax_status iterate_timed(uint32_t n, uint64_t flush, kpax_iter_timing* times, uint64_t* totals)
    {
        kpax_status st = sync_ctl();
        if(st != KPAX_OK) return st;
        Ctl c = *h_ctl;
        const Ctl c0 = c;
        c.max_iters = c.iters_done + n;
        c.stop_at_goal = 0u;
        c.done = (c.full || c.error) ? 1u : 0u;
        c.ticket1 = c.ticket2 = 0u;
        *h_ctl = c;
        KPAX_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
        if(flush > flush_cap) {
            if(d_flush) cudaFree(d_flush), d_flush = nullptr;
            KPAX_CUDA(cudaMalloc(&d_flush, flush));
            flush_cap = flush;
        }
        while(tev.size() < 4 * (size_t)n) {
            cudaEvent_t e;
            KPAX_CUDA(cudaEventCreate(&e));
            tev.push_back(e);
        }
        for(uint32_t i = 0; i < n; ++i) {
            if(flush) KPAX_CUDA(cudaMemsetAsync(d_flush, (int)(i & 0xff), flush, stream));
            launch_iteration(&tev[4 * (size_t)i]);
            KPAX_CHECK_LAUNCH();
            count_launch(4);
        }
        KPAX_CUDA(cudaStreamSynchronize(stream));
        for(uint32_t i = 0; i < n; ++i) {
            float a = 0, b = 0, d = 0, t = 0;
            cudaEvent_t* e = &tev[4 * (size_t)i];
            KPAX_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
            KPAX_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
            KPAX_CUDA(cudaEventElapsedTime(&d, e[2], e[3]));
            KPAX_CUDA(cudaEventElapsedTime(&t, e[0], e[3]));
            if(times) times[i] = kpax_iter_timing{t, a, b, d};
        }
        st = sync_ctl();
        if(st != KPAX_OK) return st;
        if(totals) {
            totals[0] = h_ctl->n_exp - c0.n_exp;
            totals[1] = h_ctl->n_valid - c0.n_valid;
            totals[2] = h_ctl->n_steps - c0.n_steps;
            totals[3] = (uint64_t)(h_ctl->tree - c0.tree);
        }
        if(h_ctl->error & kErrTimeout) return set_error("a device-side wait gave up"), KPAX_ETIMEOUT;
        return KPAX_OK;
    }

    kpax_status ensure_graph()
    {
        const void* key[4] = {env.d_obs, env.d_off, env.d_ent, cap.rows};
        if(graph && memcmp(key, graph_key, sizeof(key)) == 0) return KPAX_OK;
        if(graph) cudaGraphExecDestroy(graph), graph = nullptr;
        cudaGraph_t g = nullptr;
        KPAX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for(int i = 0; i < unroll; ++i) launch_iteration();
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if(e != cudaSuccess) return set_error("graph capture failed: %s", cudaGetErrorString(e)), KPAX_ECUDA;
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if(e != cudaSuccess) return set_error("graph instantiate failed: %s", cudaGetErrorString(e)), KPAX_ECUDA;
        memcpy(graph_key, key, sizeof(key));
        return KPAX_OK;
    }

    kpax_status begin(const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs, uint32_t max_iters,
                      uint32_t stop, bool record_start = true)
    {
        if(!h_init || !h_goal || (n_obs && !d_obstacles)) return set_error("plan: null argument"), KPAX_EINVAL;
        if(record_start) KPAX_CUDA(cudaEventRecord(ev0, stream));
        kpax_status st = env.build(p, d_obstacles, n_obs, stream);
        if(st != KPAX_OK) return st;
        KPAX_CUDA(cudaMemcpyAsync(d_init, h_init, sizeof(float) * p.S, cudaMemcpyHostToDevice, stream));
        KPAX_CUDA(cudaMemcpyAsync(d_init + p.S, h_goal, sizeof(float) * p.S, cudaMemcpyHostToDevice, stream));
        KPAX_CUDA(cudaMemsetAsync(reg.counter, 0, sizeof(int32_t) * p.num_r1, stream));
        KPAX_CUDA(cudaMemsetAsync(reg.valid, 0, sizeof(int32_t) * p.num_r1, stream));
        KPAX_CUDA(cudaMemsetAsync(reg.score, 0, sizeof(float) * p.num_r1, stream));
        KPAX_CUDA(cudaMemsetAsync(reg.cur, 0, sizeof(uint32_t) * p.r2_words, stream));
        KPAX_CUDA(cudaMemsetAsync(reg.nxt, 0, sizeof(uint32_t) * p.r2_words, stream));
        k_begin<<<1, 32, 0, stream>>>(p, tree, d_ctl, d_init, plans, max_iters, stop);
        KPAX_CHECK_LAUNCH();
        count_launch();
        ++plans;
        begun = true;
        return ensure_graph();
    }

    // Runs graphs until the device reports done; `guard` bounds the number of graph launches.
    // With poll = false all launches are queued first and the stream is synchronised once.
    kpax_status run(uint32_t guard, bool poll = true)
    {
        if(!poll) {
            for(uint32_t g = 0; g < guard; ++g) {
                KPAX_CUDA(cudaGraphLaunch(graph, stream));
                count_launch(4 * (uint64_t)unroll);
            }
        }
        for(uint32_t g = 0; poll && g < guard; ++g) {
            KPAX_CUDA(cudaGraphLaunch(graph, stream));
            count_launch(4 * (uint64_t)unroll);
            KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
            KPAX_CUDA(cudaStreamSynchronize(stream));
            if(h_ctl->done) break;
        }
        if(!poll) {
            KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
            KPAX_CUDA(cudaStreamSynchronize(stream));
        }
        if(h_ctl->error & kErrTimeout) return set_error("a device-side wait gave up"), KPAX_ETIMEOUT;
        if(h_ctl->error & kErrCapacity) return set_error("tree capacity exceeded"), KPAX_ECAPACITY;
        return KPAX_OK;
    }

    kpax_status finish(kpax_result* out)
    {
        k_path<<<1, 32, 0, stream>>>(p, tree, d_ctl, d_path, path_rows);
        KPAX_CHECK_LAUNCH();
        count_launch();
        KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        if(h_ctl->path_len)
            KPAX_CUDA(cudaMemcpyAsync(h_path, d_path, sizeof(float) * h_ctl->path_len * p.S, cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaEventRecord(ev1, stream));
        KPAX_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.0f;
        KPAX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        kpax_result r{};
        r.found = h_ctl->goal_idx != kNone;
        r.goal_idx = r.found ? h_ctl->goal_idx : 0u;
        r.path_len = h_ctl->path_len;
        r.tree_size = h_ctl->tree;
        r.iters = h_ctl->iters_done;
        r.tree_full = (int32_t)h_ctl->full;
        r.h_path = h_path;
        r.ms = ms;
        r.expansions = h_ctl->n_exp;
        r.valid_expansions = h_ctl->n_valid;
        r.path_cost = h_ctl->path_cost;
        last = r;
        if(out) *out = r;
        return KPAX_OK;
    }

    uint32_t guard_for(uint32_t iters) const { return iters / (uint32_t)unroll + 4u; }

    kpax_status sync_ctl()
    {
        KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        return KPAX_OK;
    }
};

extern "C" {

kpax_status kpax_create(const kpax_config* cfg, kpax_planner** out)
{
    if(!cfg || !out) return set_error("kpax_create: null argument"), KPAX_EINVAL;
    *out = nullptr;
    kpax_planner* pl = new kpax_planner();
    kpax_status st = pl->init(*cfg);
    if(st != KPAX_OK) {
        pl->release();
        delete pl;
        return st;
    }
    *out = pl;
    return KPAX_OK;
}

kpax_status kpax_destroy(kpax_planner* pl)
{
    if(!pl) return KPAX_OK;
    pl->release();
    delete pl;
    return KPAX_OK;
}

void* kpax_planner_stream(kpax_planner* pl) { return pl ? (void*)pl->stream : nullptr; }

kpax_status kpax_plan(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs,
                      int32_t save_tree, kpax_result* out)
{
    (void)save_tree;  // the tree always stays on the device; kpax_export_tree copies it out
    if(!pl) return set_error("kpax_plan: null planner"), KPAX_EINVAL;
    kpax_status st = pl->begin(h_init, h_goal, d_obstacles, n_obs, pl->cfg.max_iter, 1u);
    if(st != KPAX_OK) return st;
    st = pl->run(pl->guard_for(pl->cfg.max_iter));
    kpax_status st2 = pl->finish(out);
    return st != KPAX_OK ? st : st2;
}

kpax_status kpax_plan_host(kpax_planner* pl, const float* h_init, const float* h_goal, const float* h_obstacles, uint32_t n_obs,
                           kpax_result* out)
{
    if(!pl || (n_obs && !h_obstacles)) return set_error("kpax_plan_host: null argument"), KPAX_EINVAL;
    if(n_obs > pl->obs_host_cap) {
        if(pl->d_obs_host) cudaFree(pl->d_obs_host), pl->d_obs_host = nullptr;
        KPAX_CUDA(cudaMalloc(&pl->d_obs_host, sizeof(float) * 6 * n_obs));
        pl->obs_host_cap = n_obs;
    }
    KPAX_CUDA(cudaEventRecord(pl->ev0, pl->stream));
    if(n_obs)
        KPAX_CUDA(cudaMemcpyAsync(pl->d_obs_host, h_obstacles, sizeof(float) * 6 * n_obs, cudaMemcpyHostToDevice, pl->stream));
    kpax_status st = pl->begin(h_init, h_goal, pl->d_obs_host, n_obs, pl->cfg.max_iter, 1u, false);
    if(st != KPAX_OK) return st;
    st = pl->run(pl->guard_for(pl->cfg.max_iter));
    kpax_status st2 = pl->finish(out);
    return st != KPAX_OK ? st : st2;
}

kpax_status kpax_plan_begin(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs)
{
    if(!pl) return set_error("kpax_plan_begin: null planner"), KPAX_EINVAL;
    kpax_status st = pl->begin(h_init, h_goal, d_obstacles, n_obs, 0u, 0u);
    if(st != KPAX_OK) return st;
    return pl->sync_ctl();
}

kpax_status kpax_plan_iterate(kpax_planner* pl, uint32_t n_iters, int32_t stop_at_goal)
{
    if(!pl || !pl->begun) return set_error("kpax_plan_iterate: call kpax_plan_begin first"), KPAX_EINVAL;
    if(!n_iters) return KPAX_OK;
    kpax_status st = pl->sync_ctl();
    if(st != KPAX_OK) return st;
    Ctl c = *pl->h_ctl;
    if(c.full || c.error) return KPAX_OK;
    c.max_iters = c.iters_done + n_iters;
    c.stop_at_goal = stop_at_goal ? 1u : 0u;
    c.done = (stop_at_goal && c.goal_idx != kNone) ? 1u : 0u;
    c.ticket1 = c.ticket2 = 0;
    *pl->h_ctl = c;
    KPAX_CUDA(cudaMemcpyAsync(pl->d_ctl, pl->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, pl->stream));
    if(c.done) return pl->sync_ctl();
    if(!stop_at_goal) return pl->run((n_iters + (uint32_t)pl->unroll - 1u) / (uint32_t)pl->unroll, false);
    return pl->run(pl->guard_for(n_iters));
}

kpax_status kpax_plan_iterate_timed(kpax_planner* pl, uint32_t n_iters, uint64_t flush_bytes, kpax_iter_timing* h_times,
                                    uint64_t* h_totals)
{
    if(!pl || !pl->begun) return set_error("kpax_plan_iterate_timed: call kpax_plan_begin first"), KPAX_EINVAL;
    return pl->iterate_timed(n_iters, flush_bytes, h_times, h_totals);
}

kpax_status kpax_plan_result(kpax_planner* pl, kpax_result* out)
{
    if(!pl || !pl->begun) return set_error("kpax_plan_result: no plan"), KPAX_EINVAL;
    return pl->finish(out);
}

kpax_status kpax_export_tree(kpax_planner* pl, float* h_rows, int32_t* h_parents, float* h_costs, uint32_t max_rows,
                             uint32_t* n_rows)
{
    if(!pl) return set_error("kpax_export_tree: null planner"), KPAX_EINVAL;
    kpax_status st = pl->sync_ctl();
    if(st != KPAX_OK) return st;
    const uint32_t n = std::min(pl->h_ctl->tree, max_rows);
    if(n_rows) *n_rows = n;
    if(!n) return KPAX_OK;
    const KParams& p = pl->p;
    if(h_rows) {
        const int planes = p.sd == 12 ? 3 : 2;
        std::vector<float4> buf((size_t)n * (planes + 1));
        std::vector<float> dur(n);
        for(int k = 0; k < planes; ++k)
            KPAX_CUDA(cudaMemcpyAsync(buf.data() + (size_t)k * n, pl->tree.s[k], sizeof(float4) * n, cudaMemcpyDeviceToHost, pl->stream));
        KPAX_CUDA(cudaMemcpyAsync(buf.data() + (size_t)planes * n, pl->tree.ctl, sizeof(float4) * n, cudaMemcpyDeviceToHost, pl->stream));
        KPAX_CUDA(cudaMemcpyAsync(dur.data(), pl->tree.dur, sizeof(float) * n, cudaMemcpyDeviceToHost, pl->stream));
        KPAX_CUDA(cudaStreamSynchronize(pl->stream));
        for(uint32_t i = 0; i < n; ++i) {
            float* dst = h_rows + (size_t)i * p.S;
            for(int k = 0; k < p.sd; ++k) dst[k] = ((const float*)&buf[(size_t)(k / 4) * n + i])[k % 4];
            const float* c = (const float*)&buf[(size_t)planes * n + i];
            for(int k = 0; k < p.cd; ++k) dst[p.sd + k] = c[k];
            dst[p.S - 1] = dur[i];
        }
    }
    if(h_parents) KPAX_CUDA(cudaMemcpyAsync(h_parents, pl->tree.parent, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, pl->stream));
    if(h_costs) KPAX_CUDA(cudaMemcpyAsync(h_costs, pl->tree.cost, sizeof(float) * n, cudaMemcpyDeviceToHost, pl->stream));
    KPAX_CUDA(cudaStreamSynchronize(pl->stream));
    return KPAX_OK;
}

kpax_status kpax_export_regions(kpax_planner* pl, int32_t* h_counter, int32_t* h_valid, float* h_scores, uint32_t* h_r2_bits)
{
    if(!pl) return set_error("kpax_export_regions: null planner"), KPAX_EINVAL;
    const KParams& p = pl->p;
    if(h_counter) KPAX_CUDA(cudaMemcpyAsync(h_counter, pl->reg.counter, sizeof(int32_t) * p.num_r1, cudaMemcpyDeviceToHost, pl->stream));
    if(h_valid) KPAX_CUDA(cudaMemcpyAsync(h_valid, pl->reg.valid, sizeof(int32_t) * p.num_r1, cudaMemcpyDeviceToHost, pl->stream));
    if(h_scores) KPAX_CUDA(cudaMemcpyAsync(h_scores, pl->reg.score, sizeof(float) * p.num_r1, cudaMemcpyDeviceToHost, pl->stream));
    KPAX_CUDA(cudaMemcpyAsync(pl->h_ctl, pl->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, pl->stream));
    if(h_r2_bits) KPAX_CUDA(cudaMemcpyAsync(h_r2_bits, pl->reg.cur, sizeof(uint32_t) * p.r2_words, cudaMemcpyDeviceToHost, pl->stream));
    KPAX_CUDA(cudaStreamSynchronize(pl->stream));
    if(h_scores) {  // stored raw (negative = no valid sample); normalised as region_score does
        const float total = pl->h_ctl->score_total;
        const bool ready = pl->h_ctl->scores_ready != 0u;
        for(int r = 0; r < p.num_r1; ++r) {
            const float raw = h_scores[r];
            h_scores[r] = !ready ? 0.0f : (raw < 0.0f ? 1.0f : p.eps + raw / total);
        }
    }
    return KPAX_OK;
}

kpax_status kpax_export_frontier(kpax_planner* pl, uint8_t* h_repeat, int32_t* h_r1, uint32_t max_rows)
{
    if(!pl) return set_error("kpax_export_frontier: null planner"), KPAX_EINVAL;
    kpax_status st = pl->sync_ctl();
    if(st != KPAX_OK) return st;
    const uint32_t n = std::min(pl->h_ctl->tree, max_rows);
    if(pl->h_ctl->tree_old) {
        k_reactivate<<<(pl->h_ctl->tree_old + 255) / 256, 256, 0, pl->stream>>>(pl->p, pl->tree, pl->reg, pl->d_ctl);
        KPAX_CHECK_LAUNCH();
        count_launch();
    }
    if(n && h_repeat) KPAX_CUDA(cudaMemcpyAsync(h_repeat, pl->tree.rep, n, cudaMemcpyDeviceToHost, pl->stream));
    if(n && h_r1) KPAX_CUDA(cudaMemcpyAsync(h_r1, pl->tree.r1, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, pl->stream));
    KPAX_CUDA(cudaStreamSynchronize(pl->stream));
    return KPAX_OK;
}

kpax_status kpax_debug_capture(kpax_planner* pl, int32_t enable)
{
    if(!pl) return set_error("kpax_debug_capture: null planner"), KPAX_EINVAL;
    return pl->set_capture(enable != 0);
}

kpax_status kpax_export_children(kpax_planner* pl, float* h_rows, uint8_t* h_valid, int32_t* h_r1, int32_t* h_r2,
                                 uint8_t* h_next, int32_t* h_parent, uint32_t max_rows, uint32_t* n_children)
{
    if(!pl || !pl->capture_on) return set_error("kpax_export_children: capture is off"), KPAX_EINVAL;
    kpax_status st = pl->sync_ctl();
    if(st != KPAX_OK) return st;
    const uint32_t n = std::min(pl->h_ctl->n, max_rows);
    if(n_children) *n_children = n;
    if(!n) return KPAX_OK;
    const CaptureDev& c = pl->cap;
    if(h_rows) KPAX_CUDA(cudaMemcpyAsync(h_rows, c.rows, sizeof(float) * n * pl->p.S, cudaMemcpyDeviceToHost, pl->stream));
    if(h_valid) KPAX_CUDA(cudaMemcpyAsync(h_valid, c.valid, n, cudaMemcpyDeviceToHost, pl->stream));
    if(h_r1) KPAX_CUDA(cudaMemcpyAsync(h_r1, c.r1, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, pl->stream));
    if(h_r2) KPAX_CUDA(cudaMemcpyAsync(h_r2, c.r2, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, pl->stream));
    if(h_next) KPAX_CUDA(cudaMemcpyAsync(h_next, c.next, n, cudaMemcpyDeviceToHost, pl->stream));
    if(h_parent) KPAX_CUDA(cudaMemcpyAsync(h_parent, c.parent, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, pl->stream));
    KPAX_CUDA(cudaStreamSynchronize(pl->stream));
    return KPAX_OK;
}

}  // extern "C"

// kpax_plan_kernels.cuh — the per-iteration kernels of the plan loop, over a batch of queries.
//
// One iteration of the reference (KPAX.cu:94-105) is propagateFrontier (303-351),
// Graph::updateVertices (Graph.cu:207-227) and updateFrontier (520-543), with thrust scans over
// the full tree capacity and ~6 host synchronisations.  Here it is four kernels with every size
// on the device.  Each kernel serves many independent queries at once: blockIdx.y selects a
// query (through an index list), whose parameters, buffers and control block are described by a
// QueryDev copied into shared memory at block start.  A single plan is a batch of one.
//   k_frontier_count  re-activation of the previous iteration (KPAX.cu:505-517) and repeat counts
//                     of new nodes (476-479); tile sums; the last CTA scans them and sets the budget
//   k_frontier_write  order-preserving entry list (Planner.cu:52-80), strided when the budget is
//                     below the frontier; expanded nodes leave the frontier (KPAX.cu:372)
//   k_expand<model>   per child: draw, RK4 + per-step collision, R1/R2 ids, counters, frontier
//                     mark (KPAX.cu:381-396); stable append of accepted children with cost and
//                     goal test (458-502) through a decoupled look-back
//   k_scores          R2 snapshot update, region scores with a fixed-order total (Graph.cu:233-358),
//                     then the iteration bookkeeping (tree size, fAccept, stop flags)
// Deterministic replacements for the reference's races are listed in oracle/kpax_oracle.h.
#pragma once
#include <stdint.h>

#include "kpax_device.cuh"
#include "kpax_mlp_tc.cuh"

namespace kpax {
namespace plan {

constexpr uint8_t kPending = 255;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kFrontierBS = 256, kItems = 4, kTile = kFrontierBS * kItems;
constexpr int kFrontierMinBlocks = 4;  // resident count-pass CTAs per SM (register bound)
constexpr int kExpandBS = 448;  // default: 2^16 children over 148 SMs, one 14-warp block per SM
constexpr int kExpandBSMin = 128;  // smallest expansion block (sizes the look-back status array)
constexpr int kScoreBS = 256, kPartials = 1024;
constexpr uint32_t kSpinLimit = 1u << 22;  // ~4 s of polling before a wait gives up
constexpr uint32_t kErrTimeout = 1u, kErrCapacity = 2u, kErrProposal = mlp::tc::kErrWait;

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
    float* score;   // raw score; negative = region without valid samples
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
    uint32_t iters_done, path_len, scores_ready;
    uint32_t stop_req;  // persistent batch stages: the query is to finish at the next iteration's start
    float faccept, goal[3];
    float score_total, pad1[3];
    unsigned long long n_exp, n_valid, n_steps;
    unsigned long long t_begin_ns, t_done_ns;
    float path_cost, pad2;
    // k_iterate: device-clock nanoseconds spent in its phases (frontier, expansion, scores), summed
    // over launches
    unsigned long long t_front_ns, t_expand_ns, t_score_ns, pad3;
};

// Everything a kernel needs about one query.
struct alignas(16) QueryDev {
    KParams p;
    Grid g;
    TreeDev t;
    RegDev rg;
    CaptureDev cap;
    Ctl* ctl;
    uint32_t* entries;
    uint32_t* tiles;      // tile sums, then their exclusive prefixes
    uint32_t* farr;       // arrival counter of k_frontier_count
    unsigned long long* lb;  // look-back status of k_expand, one per block
    float* partials;      // kPartials partial score sums
    uint32_t* sarr;       // arrival counter of k_scores
    uint32_t* bar;        // grid barrier of k_iterate: arrivals (one word used)
    uint32_t* ctas;       // per-CTA repeat sums of k_iterate's frontier phase
    float* path;
    const float* init_goal;  // init row then goal row, S floats each
    // learned proposal (quadrotor queries that enabled it; null otherwise)
    const uint8_t* mlp_img;  // packed BF16 network image
    float* mix;              // one mixture record per frontier entry
    const uint32_t* occ;     // occupancy bits of the R1 workspace cells
    float prop_eps;          // fraction of draws kept uniform
    uint32_t path_rows, pad[2];
};

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Programmatic dependent launch: the iteration's kernels are launched so that each may start
// while its predecessor drains.  A kernel copies its (host-written) query descriptor first, then
// waits for the predecessor grid's completion and memory before touching anything it produced,
// and lets its own successor launch (the successor in turn waits for this grid to complete).
__device__ __forceinline__ void wait_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void release_successor() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Copies the block's query descriptor into shared memory (all threads call it).
__device__ __forceinline__ void load_query(const QueryDev* __restrict__ qs, const uint32_t* __restrict__ qidx, QueryDev& sq)
{
    const uint32_t q = qidx ? qidx[blockIdx.y] : blockIdx.y;
    const uint4* src = reinterpret_cast<const uint4*>(qs + q);
    uint4* dst = reinterpret_cast<uint4*>(&sq);
    for(int i = threadIdx.x; i < (int)(sizeof(QueryDev) / 16); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Marks a query finished; the first transition counts it off the batch's active count.
__device__ __forceinline__ void finish_query(Ctl* ctl, uint32_t* active)
{
    if(atomicExch(&ctl->done, 1u) == 0u) {
        ctl->t_done_ns = globaltimer();
        if(active) atomicSub(active, 1u);
    }
}

// The persistent batch stages never change `done` inside a stage (their CTAs derive their work
// from it): a query that is to stop records the request and its time, and k_batch_start applies
// it before the next iteration's first stage.
__device__ __forceinline__ void request_finish(Ctl* ctl)
{
    if(atomicExch(&ctl->stop_req, 1u) == 0u) ctl->t_done_ns = globaltimer();
}

// Status word: [epoch:30 | flag:2 | value:32]; flag 1 = block aggregate, 2 = inclusive prefix.
__device__ __forceinline__ void lb_publish(unsigned long long* slot, uint32_t epoch, uint32_t flag, uint32_t value)
{
    const unsigned long long w = ((unsigned long long)(epoch & 0x3FFFFFFFu) << 34) | ((unsigned long long)flag << 32) | value;
    __threadfence();
    atomicExch(slot, w);
}

// Exclusive prefix of tile b, computed by the 32 lanes of one warp: each probe reads the status
// of 32 predecessors at once and stops at the nearest inclusive prefix.  Returns false when a
// predecessor never published (bounded wait).
__device__ __forceinline__ bool lb_exclusive(unsigned long long* lb, uint32_t b, uint32_t epoch, uint32_t& excl,
                                             uint32_t spin_limit = kSpinLimit)
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
            if(++spins > spin_limit) {
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
        uint32_t m = __ldcg(bits + w);
        if(w == w0) m &= ~0u << (lo & 31);
        if(w == w1) {
            const uint32_t top = (uint32_t)((hi - 1) & 31);
            m &= top == 31 ? ~0u : ((1u << (top + 1)) - 1u);
        }
        n += __popc(m);
    }
    return n;
}

// Normalised score of a region (Graph.cu:297-304, 349-357) from its stored raw score; every
// score reads 0 before the first score pass of a plan (KPAX.cu:69).
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

// Root node and control block of each query (KPAX.cu:59-91).
__global__ void k_begin(const QueryDev* __restrict__ qs, uint32_t plan_base, uint32_t max_iters, uint32_t stop_at_goal)
{
    __shared__ QueryDev sq;
    load_query(qs, nullptr, sq);
    if(threadIdx.x != 0) return;
    const KParams& p = sq.p;
    const TreeDev& t = sq.t;
    const float* ig = sq.init_goal;
    float s[12] = {0};
    for(int k = 0; k < p.sd; ++k) s[k] = ig[k];
    if(p.sd == 12) store_state<12>(t, 0, s);
    else store_state<6>(t, 0, s);
    float c[4] = {0, 0, 0, 0};
    for(int k = 0; k < p.cd; ++k) c[k] = ig[p.sd + k];
    t.ctl[0] = make_float4(c[0], c[1], c[2], c[3]);
    t.dur[0] = ig[p.S - 1];
    t.parent[0] = -1;
    t.cost[0] = 0.0f;
    t.r1[0] = region_r1<12>(p, s);
    t.rep[0] = (uint8_t)p.root_repeat;
    Ctl* ctl = sq.ctl;
    const uint32_t epoch = ctl->epoch + 1;
    Ctl z;
    memset(&z, 0, sizeof(z));
    z.tree = 1, z.tree_old = 0, z.iter = 1, z.goal_idx = kNone;
    z.plan_idx = plan_base, z.max_iters = max_iters, z.stop_at_goal = stop_at_goal, z.epoch = epoch;
    z.goal[0] = ig[p.S], z.goal[1] = ig[p.S + 1], z.goal[2] = ig[p.S + 2];
    z.t_begin_ns = globaltimer();
    *ctl = z;
    sq.bar[0] = 0u;  // arrivals of k_iterate's grid barrier (a plan ended by a timeout may leave some)
    *sq.sarr = 0u, *sq.farr = 0u;
}

// Node i's repeat count after the iteration's start: r0 its stored byte, reg its region.
__device__ __forceinline__ uint32_t resolve_repeat(const KParams& p, const TreeDev& t, const RegDev& rg, uint32_t i,
                                                   uint32_t r0, int32_t reg, uint32_t tree_old, uint32_t iter,
                                                   uint32_t plan, float fa, float total, uint32_t ready)
{
    // the region's score and valid count: loaded whichever case applies
    const float raw = rg.score[reg];
    const int32_t nvalid = rg.valid[reg];
    uint32_t r = r0;
    if(r == 0u) {  // re-activation of the previous iteration (KPAX.cu:505-517)
        if(i < tree_old) {
            const float sc = region_score(raw, total, ready, p.eps);
            if(reactivate_draw(p, plan, iter - 1u, i) <= __fadd_rn(sc, fa)) r = 1u;
        }
    } else if(r == kPending) {  // repeat of a node added last iteration (KPAX.cu:476-479)
        r = nvalid < p.sparse_thr ? p.sparse_repeat : 1u;
    }
    if(r != r0) t.rep[i] = (uint8_t)r;
    return r;
}

// Exclusive scan of n tile sums in place by one CTA (kFrontierBS threads, up to kScanItems
// consecutive sums per thread and pass); returns the total.  The sums were written by other
// CTAs, so they are read through L2.
constexpr int kScanItems = 16;
__device__ __forceinline__ uint32_t scan_tiles(uint32_t* tiles, uint32_t n, uint32_t* s_warp, uint32_t* s_carry)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(threadIdx.x == 0) *s_carry = 0;
    __syncthreads();
    for(uint32_t base = 0; base < n; base += kFrontierBS * kScanItems) {
        const uint32_t i0 = base + threadIdx.x * kScanItems;
        uint32_t v[kScanItems], sum = 0;
#pragma unroll
        for(int j = 0; j < kScanItems; ++j) {
            v[j] = i0 + j < n ? __ldcg(tiles + i0 + j) : 0u;
            sum += v[j];
        }
        uint32_t x = sum;
#pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += y;
        }
        if(lane == 31) s_warp[warp] = x;
        __syncthreads();
        uint32_t wex = 0, pass = 0;
        for(int w = 0; w < kFrontierBS / 32; ++w) {
            wex += w < warp ? s_warp[w] : 0u;
            pass += s_warp[w];
        }
        uint32_t acc = *s_carry + wex + x - sum;
#pragma unroll
        for(int j = 0; j < kScanItems; ++j) {
            if(i0 + j < n) tiles[i0 + j] = acc;
            acc += v[j];
        }
        __syncthreads();
        if(threadIdx.x == 0) *s_carry += pass;
        __syncthreads();
    }
    return *s_carry;
}

// Tile b of the frontier count (kFrontierBS threads): repeats of its kTile nodes resolved, their sum
// stored in tiles[b].
__device__ __forceinline__ void count_tile(const QueryDev& sq, uint32_t b, uint32_t tree, uint32_t tree_old, uint32_t iter,
                                           uint32_t plan, float fa, float total, uint32_t ready, uint32_t* s_warp)
{
    static_assert(kItems == 4, "a thread's nodes are one 4-byte word of repeat bytes");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const TreeDev& t = sq.t;
    // four consecutive nodes per thread: their bytes and region ids in one load each when the
    // four lie inside the tree and the arrays are aligned for it (the planner's are 256-byte
    // aligned; kpax_frontier_compact's repeat bytes are the caller's)
    const uint32_t i0 = b * kTile + 4u * threadIdx.x;
    const bool vec = ((reinterpret_cast<uintptr_t>(t.rep) & 3u) | (reinterpret_cast<uintptr_t>(t.r1) & 15u)) == 0u;
    uint32_t r0[4] = {0u, 0u, 0u, 0u};
    int32_t reg[4] = {0, 0, 0, 0};
    if(vec && i0 + 3u < tree) {
        const uint32_t w = *reinterpret_cast<const uint32_t*>(t.rep + i0);
        const int4 g4 = *reinterpret_cast<const int4*>(t.r1 + i0);
        r0[0] = w & 0xFFu, r0[1] = (w >> 8) & 0xFFu, r0[2] = (w >> 16) & 0xFFu, r0[3] = w >> 24;
        reg[0] = g4.x, reg[1] = g4.y, reg[2] = g4.z, reg[3] = g4.w;
    } else {
#pragma unroll
        for(int j = 0; j < 4; ++j)
            if(i0 + j < tree) r0[j] = t.rep[i0 + j], reg[j] = t.r1[i0 + j];
    }
    uint32_t sum = 0;
#pragma unroll
    for(int j = 0; j < 4; ++j) {
        const uint32_t i = i0 + j;
        if(i < tree)
            sum += resolve_repeat(sq.p, t, sq.rg, i, r0[j], reg[j], tree_old, iter, plan, fa, total, ready);
    }
#pragma unroll
    for(int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, d);
    if(lane == 0) s_warp[warp] = sum;
    __syncthreads();
    if(threadIdx.x == 0) {
        uint32_t acc = 0;
        for(int w = 0; w < kFrontierBS / 32; ++w) acc += s_warp[w];
        sq.tiles[b] = acc;
    }
    __syncthreads();
}

// The budget of an iteration (KPAX.cu:323-350) from its frontier's R entries, by one thread:
// k children per entry and E entries taken, or B == 0 (the tree is full).
__device__ __forceinline__ void set_budget(const KParams& p, Ctl* ctl, uint64_t R, uint32_t tree, uint32_t& B)
{
    B = min(p.budget, p.cap - tree);
    uint32_t k = p.per_entry, E = 0, n = 0;
    if(B != 0 && R) {
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

__global__ void __launch_bounds__(kFrontierBS, kFrontierMinBlocks) k_frontier_count(const QueryDev* __restrict__ qs, uint32_t* __restrict__ active)
{
    __shared__ QueryDev sq;
    __shared__ uint32_t s_last, s_carry;
    __shared__ uint32_t s_warp[kFrontierBS / 32];
    load_query(qs, nullptr, sq);
    const KParams& p = sq.p;
    Ctl* ctl = sq.ctl;
    wait_predecessor();
    release_successor();
    if(__syncthreads_or(ctl->done != 0u)) return;  // one decision for the whole block: barriers follow
    const uint32_t tree = ctl->tree, tree_old = ctl->tree_old, iter = ctl->iter, plan = ctl->plan_idx;
    const uint32_t ready = ctl->scores_ready;
    const float fa = ctl->faccept, total = ctl->score_total;
    const uint32_t ntiles = (tree + kTile - 1) / kTile;
    for(uint32_t b = blockIdx.x; b < ntiles; b += gridDim.x)
        count_tile(sq, b, tree, tree_old, iter, plan, fa, total, ready, s_warp);
    __threadfence();
    __syncthreads();
    if(threadIdx.x == 0) s_last = atomicAdd(sq.farr, 1u) == gridDim.x - 1u;
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    const uint32_t R32 = scan_tiles(sq.tiles, ntiles, s_warp, &s_carry);  // exclusive prefixes; total R
    if(threadIdx.x == 0) {  // the budget of this iteration (KPAX.cu:323-350)
        *sq.farr = 0u;
        uint32_t B = 0;
        set_budget(p, ctl, R32, tree, B);
        if(B == 0) {
            ctl->full = 1u;
            finish_query(ctl, active);
        }
    }
}

// ceil(a * E / R), the first of the E entries taken at or after virtual entry a (entry j is virtual
// entry floor(j * R / E)); a <= R, so the product fits 64 bits.  A node's last bound is the next
// node's first, so a run of nodes divides once per node, and not at all when every entry is taken.
__device__ __forceinline__ uint64_t entry_ceil(uint64_t a, uint32_t E, uint64_t R)
{
    return E == R ? a : (a * E + R - 1) / R;
}

// Tile b of the entry list (kFrontierBS threads, kItems consecutive nodes each): node i owns virtual
// entries [a, a + rep) with a from the tile scan.
__device__ __forceinline__ void write_tile(const QueryDev& sq, uint32_t b, uint32_t tree, uint64_t R, uint32_t E,
                                           uint32_t* s_warp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const TreeDev& t = sq.t;
    const uint32_t i0 = b * kTile + threadIdx.x * kItems;  // consecutive nodes per thread
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
    uint64_t a = (uint64_t)__ldcg(sq.tiles + b) + wex + x - sum;
    uint64_t lo = sum ? entry_ceil(a, E, R) : 0;
#pragma unroll
    for(int j = 0; j < kItems; ++j) {
        if(!cnt[j]) continue;
        const uint64_t bnd = a + cnt[j], hi = entry_ceil(bnd, E, R);
        for(uint64_t e = lo; e < hi; ++e) sq.entries[e] = i0 + j;
        if(lo < hi) t.rep[i0 + j] = 0;
        a = bnd, lo = hi;
    }
    __syncthreads();
}

// Node i owns virtual entries [a, a + rep) with a from the tile scan.  Entry j of the E taken is
// virtual entry floor(j*R/E): node i writes entries ceil(a*E/R) .. ceil((a+rep)*E/R) - 1 (all of
// its entries when E == R).  Nodes with an entry taken leave the frontier.
__global__ void __launch_bounds__(kFrontierBS) k_frontier_write(const QueryDev* __restrict__ qs)
{
    __shared__ QueryDev sq;
    __shared__ uint32_t s_warp[kFrontierBS / 32];
    load_query(qs, nullptr, sq);
    Ctl* ctl = sq.ctl;
    wait_predecessor();
    release_successor();
    if(ctl->done) return;
    const uint32_t tree = ctl->tree, E = ctl->E;
    const uint64_t R = ctl->R;
    if(E == 0) return;
    const uint32_t ntiles = (tree + kTile - 1) / kTile;
    for(uint32_t b = blockIdx.x; b < ntiles; b += gridDim.x) write_tile(sq, b, tree, R, E, s_warp);
}

// Shared-memory scratch of the expansion tiles of one block.
template <int NW>
struct ExpandSmem {
    uint32_t excl, ok;
    uint32_t wn[NW], wv[NW], ws[NW];
};

// Expansion of a query's children (KPAX.cu:358-439 with 445-502).  Children form look-back tiles
// of BS consecutive children; this block processes tiles b = first, first + stride, ... (grid-stride
// rounds), so every tile only waits on tiles of its own round or earlier.  Per child: draws, RK4 with
// per-step checks and grid queries, R1/R2 ids, counters, frontier mark; accepted children are
// appended in child order.  Returns false when a look-back wait gave up (the query is then finished
// with an error).
template <int M, int BS>
__device__ __forceinline__ bool expand_tiles(QueryDev& sq, uint32_t n, uint32_t k, uint32_t first, uint32_t stride,
                                             uint32_t* __restrict__ active, ExpandSmem<BS / 32>& sm, bool defer_finish = false)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD, S = SD + CD + 1;
    constexpr int NW = BS / 32;
    const KParams& p = sq.p;
    Ctl* ctl = sq.ctl;
    const uint32_t tree = ctl->tree, iter = ctl->iter, plan = ctl->plan_idx, epoch = ctl->epoch;
    const uint32_t ready = ctl->scores_ready;
    const float total = ctl->score_total;
    const uint32_t ntile = n ? (n + BS - 1) / BS : 1u;
    const TreeDev& t = sq.t;
    const RegDev& rg = sq.rg;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for(uint32_t b = first; b < ntile; b += stride) {
        const uint32_t c = b * BS + threadIdx.x;
        const bool active_child = c < n;
        bool valid = false, next = false;
        float s[SD], cc[4], rc[4], u[6];
        uint32_t parent = 0;
        int r1v = 0, r2v = 0, steps = 0, steps_done = 0;
        if(active_child) {
            parent = __ldcg(sq.entries + c / k);  // written by other CTAs of a fused launch: through L2
            load_state<SD>(t, parent, s);
            const float d_parent = p.prune ? goal_distance(s, ctl->goal) : 0.0f;
            child_draws(p, plan, iter, c, u);
            if constexpr(M == KPAX_MODEL_QUADROTOR) {
                if(sq.mix) mlp::mixture_draws(p, sq.mix + (size_t)(c / k) * mlp::kMixFloats, sq.prop_eps, plan, iter, c, u);
            }
            steps = draw_controls(p, u, cc);
            valid = propagate<M>(p, sq.g, s, cc, steps, steps_done);
            r1v = region_r1<SD>(p, s);
            r2v = region_r2<SD>(p, s, r1v);
            atomicAdd(rg.counter + r1v, 1);
            if(valid) {
                atomicAdd(rg.valid + r1v, 1);
                const uint32_t word = (uint32_t)r2v >> 5, bit = 1u << (r2v & 31);
                const bool seen = (__ldg(rg.cur + word) & bit) != 0u;
                next = (u[5] < region_score(__ldg(rg.score + r1v), total, ready, p.eps)) || !seen;
                atomicOr(rg.nxt + word, bit);
                if(next && p.prune) next = prune_keep(p, d_parent, goal_distance(s, ctl->goal), plan, iter, c);
            }
            row_controls<M>(cc, rc);
            if(sq.cap.rows) {
                float* dst = sq.cap.rows + (size_t)c * S;
                for(int q = 0; q < SD; ++q) dst[q] = s[q];
                for(int q = 0; q < CD; ++q) dst[SD + q] = rc[q];
                dst[SD + CD] = __fmul_rn(p.h, (float)steps);
                sq.cap.valid[c] = valid, sq.cap.r1[c] = r1v, sq.cap.r2[c] = r2v, sq.cap.next[c] = next;
                sq.cap.parent[c] = (int32_t)parent;
            }
        }
        const uint32_t mn = __ballot_sync(0xffffffffu, next), mv = __ballot_sync(0xffffffffu, valid);
        const uint32_t rank = __popc(mn & ((1u << lane) - 1u));
        uint32_t wsteps = active_child ? (uint32_t)steps_done : 0u;  // RK4 steps executed (algorithmic work)
#pragma unroll
        for(int d = 16; d > 0; d >>= 1) wsteps += __shfl_xor_sync(0xffffffffu, wsteps, d);
        if(lane == 0) sm.wn[warp] = __popc(mn), sm.wv[warp] = __popc(mv), sm.ws[warp] = wsteps;
        __syncthreads();
        if(warp == 0) {
            uint32_t acc = 0, nv = 0;
            unsigned long long ns = 0;
            for(int w = 0; w < NW; ++w) acc += sm.wn[w], nv += sm.wv[w], ns += sm.ws[w];
            uint32_t excl = 0;
            bool ok = true;
            if(b == 0) {
                if(lane == 0) lb_publish(sq.lb, epoch, 2u, acc);
            } else {
                if(lane == 0) lb_publish(sq.lb + b, epoch, 1u, acc);
                ok = lb_exclusive(sq.lb, b, epoch, excl);
                if(ok && lane == 0) lb_publish(sq.lb + b, epoch, 2u, excl + acc);
            }
            if(lane == 0) {
                if(nv) atomicAdd(&ctl->n_valid, (unsigned long long)nv);
                if(ns) atomicAdd(&ctl->n_steps, ns);
                if(!ok) {
                    atomicOr(&ctl->error, kErrTimeout);
                    if(defer_finish) request_finish(ctl);
                    else finish_query(ctl, active);
                }
                if(ok && b == ntile - 1) ctl->appended = excl + acc;
                sm.excl = excl;
                sm.ok = ok;
            }
        }
        __syncthreads();
        const bool block_ok = sm.ok != 0u;
        if(next && block_ok) {
            uint32_t wex = 0;  // accepted children of the lower warps of this tile
            for(int w = 0; w < warp; ++w) wex += sm.wn[w];
            const uint32_t slot = tree + sm.excl + wex + rank;
            if(slot >= p.cap) {
                atomicOr(&ctl->error, kErrCapacity);
            } else {
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
        }
        if(!block_ok) return false;
        __syncthreads();  // the shared words are rewritten by the next round
    }
    return true;
}

// Expansion kernel of a batch: the children of query blockIdx.y (through qidx), tiles in grid-stride
// rounds over blockIdx.x.
template <int M, int BS>
__global__ void __launch_bounds__(BS, (512 / BS > 0 ? 512 / BS : 1)) k_expand(const QueryDev* __restrict__ qs, const uint32_t* __restrict__ qidx,
                                               uint32_t* __restrict__ active)
{
    __shared__ QueryDev sq;
    __shared__ ExpandSmem<BS / 32> sm;
    load_query(qs, qidx, sq);
    wait_predecessor();
    release_successor();
    if(__syncthreads_or(sq.ctl->done != 0u)) return;  // one decision for the whole block: barriers follow
    expand_tiles<M, BS>(sq, sq.ctl->n, sq.ctl->k, blockIdx.x, gridDim.x, active, sm);
}

// Region scores (Graph.cu:233-358): one warp per partial sum j; the warp scores groups of 32
// consecutive regions (g = j, j + 1024, ...: coalesced loads), adds each group by a xor butterfly
// and the groups in ascending order; the total is the 1024 partials added by a fixed halving tree,
// so it (and every normalised score) is bit-identical to the oracle's whichever warps compute the
// partials.  Raw scores are stored (negative = no valid sample) and normalised where they are read
// (region_score).  Threads gtid of gsize also copy the iteration's R2 bits into the snapshot;
// warps wg of nwarps compute partials.
__device__ __forceinline__ void score_partials(const QueryDev& sq, uint32_t gtid, uint32_t gsize, int wg, int nwarps)
{
    const KParams& p = sq.p;
    const RegDev& rg = sq.rg;
    const int lane = threadIdx.x & 31;
    for(uint32_t w = gtid; w < p.r2_words; w += gsize) rg.cur[w] = __ldcg(rg.nxt + w);
    const uint32_t ngroups = (p.num_r1 + 31) / 32;  // 32 consecutive regions per group
    const int used = (int)min(ngroups, (uint32_t)kPartials);  // partials at and above `used` stay 0
    for(int j = wg; j < used; j += nwarps) {
        float part = 0.0f;
        for(uint32_t grp = j; grp < ngroups; grp += kPartials) {
            const int r = 32 * grp + lane;
            float contrib = 0.0f;
            if(r < p.num_r1) {
                // counters and R2 bits were updated by atomics of other CTAs (of the same launch in
                // k_iterate): read through L2
                const int nv = __ldcg(rg.valid + r);
                float stored = -1.0f;  // region without valid samples: score 1
                if(nv > 0) {           // Graph.cu:241-256, coverage from an exact R2 popcount
                    const int cnt = __ldcg(rg.counter + r);
                    const uint32_t pc = popcount_range(rg.nxt, (uint64_t)r * p.P, (uint64_t)(r + 1) * p.P);
                    const float cov = __fdiv_rn((float)pc, (float)p.P);
                    const float fnv = __fadd_rn(p.eps, (float)nv);
                    const float fv = __fmul_rn(__fdiv_rn(fnv, __fadd_rn(fnv, (float)(cnt - nv))), p.vol);
                    const float fv2 = __fmul_rn(fv, fv), fv4 = __fmul_rn(fv2, fv2), cf = (float)cnt;
                    stored = contrib = __fdiv_rn(fv4, __fmul_rn(__fadd_rn(1.0f, cov), __fadd_rn(1.0f, __fmul_rn(cf, cf))));
                }
                rg.score[r] = stored;
            }
#pragma unroll
            for(int d = 16; d > 0; d >>= 1) contrib = __fadd_rn(contrib, __shfl_xor_sync(0xffffffffu, contrib, d));
            part = __fadd_rn(part, contrib);
        }
        if(lane == 0) sq.partials[j] = part;
    }
}

// Total of the partials by the block's first warp, then the iteration's bookkeeping by thread 0:
// tree size, fAccept (KPAX.cu:527-528), counters, stop flags.  All threads call it.
__device__ __forceinline__ void score_finish(const QueryDev& sq, uint32_t* __restrict__ active, bool defer_finish = false)
{
    constexpr int kRegs = kPartials / 32;  // partials per lane: lane l holds partials l + 32 m
    const KParams& p = sq.p;
    Ctl* ctl = sq.ctl;
    const int tid = threadIdx.x, lane = tid & 31;
    if(tid >= 32) return;
    const uint32_t ngroups = (p.num_r1 + 31) / 32;
    const int used = (int)min(ngroups, (uint32_t)kPartials);
    // halving tree over the partials (level s adds partial j + s into partial j, j < s); the levels
    // whose upper halves hold only the zero partials at and above `used` leave the lower entries
    // unchanged (x + 0 = x), so the tree starts at the first power of two not below `used` and
    // gives the same total.  Levels s >= 32 pair partials of the same lane (registers m and
    // m + s / 32), levels below 32 pair lanes (shuffles): the same additions in the same order.
    int half = 1;
    while(half < used) half <<= 1;
    float v[kRegs];
#pragma unroll
    for(int m = 0; m < kRegs; ++m) {
        const int j = lane + 32 * m;
        v[m] = j < used ? ((volatile float*)sq.partials)[j] : 0.0f;
    }
#pragma unroll
    for(int S = kRegs / 2; S >= 1; S >>= 1) {
        if(32 * 2 * S <= half) {
#pragma unroll
            for(int m = 0; m < S; ++m) v[m] = __fadd_rn(v[m], v[m + S]);
        }
    }
    for(int sh = min(half, 32) / 2; sh > 0; sh >>= 1) {
        const float o = __shfl_down_sync(0xffffffffu, v[0], sh);
        if(lane < sh) v[0] = __fadd_rn(v[0], o);
    }
    if(tid == 0) {
        ctl->score_total = v[0];
        ctl->scores_ready = 1u;
        // the block may hold the control block's line in L1 from earlier in a fused launch, while
        // other CTAs updated it since: volatile reads
        const volatile Ctl* vc = ctl;
        const uint32_t iter = vc->iter, tree_old = vc->tree, tree_new = tree_old + vc->appended;
        ctl->tree_old = tree_old;
        ctl->tree = tree_new;
        const float a = __fsub_rn(1.0f, __fdiv_rn((float)tree_new, (float)p.cap));  // KPAX.cu:527-528
        const float a2 = __fmul_rn(a, a), a4 = __fmul_rn(a2, a2), a5 = __fmul_rn(a4, a);
        ctl->faccept = __fmul_rn(__fmul_rn((float)iter, p.eps), a5);
        ctl->n_exp = vc->n_exp + vc->n;
        ctl->iters_done = iter;
        ctl->iter = iter + 1u;
        ctl->epoch = vc->epoch + 1u;
        if((vc->goal_idx != kNone && vc->stop_at_goal) || iter >= vc->max_iters) {
            if(defer_finish) request_finish(ctl);
            else finish_query(ctl, active);
        }
    }
}

// The score pass of a batch: query blockIdx.y; the last CTA of a query adds its partials.
__global__ void __launch_bounds__(kScoreBS) k_scores(const QueryDev* __restrict__ qs, uint32_t* __restrict__ active)
{
    __shared__ QueryDev sq;
    __shared__ uint32_t s_last;
    load_query(qs, nullptr, sq);
    const int tid = threadIdx.x;
    wait_predecessor();
    release_successor();
    if(sq.ctl->done) return;
    score_partials(sq, blockIdx.x * blockDim.x + tid, gridDim.x * blockDim.x, blockIdx.x * (kScoreBS / 32) + (tid >> 5),
                   gridDim.x * (kScoreBS / 32));
    __threadfence();
    __syncthreads();
    if(gridDim.x > 1) {  // the last CTA to arrive adds the partials
        if(tid == 0) s_last = atomicAdd(sq.sarr, 1u) == gridDim.x - 1u;
        __syncthreads();
        if(!s_last) return;
        __threadfence();
        if(tid == 0) *sq.sarr = 0u;
    }
    score_finish(sq, active);
}

// ---------------------------------------------------------------- fused iteration (single query)
// k_iterate runs one whole iteration in one launch: frontier count, entry list, expansion and
// region scores, separated by grid-wide barriers.  Every CTA must be resident (the host sizes the
// grid by the occupancy of the kernel), every barrier is bounded, and each phase computes exactly
// what the corresponding per-stage kernel computes (same per-node, per-child and per-region
// arithmetic, same partial sums), so plans are bit-identical to the per-stage path.

constexpr int kIterMaxCTAs = 1024;  // CTAs of a k_iterate launch
constexpr int kIterBatch = 8;       // nodes per thread whose loads are issued together

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a launch whose CTAs are all resident.  bar[0] counts arrivals over the
// launch's barriers without being reset in between: the CTA whose arrival returns `old` waits
// until the count reaches the next multiple of nblocks above it, so the last CTA to arrive passes
// at once and the others need one poll that sees its arrival (the last CTA of the launch resets
// the count once every CTA is past the last barrier).  Bounded: returns false after spin_limit
// polls.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t nblocks, uint32_t* s_flag,
                                             uint32_t spin_limit = kSpinLimit)
{
    __syncthreads();
    if(threadIdx.x == 0) {
        __threadfence();  // the block's writes before its arrival
        const uint32_t target = (atomicAdd(bar, 1u) / nblocks + 1u) * nblocks;
        bool ok = true;
        uint32_t spins = 0;
        while(ld_acquire(bar) < target) {
            if(++spins > spin_limit) {
                ok = false;
                break;
            }
            if(spins > 16) __nanosleep(32);
        }
        __threadfence();
        *s_flag = ok ? 1u : 0u;
    }
    __syncthreads();
    return *s_flag != 0u;
}

// Sum of v over the block (all threads call it; s_warp holds one word per warp).
template <int NW>
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* s_warp)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for(int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    __syncthreads();
    if(lane == 0) s_warp[warp] = v;
    __syncthreads();
    uint32_t t = 0;
    for(int w = 0; w < NW; ++w) t += s_warp[w];
    return t;
}

// ctl_line: the query's control block, whose line thread 0 prefetches into L2 while the block
// copies its descriptor (L2 is where the predecessor's writes land, so the prefetch cannot serve a
// stale copy; the fields are read after the predecessor completes).
// The whole iteration in one launch (kIterWhole), or split around the learned proposal pass:
// kIterFront (frontier count, budget, entry list) and kIterBack (expansion, scores), with
// k_propose launched between them.
constexpr int kIterWhole = 0, kIterFront = 1, kIterBack = 2;

template <int M, int BS, int PART = kIterWhole>
__global__ void __launch_bounds__(BS, (512 / BS > 0 ? 512 / BS : 1)) k_iterate(const QueryDev* __restrict__ qs,
                                                                             const Ctl* ctl_line,
                                                                             uint32_t* __restrict__ active)
{
    constexpr int NW = BS / 32;
    __shared__ QueryDev sq;
    __shared__ ExpandSmem<NW> sm;
    __shared__ uint32_t s_flag, s_last;
    __shared__ uint32_t s_warp[NW], s_warp2[NW];
    __shared__ unsigned long long s_t[3];  // phase start times (thread 0)
    if(threadIdx.x == 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(ctl_line));
    load_query(qs, nullptr, sq);
    const KParams& p = sq.p;
    const TreeDev& t = sq.t;
    const RegDev& rg = sq.rg;
    Ctl* ctl = sq.ctl;
    const uint32_t G = gridDim.x, cb = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    wait_predecessor();
    if(__syncthreads_or(ctl->done != 0u)) return;  // one decision for the whole grid: barriers follow
    if(tid == 0) s_t[0] = globaltimer();
    uint32_t k = 0, n = 0;  // children per entry and children of this iteration
    if constexpr(PART != kIterBack) {
        const uint32_t tree = ctl->tree, tree_old = ctl->tree_old, iter = ctl->iter, plan = ctl->plan_idx;
        const uint32_t ready = ctl->scores_ready;
        const float fa = ctl->faccept, total = ctl->score_total;

        // ---- frontier count (k_frontier_count): re-activation of the previous iteration
        // (KPAX.cu:505-517) and repeats of its new nodes (476-479) over this thread's contiguous nodes
        const uint32_t per_cta = (tree + G - 1) / G, per_thr = (per_cta + BS - 1) / BS;
        const uint32_t c_lo = min(tree, cb * per_cta), c_hi = min(tree, c_lo + per_cta);
        const uint32_t lo = min(c_hi, c_lo + (uint32_t)tid * per_thr), hi = min(c_hi, lo + per_thr);
        uint32_t sum = 0;
        for(uint32_t i0 = lo; i0 < hi; i0 += kIterBatch) {
            uint32_t r0[kIterBatch];
            int32_t reg[kIterBatch], nv[kIterBatch];
            float raw[kIterBatch];
    #pragma unroll
            for(int j = 0; j < kIterBatch; ++j) {  // each node's byte and region id, then its region's
                const uint32_t i = i0 + j;         // score and valid count: two rounds of loads per batch
                r0[j] = i < hi ? (uint32_t)t.rep[i] : 0u;
                reg[j] = i < hi ? t.r1[i] : 0;
            }
    #pragma unroll
            for(int j = 0; j < kIterBatch; ++j) raw[j] = rg.score[reg[j]], nv[j] = rg.valid[reg[j]];
    #pragma unroll
            for(int j = 0; j < kIterBatch; ++j) {
                const uint32_t i = i0 + j;
                if(i >= hi) continue;
                uint32_t r = r0[j];
                if(r == 0u) {
                    if(i < tree_old) {
                        const float sc = region_score(raw[j], total, ready, p.eps);
                        if(reactivate_draw(p, plan, iter - 1u, i) <= __fadd_rn(sc, fa)) r = 1u;
                    }
                } else if(r == kPending) {
                    r = nv[j] < p.sparse_thr ? p.sparse_repeat : 1u;
                }
                if(r != r0[j]) t.rep[i] = (uint8_t)r;
                sum += r;
            }
        }
        // this thread's exclusive prefix inside the CTA, and the CTA's sum
        uint32_t x = sum;
    #pragma unroll
        for(int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if(lane >= d) x += y;
        }
        if(lane == 31) s_warp[warp] = x;
        __syncthreads();
        uint32_t wex = 0, cta_sum = 0;
        for(int w = 0; w < NW; ++w) {
            wex += w < warp ? s_warp[w] : 0u;
            cta_sum += s_warp[w];
        }
        const uint32_t thr_excl = wex + x - sum;
        if(tid == 0) sq.ctas[cb] = cta_sum;
        if(!grid_barrier(sq.bar, G, &s_flag)) {
            if(tid == 0) atomicOr(&ctl->error, kErrTimeout), finish_query(ctl, active);
            return;
        }
        release_successor();  // every CTA is resident now

        // ---- budget (KPAX.cu:323-350) from the CTA sums, then the entry list (k_frontier_write)
        uint32_t tot = 0, pre = 0;
        for(uint32_t j = tid; j < G; j += BS) {
            const uint32_t v = __ldcg(sq.ctas + j);
            tot += v;
            pre += j < cb ? v : 0u;
        }
        const uint64_t R = block_sum<NW>(tot, s_warp);
        const uint32_t a_cta = block_sum<NW>(pre, s_warp2);
        const uint32_t B = min(p.budget, p.cap - tree);
        k = p.per_entry;
        uint32_t E = 0;
        if(B != 0 && R) {
            if(R * k > B) {
                k = (uint32_t)(B / R);
                if(k == 0) k = 1;
            }
            E = (uint32_t)(R < (uint64_t)(B / k) ? R : (uint64_t)(B / k));
            n = E * k;
        }
        if(cb == 0 && tid == 0) {
            ctl->R = (uint32_t)R;
            ctl->k = k, ctl->E = E, ctl->n = n;
            if(B == 0) {
                ctl->full = 1u;
                finish_query(ctl, active);
            }
        }
        if(B == 0) return;  // every CTA decides alike
        if(E) {
            uint64_t a = (uint64_t)a_cta + thr_excl;  // node i owns virtual entries [a, a + rep)
            uint64_t elo = sum ? entry_ceil(a, E, R) : 0;
            for(uint32_t i = lo; i < hi; ++i) {
                const uint32_t cnt = t.rep[i];
                if(!cnt) continue;
                const uint64_t bnd = a + cnt, ehi = entry_ceil(bnd, E, R);
                for(uint64_t e = elo; e < ehi; ++e) sq.entries[e] = i;
                if(elo < ehi) t.rep[i] = 0;
                a = bnd, elo = ehi;
            }
        }
        if constexpr(PART == kIterFront) {  // the proposal pass and kIterBack follow
            if(cb == 0 && tid == 0) ctl->t_front_ns += globaltimer() - s_t[0];
            return;
        }
        if(!grid_barrier(sq.bar, G, &s_flag)) {
            if(tid == 0) atomicOr(&ctl->error, kErrTimeout), finish_query(ctl, active);
            return;
        }
    } else {
        k = ctl->k, n = ctl->n;  // the budget and entry list of the front launch
    }
    if(tid == 0) s_t[1] = globaltimer();

    // ---- expansion (k_expand); a CTA whose look-back wait gave up has finished the query with an
    // error and still takes part in the barrier
    expand_tiles<M, BS>(sq, n, k, cb, G, active, sm);
    if(!grid_barrier(sq.bar, G, &s_flag)) {
        if(tid == 0) atomicOr(&ctl->error, kErrTimeout), finish_query(ctl, active);
        return;
    }
    if constexpr(PART == kIterBack) release_successor();  // every CTA is resident now
    if(tid == 0) s_t[2] = globaltimer();

    // ---- region scores (k_scores); the last CTA to finish adds the partials and closes the iteration
    score_partials(sq, cb * BS + tid, G * BS, (int)(cb * NW) + warp, (int)(G * NW));
    __threadfence();
    __syncthreads();
    if(tid == 0) s_last = atomicAdd(sq.sarr, 1u) == G - 1u;
    __syncthreads();
    if(!s_last) return;
    __threadfence();
    if(tid == 0) *sq.sarr = 0u, sq.bar[0] = 0u;  // every CTA is past the last grid barrier
    score_finish(sq, active);
    if(tid == 0) {
        const unsigned long long t4 = globaltimer();
        if constexpr(PART == kIterWhole) ctl->t_front_ns += s_t[1] - s_t[0];
        ctl->t_expand_ns += s_t[2] - s_t[1];
        ctl->t_score_ns += t4 - s_t[2];
    }
}

// Features of frontier entry `row` of query q: the entry's node and the query's goal.
__device__ __forceinline__ void entry_features(const QueryDev& q, uint32_t row, float x[mlp::kInPad])
{
    float s[12];
    load_state<12>(q.t, q.entries[row], s);
    const float g[3] = {q.ctl->goal[0], q.ctl->goal[1], q.ctl->goal[2]};
    mlp::features(q.p, q.occ, s, g, x);
}

// Rows of the proposal pass: the frontier entries of the iteration (k_frontier_write).
struct EntrySrc {
    static constexpr bool kDebug = false;
    const QueryDev* q;
    uint32_t E, row0;
    __device__ uint32_t tiles() const { return (E + mlp::tc::kRows - 1) / mlp::tc::kRows; }
    __device__ void seek(uint32_t tile) { row0 = tile * mlp::tc::kRows; }
    __device__ uint32_t rows() const { return min((uint32_t)mlp::tc::kRows, E - row0); }
    __device__ float* records() const { return q->mix + (size_t)row0 * mlp::kMixFloats; }
    __device__ void row_features(uint32_t r, float x[mlp::kInPad]) const { entry_features(*q, row0 + r, x); }
    __device__ void dump_h(int, uint32_t, uint32_t, const uint4*) const {}
    __device__ void dump_out(uint32_t, uint32_t, float) const {}
};

// Learned proposal of the quadrotor queries in qidx: one mixture record per frontier entry,
// from the BF16 tensor-core forward pass of the entry's node.  Runs between k_frontier_write
// and k_expand, which samples each child's draws from its entry's record.
__global__ void __launch_bounds__(mlp::tc::kThreads, 1) k_propose(const QueryDev* __restrict__ qs, const uint32_t* __restrict__ qidx)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ QueryDev sq;
    load_query(qs, qidx, sq);
    wait_predecessor();
    release_successor();
    if(sq.ctl->done || !sq.mix) return;
    EntrySrc src{&sq, sq.ctl->E, 0u};
    mlp::tc::forward(src, sq.mlp_img, smem, &sq.ctl->error);
}

__global__ void k_reactivate(const QueryDev* __restrict__ qs)
{
    __shared__ QueryDev sq;
    load_query(qs, nullptr, sq);
    const KParams& p = sq.p;
    const Ctl* ctl = sq.ctl;
    const uint32_t tree_old = ctl->tree_old;
    if(ctl->iters_done == 0u) return;
    for(uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < tree_old; i += gridDim.x * blockDim.x) {
        const float sc = region_score(sq.rg.score[sq.t.r1[i]], ctl->score_total, ctl->scores_ready, p.eps);
        if(sq.t.rep[i] == 0 && reactivate_draw(p, ctl->plan_idx, ctl->iter - 1u, i) <= __fadd_rn(sc, ctl->faccept))
            sq.t.rep[i] = 1;
    }
}

// Goal-to-root walk (KPAX.cu:482-501), goal row first, root row last.
__global__ void k_path(const QueryDev* __restrict__ qs)
{
    __shared__ QueryDev sq;
    load_query(qs, nullptr, sq);
    if(threadIdx.x != 0) return;
    const KParams& p = sq.p;
    const TreeDev& t = sq.t;
    Ctl* ctl = sq.ctl;
    int32_t node = ctl->goal_idx == kNone ? -1 : (int32_t)ctl->goal_idx;
    uint32_t len = 0;
    float cost = 0.0f;  // FP32 like every planner quantity, summed goal to root
    while(node >= 0 && len < sq.path_rows) {
        float s[12] = {0};
        if(p.sd == 12) load_state<12>(t, (uint32_t)node, s);
        else load_state<6>(t, (uint32_t)node, s);
        const float4 c = t.ctl[node];
        const float cv[4] = {c.x, c.y, c.z, c.w};
        float* dst = sq.path + (size_t)len * p.S;
        for(int k = 0; k < p.sd; ++k) dst[k] = s[k];
        for(int k = 0; k < p.cd; ++k) dst[p.sd + k] = cv[k];
        dst[p.S - 1] = t.dur[node];
        const int32_t par = t.parent[node];
        if(par >= 0) cost = __fadd_rn(cost, t.dur[node]);
        ++len;
        node = par;
    }
    ctl->path_len = len;
    ctl->path_cost = cost;
}

}  // namespace plan
}  // namespace kpax

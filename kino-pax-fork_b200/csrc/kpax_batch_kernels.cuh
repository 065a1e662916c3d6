// kpax_batch_kernels.cuh — the iteration stages of a batch of independent queries as persistent
// launches over all queries' work, with per-query offsets.
//
// A stage's work comes in units (node tiles of the frontier passes, child tiles of the expansion,
// groups of region partials of the score pass).  Every CTA computes the per-query unit counts and
// their exclusive offsets in shared memory, then takes its units — a contiguous share in the
// frontier and score passes, units b, b + G, b + 2G, ... in the expansion (whose look-back must
// only wait on lower units already taken) — finds each unit's query by binary search in the
// offsets, and loads that query's descriptor when the query changes.  A query's last unit to finish (per-query arrival counter) closes the query's
// stage: the tile scan and budget of the count pass, the score total and bookkeeping of the score
// pass.  Each unit runs the per-tile code of the single-query kernels (count_tile, write_tile,
// expand_tiles, score_partials, score_finish), so a query planned in a batch gives its single plan
// bit for bit.
//
// The offsets must be the same in every CTA, so a stage derives unit counts only from control-block
// fields that no kernel of the same stage writes: `done` changes only in k_batch_start, at the
// start of an iteration, which applies the finish requests the stages record (tree full in the count
// pass, goal or iteration cap in the score pass, a wait that gave up in the expansion).
#pragma once
#include "kpax_plan_kernels.cuh"

namespace kpax {
namespace plan {

constexpr uint32_t kBatchMaxQueries = 8192;  // per-query offsets in shared memory (32 KB)
constexpr int kBatchStartBS = 256;

// Unit counts of the nq queries -> exclusive offsets s_off[0..nq] (all threads of the block call
// it; s_warp holds one word per warp).  Returns the total.
template <int NW, class F>
__device__ __forceinline__ uint32_t query_offsets(uint32_t nq, uint32_t* s_off, uint32_t* s_warp, F units)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t per = (nq + blockDim.x - 1) / blockDim.x;
    const uint32_t lo = min(nq, threadIdx.x * per), hi = min(nq, lo + per);
    uint32_t sum = 0;
    for(uint32_t q = lo; q < hi; ++q) {
        const uint32_t c = units(q);
        s_off[q] = c;
        sum += c;
    }
    uint32_t x = sum;
#pragma unroll
    for(int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if(lane >= d) x += y;
    }
    __syncthreads();
    if(lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t a = x - sum, total = 0;
    for(int w = 0; w < NW; ++w) {
        a += w < warp ? s_warp[w] : 0u;
        total += s_warp[w];
    }
    for(uint32_t q = lo; q < hi; ++q) {
        const uint32_t c = s_off[q];
        s_off[q] = a;
        a += c;
    }
    if(threadIdx.x == 0) s_off[nq] = total;
    __syncthreads();
    return total;
}

// The query whose units hold global unit g (s_off[q] <= g < s_off[q + 1]).
__device__ __forceinline__ uint32_t find_query(const uint32_t* s_off, uint32_t nq, uint32_t g)
{
    uint32_t lo = 0, hi = nq;
    while(hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if(s_off[mid] <= g) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Contiguous share [lo, hi) of `total` units for this CTA: consecutive units mostly belong to the
// same query, so a CTA loads few descriptors (stages without waits between CTAs only).
__device__ __forceinline__ void unit_range(uint32_t total, uint32_t& lo, uint32_t& hi)
{
    const uint32_t per = (total + gridDim.x - 1) / gridDim.x;
    lo = min(total, blockIdx.x * per);
    hi = min(total, lo + per);
}

// Copies query q's descriptor into shared memory (all threads; the previous one is no longer read).
__device__ __forceinline__ void load_query_at(const QueryDev* __restrict__ qs, uint32_t q, QueryDev& sq)
{
    __syncthreads();
    const uint4* src = reinterpret_cast<const uint4*>(qs + q);
    uint4* dst = reinterpret_cast<uint4*>(&sq);
    for(int i = threadIdx.x; i < (int)(sizeof(QueryDev) / 16); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Start of an iteration: the finish requests of the previous stages take effect.
__global__ void __launch_bounds__(kBatchStartBS) k_batch_start(Ctl* __restrict__ ctls, uint32_t nq, uint32_t* __restrict__ active)
{
    wait_predecessor();
    release_successor();
    for(uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += gridDim.x * blockDim.x) {
        Ctl* c = ctls + q;
        if(!c->done && (c->full || c->error || c->stop_req)) {
            const unsigned long long t = c->t_done_ns;
            finish_query(c, active);
            if(c->stop_req && t) c->t_done_ns = t;  // the time the query stopped, not this launch's
        }
    }
}

// Frontier count over all queries: units are node tiles (k_frontier_count's tiles); the last tile
// of a query scans its tile sums and sets its budget, or marks the query full.
__global__ void __launch_bounds__(kFrontierBS) k_count_all(const QueryDev* __restrict__ qs,
                                                                              const Ctl* __restrict__ ctls, uint32_t nq)
{
    extern __shared__ uint32_t s_off[];
    __shared__ QueryDev sq;
    __shared__ uint32_t s_warp[kFrontierBS / 32], s_last, s_carry;
    wait_predecessor();
    release_successor();
    const uint32_t total = query_offsets<kFrontierBS / 32>(nq, s_off, s_warp, [&](uint32_t q) {
        const Ctl& c = ctls[q];
        return c.done ? 0u : (c.tree + kTile - 1) / kTile;
    });
    uint32_t cur = kNone, tree = 0, tree_old = 0, iter = 0, plan = 0, ready = 0, ntiles = 0;
    float fa = 0.0f, ftotal = 0.0f;
    uint32_t g0, g1;
    unit_range(total, g0, g1);
    for(uint32_t g = g0; g < g1; ++g) {
        const uint32_t q = find_query(s_off, nq, g);
        if(q != cur) {
            load_query_at(qs, q, sq);
            const Ctl* c = sq.ctl;
            tree = c->tree, tree_old = c->tree_old, iter = c->iter, plan = c->plan_idx, ready = c->scores_ready;
            fa = c->faccept, ftotal = c->score_total;
            ntiles = s_off[q + 1] - s_off[q];
            cur = q;
        }
        count_tile(sq, g - s_off[q], tree, tree_old, iter, plan, fa, ftotal, ready, s_warp);
        __threadfence();
        if(threadIdx.x == 0) s_last = atomicAdd(sq.farr, 1u) == ntiles - 1u;
        __syncthreads();
        if(s_last) {  // this query's last tile: scan its tile sums, set the budget
            __threadfence();
            const uint32_t R32 = scan_tiles(sq.tiles, ntiles, s_warp, &s_carry);
            if(threadIdx.x == 0) {
                *sq.farr = 0u;
                uint32_t B = 0;
                set_budget(sq.p, sq.ctl, R32, tree, B);
                if(B == 0) sq.ctl->full = 1u;  // finished by k_batch_start; later stages skip it
            }
            __syncthreads();
        }
    }
}

// Entry lists of all queries: units are node tiles of the queries that take entries.
__global__ void __launch_bounds__(kFrontierBS) k_write_all(const QueryDev* __restrict__ qs, const Ctl* __restrict__ ctls,
                                                          uint32_t nq)
{
    extern __shared__ uint32_t s_off[];
    __shared__ QueryDev sq;
    __shared__ uint32_t s_warp[kFrontierBS / 32];
    wait_predecessor();
    release_successor();
    const uint32_t total = query_offsets<kFrontierBS / 32>(nq, s_off, s_warp, [&](uint32_t q) {
        const Ctl& c = ctls[q];
        return (c.done || c.full || c.E == 0u) ? 0u : (c.tree + kTile - 1) / kTile;
    });
    uint32_t cur = kNone, tree = 0, E = 0;
    uint64_t R = 0;
    uint32_t g0, g1;
    unit_range(total, g0, g1);
    for(uint32_t g = g0; g < g1; ++g) {
        const uint32_t q = find_query(s_off, nq, g);
        if(q != cur) {
            load_query_at(qs, q, sq);
            tree = sq.ctl->tree, E = sq.ctl->E, R = sq.ctl->R;
            cur = q;
        }
        write_tile(sq, g - s_off[q], tree, R, E, s_warp);
    }
}

// Expansion of one model's queries (qidx, nq of them): units are BS-child tiles (one tile for a
// query without children, which publishes its empty append).  Look-back waits only on lower tiles
// of the same query, which lower global units hold: every CTA must be resident (the host sizes the
// grid by occupancy), and the successor is released only at completion.
// CTAs per SM the batch expansion is compiled for.  A batch has children for every SM many times
// over, so its expansion is bound by how many warps each SM interleaves: 256-child tiles run four
// (quadrotor, 64 registers a thread) or five (the 6-state models, 48) CTAs per SM, whatever that
// spills.  1024 mixed queries on a B200: 790 M valid expansions/s, against 785 at four CTAs for
// every model, 757 at three, 683 at one 512-child CTA (16 warps) and 629 at one 448-child CTA.
// Other tile sizes keep the single-query bound.
template <int M, int BS>
constexpr int kExpandAllMinBlocks = BS == 256 ? (M == KPAX_MODEL_QUADROTOR ? 4 : 5) : (512 / BS > 0 ? 512 / BS : 1);

template <int M, int BS>
__global__ void __launch_bounds__(BS, (kExpandAllMinBlocks<M, BS>)) k_expand_all(const QueryDev* __restrict__ qs,
                                                                                const Ctl* __restrict__ ctls,
                                                                                const uint32_t* __restrict__ qidx,
                                                                                uint32_t nq, uint32_t* __restrict__ active)
{
    extern __shared__ uint32_t s_off[];
    __shared__ QueryDev sq;
    __shared__ ExpandSmem<BS / 32> sm;
    __shared__ uint32_t s_warp[BS / 32];
    wait_predecessor();
    const uint32_t total = query_offsets<BS / 32>(nq, s_off, s_warp, [&](uint32_t i) {
        const Ctl& c = ctls[qidx[i]];
        return (c.done || c.full) ? 0u : (c.n ? (c.n + BS - 1) / BS : 1u);
    });
    uint32_t cur = kNone, n = 0, k = 0;
    for(uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
        const uint32_t i = find_query(s_off, nq, g);
        if(i != cur) {
            load_query_at(qs, qidx[i], sq);
            n = sq.ctl->n, k = sq.ctl->k;
            cur = i;
        }
        if(!expand_tiles<M, BS>(sq, n, k, g - s_off[i], 0x80000000u, active, sm, true)) return;
    }
}

// Expansion of all queries of every model in one launch (their models share the block size BS):
// the same units as k_expand_all over qidx, which lists the quadrotor queries first, then Dubins,
// then the double integrator, so the costliest tiles are taken first and the cheap ones fill the
// launch's tail.  Each unit runs the expansion of its query's model.
template <int BS>
__global__ void __launch_bounds__(BS, (512 / BS > 0 ? 512 / BS : 1)) k_expand_mixed(const QueryDev* __restrict__ qs,
                                                                                  const Ctl* __restrict__ ctls,
                                                                                  const uint32_t* __restrict__ qidx,
                                                                                  uint32_t nq, uint32_t* __restrict__ active)
{
    extern __shared__ uint32_t s_off[];
    __shared__ QueryDev sq;
    __shared__ ExpandSmem<BS / 32> sm;
    __shared__ uint32_t s_warp[BS / 32];
    wait_predecessor();
    const uint32_t total = query_offsets<BS / 32>(nq, s_off, s_warp, [&](uint32_t i) {
        const Ctl& c = ctls[qidx[i]];
        return (c.done || c.full) ? 0u : (c.n ? (c.n + BS - 1) / BS : 1u);
    });
    uint32_t cur = kNone, n = 0, k = 0;
    int model = 0;
    for(uint32_t g = blockIdx.x; g < total; g += gridDim.x) {
        const uint32_t i = find_query(s_off, nq, g);
        if(i != cur) {
            load_query_at(qs, qidx[i], sq);
            n = sq.ctl->n, k = sq.ctl->k, model = sq.p.model;
            cur = i;
        }
        const uint32_t t = g - s_off[i];
        bool ok;
        if(model == KPAX_MODEL_QUADROTOR) ok = expand_tiles<KPAX_MODEL_QUADROTOR, BS>(sq, n, k, t, 0x80000000u, active, sm, true);
        else if(model == KPAX_MODEL_DUBINS_AIRPLANE)
            ok = expand_tiles<KPAX_MODEL_DUBINS_AIRPLANE, BS>(sq, n, k, t, 0x80000000u, active, sm, true);
        else ok = expand_tiles<KPAX_MODEL_DOUBLE_INTEGRATOR, BS>(sq, n, k, t, 0x80000000u, active, sm, true);
        if(!ok) return;
    }
}

constexpr int kScoreUnitWarps = kScoreBS / 32;  // partial sums per score unit

// Region scores of all queries: a unit is kScoreUnitWarps consecutive partial sums of one query (and
// its share of the R2 snapshot copy); the query's last unit adds the partials and closes its
// iteration.
__global__ void __launch_bounds__(kScoreBS) k_scores_all(const QueryDev* __restrict__ qs, const Ctl* __restrict__ ctls,
                                                        uint32_t nq, uint32_t* __restrict__ active)
{
    extern __shared__ uint32_t s_off[];
    __shared__ QueryDev sq;
    __shared__ uint32_t s_warp[kScoreBS / 32], s_last;
    wait_predecessor();
    release_successor();
    const uint32_t total = query_offsets<kScoreBS / 32>(nq, s_off, s_warp, [&](uint32_t q) {
        const Ctl& c = ctls[q];  // not stop_req: this stage writes it
        if(c.done || c.full || c.error) return 0u;
        const uint32_t used = min(((uint32_t)qs[q].p.num_r1 + 31) / 32, (uint32_t)kPartials);
        return (used + kScoreUnitWarps - 1) / kScoreUnitWarps;
    });
    uint32_t cur = kNone, units = 0;
    const int tid = threadIdx.x;
    uint32_t g0, g1;
    unit_range(total, g0, g1);
    for(uint32_t g = g0; g < g1; ++g) {
        const uint32_t q = find_query(s_off, nq, g);
        if(q != cur) {
            load_query_at(qs, q, sq);
            units = s_off[q + 1] - s_off[q];
            cur = q;
        }
        const uint32_t u = g - s_off[q];
        score_partials(sq, u * kScoreBS + tid, units * kScoreBS, (int)(u * kScoreUnitWarps) + (tid >> 5),
                       (int)(units * kScoreUnitWarps));
        __threadfence();
        __syncthreads();
        if(tid == 0) s_last = atomicAdd(sq.sarr, 1u) == units - 1u;
        __syncthreads();
        if(s_last) {
            __threadfence();
            if(tid == 0) *sq.sarr = 0u;
            score_finish(sq, active, true);
        }
        __syncthreads();
    }
}

// The proposal pass of a batch as one persistent launch: the entries of every learned query,
// concatenated tile by tile, are spread over all CTAs (CTA b takes tiles b, b + gridDim.x, ...),
// so the pass is balanced however the entries are spread over the queries.  off[j] is the first
// tile of learned query j (k_propose_tiles), off[nl] the number of tiles.
struct BatchEntrySrc {
    static constexpr bool kDebug = false;
    const QueryDev* qs;
    const uint32_t* qidx;
    const uint32_t* off;
    uint32_t nl;
    uint32_t j, row0, E;  // cursor: learned query, first row of the tile, the query's entries
    const QueryDev* q;
    __device__ uint32_t tiles() const { return off[nl]; }
    __device__ void seek(uint32_t tile)
    {
        while(off[j + 1] <= tile) ++j;  // tile < off[nl], so j stays below nl
        q = qs + qidx[j];
        row0 = (tile - off[j]) * mlp::tc::kRows;
        E = q->ctl->E;
    }
    __device__ uint32_t rows() const { return min((uint32_t)mlp::tc::kRows, E - row0); }
    __device__ float* records() const { return q->mix + (size_t)row0 * mlp::kMixFloats; }
    __device__ void row_features(uint32_t r, float x[mlp::kInPad]) const { entry_features(*q, row0 + r, x); }
    __device__ void dump_h(int, uint32_t, uint32_t, const uint4*) const {}
    __device__ void dump_out(uint32_t, uint32_t, float) const {}
};

// Tile offsets of the batch proposal pass (one CTA of kPropTilesBS threads, nl <= kBatchMaxQueries): off[j] = tiles of
// the learned queries before j, off[nl] = all; a query that has finished, or takes no entries
// this iteration, has none.
constexpr int kPropTilesBS = 1024;
__global__ void __launch_bounds__(kPropTilesBS) k_propose_tiles(const QueryDev* __restrict__ qs, const uint32_t* __restrict__ qidx,
                                                                uint32_t nl, uint32_t* __restrict__ off)
{
    constexpr int kPer = (kBatchMaxQueries + kPropTilesBS - 1) / kPropTilesBS;
    __shared__ uint32_t s_warp[kPropTilesBS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    wait_predecessor();
    release_successor();
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for(int i = 0; i < kPer; ++i) {
        const uint32_t j = (uint32_t)tid * kPer + i;
        v[i] = 0u;
        if(j < nl) {
            const QueryDev& q = qs[qidx[j]];
            const Ctl* ctl = q.ctl;
            v[i] = (ctl->done || !q.mix) ? 0u : (ctl->E + mlp::tc::kRows - 1) / mlp::tc::kRows;
        }
        sum += v[i];
    }
    uint32_t x = sum;
#pragma unroll
    for(int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if(lane >= d) x += y;
    }
    if(lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t acc = x - sum;
    for(int w = 0; w < warp; ++w) acc += s_warp[w];
#pragma unroll
    for(int i = 0; i < kPer; ++i) {
        const uint32_t j = (uint32_t)tid * kPer + i;
        if(j < nl) off[j] = acc;
        acc += v[i];
        if(j + 1 == nl) off[nl] = acc;
    }
}

__global__ void __launch_bounds__(mlp::tc::kThreads, 1) k_propose_all(const QueryDev* __restrict__ qs, const uint32_t* __restrict__ qidx,
                                                                       uint32_t nl, const uint32_t* __restrict__ off, uint32_t* __restrict__ err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    wait_predecessor();
    release_successor();
    BatchEntrySrc src{qs, qidx, off, nl, 0u, 0u, 0u, nullptr};
    const bool ok = mlp::tc::forward(src, qs[qidx[0]].mlp_img, smem, err);
    if(!ok && threadIdx.x == 0)  // a wait gave up: the learned queries stop at this iteration's scores
        for(uint32_t j = 0; j < nl; ++j) atomicOr(&qs[qidx[j]].ctl->error, mlp::tc::kErrWait);
}

}  // namespace plan
}  // namespace kpax

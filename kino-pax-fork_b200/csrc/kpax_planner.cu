// kpax_planner.cu — host side of the plan loop: per-query buffers, descriptors, CUDA-graph
// capture of the iteration kernels (kpax_plan_kernels.cuh), and the C ABI for single plans
// (KPAX::plan, KPAX.cu:51-115) and batches of independent queries.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <filesystem>
#include <new>
#include <string>
#include <vector>

#include "kpax_batch_kernels.cuh"
#include "kpax_internal.h"
#include "kpax_plan_kernels.cuh"

using namespace kpax;
using namespace kpax::plan;

namespace {

constexpr int kFrontierCTAs = kFrontierMinBlocks * 148;  // one round over the tiles of a 600k-node tree
constexpr int kScoreCTAs = 128;
constexpr size_t kAlign = 256;

// Sub-allocations of one device allocation.
struct Carver {
    char* base = nullptr;
    size_t used = 0;
    template <class T>
    T* take(size_t n)
    {
        used = (used + kAlign - 1) / kAlign * kAlign;
        T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
        used += sizeof(T) * (n ? n : 1);
        return p;
    }
};

// Launch of an iteration kernel that may start while the previous kernel of its stream drains
// (programmatic dependent launch; the kernel waits on its predecessor before reading its results).
template <typename... P, typename... A>
void launch_chained(void (*kernel)(P...), dim3 grid, unsigned block, size_t smem, cudaStream_t s, A... args)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = dim3(block);
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    cudaLaunchKernelEx(&lc, kernel, static_cast<P>(args)...);
}

// The expansion kernel at one of its block sizes (validated by kpax_config_validate).
template <int M>
void launch_expand(int bs, dim3 grid, cudaStream_t s, const QueryDev* dq, const uint32_t* qidx, uint32_t* active)
{
    switch(bs) {
        case 128: launch_chained(k_expand<M, 128>, grid, 128, 0, s, dq, qidx, active); break;
        case 256: launch_chained(k_expand<M, 256>, grid, 256, 0, s, dq, qidx, active); break;
        case 512: launch_chained(k_expand<M, 512>, grid, 512, 0, s, dq, qidx, active); break;
        default: launch_chained(k_expand<M, kExpandBS>, grid, kExpandBS, 0, s, dq, qidx, active); break;
    }
}

// The fused iteration kernel (or one of its two parts around the proposal pass) at one of its
// block sizes.
template <int M, int PART = kIterWhole>
void* iterate_kernel(int bs)
{
    switch(bs) {
        case 128: return (void*)k_iterate<M, 128, PART>;
        case 256: return (void*)k_iterate<M, 256, PART>;
        case 512: return (void*)k_iterate<M, 512, PART>;
        default: return (void*)k_iterate<M, kExpandBS, PART>;
    }
}

template <int M, int PART = kIterWhole>
void launch_iterate(int bs, uint32_t gx, cudaStream_t s, const QueryDev* dq, const Ctl* ctl, uint32_t* active)
{
    switch(bs) {
        case 128: launch_chained(k_iterate<M, 128, PART>, dim3(gx), 128, 0, s, dq, ctl, active); break;
        case 256: launch_chained(k_iterate<M, 256, PART>, dim3(gx), 256, 0, s, dq, ctl, active); break;
        case 512: launch_chained(k_iterate<M, 512, PART>, dim3(gx), 512, 0, s, dq, ctl, active); break;
        default: launch_chained(k_iterate<M, kExpandBS, PART>, dim3(gx), kExpandBS, 0, s, dq, ctl, active); break;
    }
}

// The persistent expansion of a batch's model group at one of its block sizes.
template <int M>
void* expand_all_kernel(int bs)
{
    switch(bs) {
        case 128: return (void*)k_expand_all<M, 128>;
        case 256: return (void*)k_expand_all<M, 256>;
        case 512: return (void*)k_expand_all<M, 512>;
        default: return (void*)k_expand_all<M, kExpandBS>;
    }
}

template <int M>
void launch_expand_all(int bs, uint32_t gx, size_t smem, cudaStream_t s, const QueryDev* dq, const Ctl* ctls,
                       const uint32_t* qidx, uint32_t nq, uint32_t* active)
{
    switch(bs) {
        case 128: launch_chained(k_expand_all<M, 128>, dim3(gx), 128, smem, s, dq, ctls, qidx, nq, active); break;
        case 256: launch_chained(k_expand_all<M, 256>, dim3(gx), 256, smem, s, dq, ctls, qidx, nq, active); break;
        case 512: launch_chained(k_expand_all<M, 512>, dim3(gx), 512, smem, s, dq, ctls, qidx, nq, active); break;
        default: launch_chained(k_expand_all<M, kExpandBS>, dim3(gx), kExpandBS, smem, s, dq, ctls, qidx, nq, active); break;
    }
}

void* expand_mixed_kernel(int bs)
{
    switch(bs) {
        case 128: return (void*)k_expand_mixed<128>;
        case 256: return (void*)k_expand_mixed<256>;
        case 512: return (void*)k_expand_mixed<512>;
        default: return (void*)k_expand_mixed<kExpandBS>;
    }
}

void launch_expand_mixed(int bs, uint32_t gx, size_t smem, cudaStream_t s, const QueryDev* dq, const Ctl* ctls,
                         const uint32_t* qidx, uint32_t nq, uint32_t* active)
{
    switch(bs) {
        case 128: launch_chained(k_expand_mixed<128>, dim3(gx), 128, smem, s, dq, ctls, qidx, nq, active); break;
        case 256: launch_chained(k_expand_mixed<256>, dim3(gx), 256, smem, s, dq, ctls, qidx, nq, active); break;
        case 512: launch_chained(k_expand_mixed<512>, dim3(gx), 512, smem, s, dq, ctls, qidx, nq, active); break;
        default: launch_chained(k_expand_mixed<kExpandBS>, dim3(gx), kExpandBS, smem, s, dq, ctls, qidx, nq, active); break;
    }
}

struct PlanBatch {
    uint32_t nq = 0;
    std::vector<kpax_config> cfg;
    std::vector<KParams> prm;
    std::vector<Env> env;
    std::vector<QueryDev> hq;
    std::vector<uint32_t> path_off;  // row offset of each query's path in the path buffers
    QueryDev* dq = nullptr;
    char* pool = nullptr;
    size_t region_lo = 0, region_hi = 0;  // byte range of all region buffers (cleared per plan)
    std::vector<uint32_t> groups[3];      // query indices per model (DI, Dubins, quad)
    uint32_t* d_groups[3] = {nullptr, nullptr, nullptr};
    uint32_t expand_gx[3] = {0, 0, 0};
    int expand_bs[3] = {kExpandBS, kExpandBS, kExpandBS};  // block size per model group (its first query's)
    uint32_t gx_front = 1, gx_score = 1;
    bool persistent = false;  // batch: persistent stage launches over all queries (per-query offsets)
    uint32_t gx_count_all = 0, gx_write_all = 0, gx_scores_all = 0, gx_expand_all[3] = {0, 0, 0};
    // every model group at one block size: one mixed-model expansion over all queries, quadrotor first
    int mixed_bs = 0;
    uint32_t gx_mixed = 0;
    uint32_t* d_mixed = nullptr;
    // the batch's expansion: 1 (default) one persistent launch per model group over its queries'
    // tiles, groups one after another, each at its model's own occupancy; 2 one persistent launch
    // for every model (the quadrotor's register budget for all); 0 one block per child tile of every
    // query, model groups on concurrent streams.  KPAX_BATCH_EXPAND=0|2 selects the alternatives
    // for measurements; the plans are the same.
    int expand_mode = 1;
    bool fused = false;      // single query without the proposal: one k_iterate launch per iteration
    bool fused_split = false;  // single quadrotor query with the proposal: front, proposal pass, back
    uint32_t gx_split = 0;     // CTAs of the front and back launches (all resident), 0 if unusable
    uint32_t gx_iter = 0;    // its CTAs (all resident), 0 when the kernel cannot be used
    Ctl* d_ctl = nullptr;
    Ctl* h_ctl = nullptr;
    uint32_t* d_active = nullptr;
    uint32_t* h_active = nullptr;
    float* d_ig = nullptr;  // nq x 2 x s_max init/goal rows
    float* h_ig = nullptr;
    float* d_path = nullptr;
    float* h_path = nullptr;
    uint32_t s_max = 0, path_total = 0;
    cudaStream_t stream = nullptr, side[2] = {nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<const void*> graph_key;
    int unroll = 8;
    uint32_t plans = 0;
    bool begun = false;
    // single-query extras: debug capture and benchmark timing
    CaptureDev cap{};
    bool capture_on = false;
    void* d_flush = nullptr;
    uint64_t flush_cap = 0;
    std::vector<cudaEvent_t> tev;
    // learned proposal
    uint8_t* d_img = nullptr;        // copy of the packed network image
    char* d_learn = nullptr;         // mixture records and occupancy bits of the learned queries
    uint32_t* d_learned = nullptr;   // indices of the learned queries
    uint32_t n_learned = 0, gx_prop = 1;
    // more than one learned query: one persistent proposal launch over all of their entries,
    // after k_propose_tiles has laid their tiles out (d_prop_off: nl + 1 offsets, an error word)
    uint32_t* d_prop_off = nullptr;
    uint32_t gx_prop_all = 0;

    kpax_status init(const kpax_config* cfgs, uint32_t n)
    {
        if(!cfgs || !n) return set_error("planner: no queries"), KPAX_EINVAL;
        nq = n;
        cfg.assign(cfgs, cfgs + n);
        prm.resize(n);
        env.resize(n);
        hq.assign(n, QueryDev{});
        path_off.resize(n);
        int unroll_cfg = 0;
        for(uint32_t q = 0; q < n; ++q) {
            kpax_status st = derive_params(cfg[q], &prm[q]);
            if(st != KPAX_OK) return st;
            s_max = std::max<uint32_t>(s_max, (uint32_t)prm[q].S);
            unroll_cfg = std::max(unroll_cfg, cfg[q].unroll_iters);
        }
        unroll = unroll_cfg > 0 ? unroll_cfg : 8;
        // two passes: size the pool, then carve it
        for(int pass = 0; pass < 2; ++pass) {
            Carver cv;
            cv.base = pool;
            uint32_t prow = 0;
            for(uint32_t q = 0; q < n; ++q) {
                const KParams& p = prm[q];
                QueryDev& d = hq[q];
                d.p = p;
                const size_t cap_n = p.cap;
                d.t.s[0] = cv.take<float4>(cap_n);
                d.t.s[1] = cv.take<float4>(cap_n);
                d.t.s[2] = p.sd == 12 ? cv.take<float4>(cap_n) : d.t.s[1];
                d.t.ctl = cv.take<float4>(cap_n);
                d.t.dur = cv.take<float>(cap_n);
                d.t.parent = cv.take<int32_t>(cap_n);
                d.t.cost = cv.take<float>(cap_n);
                d.t.r1 = cv.take<int32_t>(cap_n);
                d.t.rep = cv.take<uint8_t>(cap_n);
                d.entries = cv.take<uint32_t>(p.budget);
                d.tiles = cv.take<uint32_t>((cap_n + kTile - 1) / kTile + 1);
                d.lb = cv.take<unsigned long long>((p.budget + kExpandBSMin - 1) / kExpandBSMin + 1);
                d.partials = cv.take<float>(kPartials);
                d.farr = cv.take<uint32_t>(1);
                d.sarr = cv.take<uint32_t>(1);
                d.bar = cv.take<uint32_t>(2);
                d.ctas = cv.take<uint32_t>(kIterMaxCTAs);
                d.path_rows = cfg[q].max_iter + 2;
                path_off[q] = prow;
                prow += d.path_rows;
            }
            // region buffers contiguous, cleared with one memset per plan
            cv.used = (cv.used + kAlign - 1) / kAlign * kAlign;
            region_lo = cv.used;
            for(uint32_t q = 0; q < n; ++q) {
                const KParams& p = prm[q];
                QueryDev& d = hq[q];
                d.rg.counter = cv.take<int32_t>(p.num_r1);
                d.rg.valid = cv.take<int32_t>(p.num_r1);
                d.rg.score = cv.take<float>(p.num_r1);
                d.rg.cur = cv.take<uint32_t>(p.r2_words);
                d.rg.nxt = cv.take<uint32_t>(p.r2_words);
            }
            region_hi = cv.used;
            path_total = prow;
            if(pass == 0) KPAX_CUDA(cudaMalloc(&pool, cv.used));
        }
        KPAX_CUDA(cudaMalloc(&dq, sizeof(QueryDev) * n));
        KPAX_CUDA(cudaMalloc(&d_ctl, sizeof(Ctl) * n));
        KPAX_CUDA(cudaMallocHost(&h_ctl, sizeof(Ctl) * n));
        KPAX_CUDA(cudaMalloc(&d_active, sizeof(uint32_t)));
        KPAX_CUDA(cudaMallocHost(&h_active, sizeof(uint32_t)));
        KPAX_CUDA(cudaMalloc(&d_ig, sizeof(float) * n * 2 * s_max));
        KPAX_CUDA(cudaMallocHost(&h_ig, sizeof(float) * n * 2 * s_max));
        KPAX_CUDA(cudaMalloc(&d_path, sizeof(float) * (size_t)path_total * s_max));
        KPAX_CUDA(cudaMallocHost(&h_path, sizeof(float) * (size_t)path_total * s_max));
        for(uint32_t q = 0; q < n; ++q) {
            hq[q].ctl = d_ctl + q;
            hq[q].init_goal = d_ig + (size_t)q * 2 * s_max;
            hq[q].path = d_path + (size_t)path_off[q] * s_max;
        }
        KPAX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        for(int k = 0; k < 2; ++k) {
            KPAX_CUDA(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
            KPAX_CUDA(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
        }
        KPAX_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        KPAX_CUDA(cudaEventCreate(&ev0));
        KPAX_CUDA(cudaEventCreate(&ev1));
        uint32_t max_tiles = 1;
        for(uint32_t q = 0; q < n; ++q) {
            const int m = prm[q].model - 1;
            if(groups[m].empty()) expand_bs[m] = cfg[q].block_size > 0 ? cfg[q].block_size : kExpandBS;
            groups[m].push_back(q);
            const uint32_t bs = (uint32_t)expand_bs[m], spt = cfg[q].samples_per_thread > 0 ? cfg[q].samples_per_thread : 1;
            const uint32_t tiles = (prm[q].budget + bs - 1) / bs;
            expand_gx[m] = std::max<uint32_t>(expand_gx[m], (tiles + spt - 1) / spt);
            max_tiles = std::max<uint32_t>(max_tiles, (prm[q].cap + kTile - 1) / kTile);
        }
        for(int m = 0; m < 3; ++m) {
            if(groups[m].empty()) continue;
            KPAX_CUDA(cudaMalloc(&d_groups[m], sizeof(uint32_t) * groups[m].size()));
            KPAX_CUDA(cudaMemcpyAsync(d_groups[m], groups[m].data(), sizeof(uint32_t) * groups[m].size(),
                                      cudaMemcpyHostToDevice, stream));
        }
        gx_front = n == 1 ? std::min<uint32_t>(max_tiles, kFrontierCTAs)
                          : std::max<uint32_t>(1, std::min<uint32_t>(max_tiles, 8 * 148 * 2 / n));
        // a single query: enough CTAs for its 32-region groups (eight warps each), at most kScoreCTAs
        const uint32_t groups0 = ((uint32_t)prm[0].num_r1 + 31) / 32;
        gx_score = n == 1 ? std::min<uint32_t>(kScoreCTAs, std::max<uint32_t>(1, (groups0 + 7) / 8))
                          : std::max<uint32_t>(1, 1024 / n);
        if(n == 1) {  // the fused iteration: as many CTAs as the expansion wants and can stay resident
            int dev = 0, sms = 148, per_sm = 0;
            KPAX_CUDA(cudaGetDevice(&dev));
            KPAX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            const int m = prm[0].model - 1, bs = expand_bs[m];
            void* fn = m == 0 ? iterate_kernel<KPAX_MODEL_DOUBLE_INTEGRATOR>(bs)
                              : m == 1 ? iterate_kernel<KPAX_MODEL_DUBINS_AIRPLANE>(bs) : iterate_kernel<KPAX_MODEL_QUADROTOR>(bs);
            KPAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bs, 0));
            const uint32_t resident = (uint32_t)std::max(per_sm, 0) * (uint32_t)sms;
            // every resident CTA: the frontier and score phases use them all, the expansion as many as
            // it has tiles (a small budget's iteration leaves the rest idle in that phase)
            gx_iter = std::min<uint32_t>(resident, (uint32_t)kIterMaxCTAs);
            if(m == 2) {  // the two parts around the proposal pass: the smaller occupancy of the two
                int front = 0, back = 0;
                KPAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &front, iterate_kernel<KPAX_MODEL_QUADROTOR, kIterFront>(bs), bs, 0));
                KPAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &back, iterate_kernel<KPAX_MODEL_QUADROTOR, kIterBack>(bs), bs, 0));
                gx_split = std::min<uint32_t>((uint32_t)std::max(std::min(front, back), 0) * (uint32_t)sms,
                                              (uint32_t)kIterMaxCTAs);
            }
        }
        if(n > 1 && n <= kBatchMaxQueries) {  // persistent stages: grids of resident CTAs
            int dev = 0, sms = 148;
            KPAX_CUDA(cudaGetDevice(&dev));
            KPAX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            auto resident = [&](const void* fn, int bs, size_t smem, uint32_t& gx) -> kpax_status {
                int per_sm = 0;
                KPAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, bs, smem));
                gx = (uint32_t)std::max(per_sm, 0) * (uint32_t)sms;
                return KPAX_OK;
            };
            const size_t sq = 4 * ((size_t)n + 1);
            kpax_status st = resident((const void*)k_count_all, kFrontierBS, sq, gx_count_all);
            if(st == KPAX_OK) st = resident((const void*)k_write_all, kFrontierBS, sq, gx_write_all);
            if(st == KPAX_OK) st = resident((const void*)k_scores_all, kScoreBS, sq, gx_scores_all);
            for(int m = 0; m < 3 && st == KPAX_OK; ++m) {
                if(groups[m].empty()) continue;
                const size_t sg = 4 * (groups[m].size() + 1);
                const void* fn = m == 0 ? expand_all_kernel<KPAX_MODEL_DOUBLE_INTEGRATOR>(expand_bs[m])
                                        : m == 1 ? expand_all_kernel<KPAX_MODEL_DUBINS_AIRPLANE>(expand_bs[m])
                                                 : expand_all_kernel<KPAX_MODEL_QUADROTOR>(expand_bs[m]);
                st = resident(fn, expand_bs[m], sg, gx_expand_all[m]);
            }
            if(st != KPAX_OK) return st;
            persistent = gx_count_all && gx_write_all && gx_scores_all && (groups[0].empty() || gx_expand_all[0]) &&
                         (groups[1].empty() || gx_expand_all[1]) && (groups[2].empty() || gx_expand_all[2]);
            int bs0 = 0, ngroups = 0;
            bool same_bs = true;
            for(int m = 0; m < 3; ++m) {
                if(groups[m].empty()) continue;
                ++ngroups;
                if(!bs0) bs0 = expand_bs[m];
                same_bs = same_bs && expand_bs[m] == bs0;
            }
            if(const char* e = getenv("KPAX_BATCH_EXPAND")) expand_mode = atoi(e) == 0 ? 0 : atoi(e) == 2 ? 2 : 1;
            if(persistent && ngroups > 1 && same_bs) {
                std::vector<uint32_t> order;
                for(int m = 2; m >= 0; --m) order.insert(order.end(), groups[m].begin(), groups[m].end());
                KPAX_CUDA(cudaMalloc(&d_mixed, sizeof(uint32_t) * order.size()));
                KPAX_CUDA(cudaMemcpyAsync(d_mixed, order.data(), sizeof(uint32_t) * order.size(), cudaMemcpyHostToDevice,
                                          stream));
                uint32_t gx = 0;
                if((st = resident(expand_mixed_kernel(bs0), bs0, 4 * ((size_t)n + 1), gx)) != KPAX_OK) return st;
                if(gx) mixed_bs = bs0, gx_mixed = gx;
            }
        }
        update_fused();
        // control blocks, counters and arrival flags start at zero; no node is in a frontier
        KPAX_CUDA(cudaMemsetAsync(pool, 0, region_lo, stream));
        KPAX_CUDA(cudaMemsetAsync(d_ctl, 0, sizeof(Ctl) * n, stream));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        return KPAX_OK;
    }

    void update_fused()
    {
        fused = nq == 1 && gx_iter > 0 && cfg[0].iteration_kernels == 0 && n_learned == 0;
        fused_split = nq == 1 && gx_split > 0 && cfg[0].iteration_kernels == 0 && n_learned == 1;
    }

    void release()
    {
        if(stream) cudaStreamSynchronize(stream);
        if(graph) cudaGraphExecDestroy(graph);
        for(Env& e : env) e.release();
        for(int m = 0; m < 3; ++m)
            if(d_groups[m]) cudaFree(d_groups[m]);
        void* dev[] = {pool, dq, d_ctl, d_active, d_ig, d_path, d_flush, d_img, d_learn, d_learned, d_mixed, d_prop_off};
        for(void* p : dev)
            if(p) cudaFree(p);
        void* host[] = {h_ctl, h_active, h_ig, h_path};
        for(void* p : host)
            if(p) cudaFreeHost(p);
        release_capture();
        for(cudaEvent_t e : tev) cudaEventDestroy(e);
        cudaEvent_t evs[] = {ev_fork, ev_join[0], ev_join[1], ev0, ev1};
        for(cudaEvent_t e : evs)
            if(e) cudaEventDestroy(e);
        for(int k = 0; k < 2; ++k)
            if(side[k]) cudaStreamDestroy(side[k]);
        if(stream) cudaStreamDestroy(stream);
        graph = nullptr, stream = nullptr, pool = nullptr;
    }

    void release_capture()
    {
        void* bufs[6] = {cap.rows, cap.valid, cap.r1, cap.r2, cap.next, cap.parent};
        for(void* b : bufs)
            if(b) cudaFree(b);
        cap = CaptureDev{};
        if(!hq.empty()) hq[0].cap = cap;
    }

    kpax_status set_capture(bool on)
    {
        if(nq != 1) return set_error("debug capture needs a single query"), KPAX_EINVAL;
        if(on == capture_on) return KPAX_OK;
        if(graph) cudaGraphExecDestroy(graph), graph = nullptr;
        release_capture();
        capture_on = on;
        if(on) {
            const size_t n = prm[0].budget, S = prm[0].S;
            KPAX_CUDA(cudaMalloc(&cap.rows, sizeof(float) * n * S));
            KPAX_CUDA(cudaMalloc(&cap.valid, n));
            KPAX_CUDA(cudaMalloc(&cap.r1, sizeof(int32_t) * n));
            KPAX_CUDA(cudaMalloc(&cap.r2, sizeof(int32_t) * n));
            KPAX_CUDA(cudaMalloc(&cap.next, n));
            KPAX_CUDA(cudaMalloc(&cap.parent, sizeof(int32_t) * n));
        }
        hq[0].cap = cap;
        return upload_descriptors();
    }

    kpax_status upload_descriptors()
    {
        KPAX_CUDA(cudaMemcpyAsync(dq, hq.data(), sizeof(QueryDev) * nq, cudaMemcpyHostToDevice, stream));
        return KPAX_OK;
    }

    // ev (optional): four events recorded before the frontier, expansion and score kernels and after;
    // with split == false only the first and the last, so the launches still overlap.
    void launch_iteration(cudaEvent_t* ev = nullptr, bool split = true)
    {
        if(ev) cudaEventRecord(ev[0], stream);
        if(fused_split) {  // front launch, proposal pass, back launch; phase times from the device clock
            launch_iterate<KPAX_MODEL_QUADROTOR, kIterFront>(expand_bs[2], gx_split, stream, dq, d_ctl, d_active);
            launch_proposal(stream);
            launch_iterate<KPAX_MODEL_QUADROTOR, kIterBack>(expand_bs[2], gx_split, stream, dq, d_ctl, d_active);
            if(ev) cudaEventRecord(ev[3], stream);
            return;
        }
        if(fused) {  // one launch: its phase times come from the device clock (Ctl::t_*_ns)
            const int m = prm[0].model - 1;
            const Ctl* c0 = d_ctl;  // the single query's control block
            if(m == 0) launch_iterate<KPAX_MODEL_DOUBLE_INTEGRATOR>(expand_bs[m], gx_iter, stream, dq, c0, d_active);
            else if(m == 1) launch_iterate<KPAX_MODEL_DUBINS_AIRPLANE>(expand_bs[m], gx_iter, stream, dq, c0, d_active);
            else launch_iterate<KPAX_MODEL_QUADROTOR>(expand_bs[m], gx_iter, stream, dq, c0, d_active);
            if(ev) cudaEventRecord(ev[3], stream);
            return;
        }
        if(persistent) {  // one launch per stage over all queries; model groups one after another
            const size_t sq = 4 * ((size_t)nq + 1);
            launch_chained(k_batch_start, dim3((nq + kBatchStartBS - 1) / kBatchStartBS), kBatchStartBS, 0, stream, d_ctl, nq,
                           d_active);
            launch_chained(k_count_all, dim3(gx_count_all), kFrontierBS, sq, stream, dq, (const Ctl*)d_ctl, nq);
            launch_chained(k_write_all, dim3(gx_write_all), kFrontierBS, sq, stream, dq, (const Ctl*)d_ctl, nq);
            if(ev && split) cudaEventRecord(ev[1], stream);
            if(n_learned) launch_proposal(stream);
            if(expand_mode == 0) {  // per model group: one block per child tile of every query, groups concurrent
                int used[3], nused = 0;
                for(int m = 0; m < 3; ++m)
                    if(!groups[m].empty()) used[nused++] = m;
                if(nused > 1) cudaEventRecord(ev_fork, stream);
                for(int u = 0; u < nused; ++u) {
                    const int m = used[u];
                    cudaStream_t s = stream;
                    if(u < nused - 1) {
                        s = side[u];
                        cudaStreamWaitEvent(s, ev_fork, 0);
                    }
                    const dim3 grid(expand_gx[m], (uint32_t)groups[m].size());
                    if(m == 0) launch_expand<KPAX_MODEL_DOUBLE_INTEGRATOR>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
                    else if(m == 1) launch_expand<KPAX_MODEL_DUBINS_AIRPLANE>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
                    else launch_expand<KPAX_MODEL_QUADROTOR>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
                    if(u < nused - 1) cudaEventRecord(ev_join[u], s);
                }
                for(int u = 0; u + 1 < nused; ++u) cudaStreamWaitEvent(stream, ev_join[u], 0);
            } else if(expand_mode == 2 && mixed_bs) {
                launch_expand_mixed(mixed_bs, gx_mixed, sq, stream, dq, d_ctl, d_mixed, nq, d_active);
            } else {
                for(int m = 0; m < 3; ++m) {
                    if(groups[m].empty()) continue;
                    const uint32_t g = (uint32_t)groups[m].size();
                    const size_t sg = 4 * ((size_t)g + 1);
                    if(m == 0)
                        launch_expand_all<KPAX_MODEL_DOUBLE_INTEGRATOR>(expand_bs[m], gx_expand_all[m], sg, stream, dq, d_ctl,
                                                                        d_groups[m], g, d_active);
                    else if(m == 1)
                        launch_expand_all<KPAX_MODEL_DUBINS_AIRPLANE>(expand_bs[m], gx_expand_all[m], sg, stream, dq, d_ctl,
                                                                      d_groups[m], g, d_active);
                    else
                        launch_expand_all<KPAX_MODEL_QUADROTOR>(expand_bs[m], gx_expand_all[m], sg, stream, dq, d_ctl,
                                                                d_groups[m], g, d_active);
                }
            }
            if(ev && split) cudaEventRecord(ev[2], stream);
            launch_chained(k_scores_all, dim3(gx_scores_all), kScoreBS, sq, stream, dq, (const Ctl*)d_ctl, nq, d_active);
            if(ev) cudaEventRecord(ev[3], stream);
            return;
        }
        launch_chained(k_frontier_count, dim3(gx_front, nq), kFrontierBS, 0, stream, dq, d_active);
        launch_chained(k_frontier_write, dim3(gx_front, nq), kFrontierBS, 0, stream, dq);
        if(ev && split) cudaEventRecord(ev[1], stream);
        int used[3], nused = 0;
        for(int m = 0; m < 3; ++m)
            if(!groups[m].empty()) used[nused++] = m;
        if(nused > 1) cudaEventRecord(ev_fork, stream);
        for(int u = 0; u < nused; ++u) {
            const int m = used[u];
            cudaStream_t s = stream;
            if(u < nused - 1) {  // model groups run as parallel branches
                s = side[u];
                cudaStreamWaitEvent(s, ev_fork, 0);
            }
            const dim3 grid(expand_gx[m], (uint32_t)groups[m].size());
            if(m == 2 && n_learned) launch_proposal(s);
            if(m == 0) launch_expand<KPAX_MODEL_DOUBLE_INTEGRATOR>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
            else if(m == 1) launch_expand<KPAX_MODEL_DUBINS_AIRPLANE>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
            else launch_expand<KPAX_MODEL_QUADROTOR>(expand_bs[m], grid, s, dq, d_groups[m], d_active);
            if(u < nused - 1) cudaEventRecord(ev_join[u], s);
        }
        for(int u = 0; u + 1 < nused; ++u) cudaStreamWaitEvent(stream, ev_join[u], 0);
        if(ev && split) cudaEventRecord(ev[2], stream);
        launch_chained(k_scores, dim3(gx_score, nq), kScoreBS, 0, stream, dq, d_active);
        if(ev) cudaEventRecord(ev[3], stream);
    }

    // The learned proposal pass: one grid row per learned query, or (more than one) one launch
    // whose CTAs share all their entry tiles.
    void launch_proposal(cudaStream_t s)
    {
        if(d_prop_off) {
            launch_chained(k_propose_tiles, dim3(1), kPropTilesBS, 0, s, dq, d_learned, n_learned, d_prop_off);
            launch_chained(k_propose_all, dim3(gx_prop_all), mlp::tc::kThreads, mlp::tc::kSmemBytes, s, dq, d_learned, n_learned,
                           d_prop_off, d_prop_off + n_learned + 1);
        } else {
            launch_chained(k_propose, dim3(gx_prop, n_learned), mlp::tc::kThreads, mlp::tc::kSmemBytes, s, dq, d_learned);
        }
    }

    // Learned proposal for the quadrotor queries with enable[q] != 0 (all when enable is null);
    // net == nullptr turns it off.
    kpax_status set_proposal(const kpax_mlp* net, float eps, const uint8_t* enable)
    {
        if(net && !mlp_image(net)) return set_error("set_proposal: network not packed"), KPAX_EINVAL;
        if(!(eps >= 0.0f && eps <= 1.0f)) return set_error("set_proposal: epsilon %g not in [0,1]", (double)eps), KPAX_EINVAL;
        std::vector<uint32_t> sel;
        for(uint32_t q = 0; net && q < nq; ++q) {
            const bool want = enable ? enable[q] != 0 : prm[q].model == KPAX_MODEL_QUADROTOR;
            if(!want) continue;
            if(prm[q].model != KPAX_MODEL_QUADROTOR)
                return set_error("set_proposal: query %u is not a quadrotor query", q), KPAX_EINVAL;
            sel.push_back(q);
        }
        KPAX_CUDA(cudaStreamSynchronize(stream));
        if(graph) cudaGraphExecDestroy(graph), graph = nullptr;
        graph_key.clear();
        for(void* p : {(void*)d_img, (void*)d_learn, (void*)d_learned, (void*)d_prop_off})
            if(p) cudaFree(p);
        d_img = nullptr, d_learn = nullptr, d_learned = nullptr, d_prop_off = nullptr;
        n_learned = 0, gx_prop_all = 0;
        for(QueryDev& d : hq) d.mlp_img = nullptr, d.mix = nullptr, d.occ = nullptr, d.prop_eps = 1.0f;
        if(!sel.empty()) {
            KPAX_CUDA(cudaMalloc(&d_img, mlp::kImgBytes));
            KPAX_CUDA(cudaMemcpyAsync(d_img, mlp_image(net), mlp::kImgBytes, cudaMemcpyDeviceToDevice, stream));
            size_t bytes = 0;
            for(uint32_t q : sel) {
                const uint32_t words = (uint32_t)((prm[q].W1 * prm[q].W1 * prm[q].W1 + 31) / 32);
                bytes += ((size_t)prm[q].budget * mlp::kMixFloats * 4 + (size_t)words * 4 + kAlign - 1) / kAlign * kAlign;
            }
            KPAX_CUDA(cudaMalloc(&d_learn, bytes));
            size_t off = 0;
            uint32_t max_tiles = 1;
            for(uint32_t q : sel) {
                QueryDev& d = hq[q];
                const uint32_t words = (uint32_t)((prm[q].W1 * prm[q].W1 * prm[q].W1 + 31) / 32);
                d.mix = reinterpret_cast<float*>(d_learn + off);
                d.occ = reinterpret_cast<uint32_t*>(d_learn + off + (size_t)prm[q].budget * mlp::kMixFloats * 4);
                d.mlp_img = d_img;
                d.prop_eps = eps;
                off += ((size_t)prm[q].budget * mlp::kMixFloats * 4 + (size_t)words * 4 + kAlign - 1) / kAlign * kAlign;
                max_tiles = std::max<uint32_t>(max_tiles, (prm[q].budget + mlp::tc::kRows - 1) / mlp::tc::kRows);
            }
            KPAX_CUDA(cudaMalloc(&d_learned, sizeof(uint32_t) * sel.size()));
            KPAX_CUDA(cudaMemcpyAsync(d_learned, sel.data(), sizeof(uint32_t) * sel.size(), cudaMemcpyHostToDevice, stream));
            n_learned = (uint32_t)sel.size();
            int dev = 0, sms = 148;
            KPAX_CUDA(cudaGetDevice(&dev));
            KPAX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            gx_prop = std::max<uint32_t>(1, std::min<uint32_t>(max_tiles, (2u * (uint32_t)sms + n_learned - 1) / n_learned));
            KPAX_CUDA(cudaFuncSetAttribute(k_propose, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::tc::kSmemBytes));
            if(n_learned > 1 && n_learned <= kBatchMaxQueries) {
                KPAX_CUDA(cudaFuncSetAttribute(k_propose_all, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp::tc::kSmemBytes));
                int per_sm = 0;
                KPAX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_propose_all, mlp::tc::kThreads, mlp::tc::kSmemBytes));
                KPAX_CUDA(cudaMalloc(&d_prop_off, sizeof(uint32_t) * (n_learned + 2)));
                KPAX_CUDA(cudaMemsetAsync(d_prop_off, 0, sizeof(uint32_t) * (n_learned + 2), stream));
                gx_prop_all = (uint32_t)std::max(1, per_sm) * (uint32_t)sms;
            }
            if(begun)  // a plan in progress: occupancy of the current environments
                for(uint32_t q : sel) {
                    kpax_status st = launch_occupancy(prm[q], env[q].view(), const_cast<uint32_t*>(hq[q].occ), stream);
                    if(st != KPAX_OK) return st;
                }
        }
        update_fused();
        kpax_status st = upload_descriptors();
        if(st != KPAX_OK) return st;
        KPAX_CUDA(cudaStreamSynchronize(stream));
        return begun ? ensure_graph() : KPAX_OK;
    }

    uint64_t kernels_per_iteration() const
    {
        if(fused) return 1;
        if(fused_split) return 3;
        if(persistent) {  // start, count, write, (proposal), the expansion(s), scores
            uint64_t k = n_learned ? (d_prop_off ? 6 : 5) : 4;
            if(expand_mode == 2 && mixed_bs) return k + 1;
            for(int m = 0; m < 3; ++m) k += groups[m].empty() ? 0 : 1;
            return k;
        }
        uint64_t k = n_learned ? (d_prop_off ? 5 : 4) : 3;  // two frontier passes, the score pass, the proposal pass(es)
        for(int m = 0; m < 3; ++m) k += groups[m].empty() ? 0 : 1;
        return k;
    }

    kpax_status ensure_graph()
    {
        std::vector<const void*> key;
        for(uint32_t q = 0; q < nq; ++q) key.push_back(env[q].d_ent), key.push_back(env[q].d_obs);
        key.push_back(cap.rows);
        if(graph && key == graph_key) return KPAX_OK;
        if(graph) cudaGraphExecDestroy(graph), graph = nullptr;
        cudaGraph_t g = nullptr;
        KPAX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for(int i = 0; i < unroll; ++i) launch_iteration();
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if(e != cudaSuccess) return set_error("graph capture failed: %s", cudaGetErrorString(e)), KPAX_ECUDA;
        e = cudaGraphInstantiate(&graph, g, 0);
        cudaGraphDestroy(g);
        if(e != cudaSuccess) return set_error("graph instantiate failed: %s", cudaGetErrorString(e)), KPAX_ECUDA;
        graph_key = key;
        return KPAX_OK;
    }

    // h_init / h_goal: nq rows with `stride` floats between queries.
    kpax_status begin(const float* h_init, const float* h_goal, uint32_t stride, const float* const* d_obstacles,
                      const uint32_t* n_obs, uint32_t max_iters, uint32_t stop, bool record_start = true)
    {
        if(!h_init || !h_goal) return set_error("plan: null start or goal"), KPAX_EINVAL;
        if(record_start) KPAX_CUDA(cudaEventRecord(ev0, stream));
        for(uint32_t q = 0; q < nq; ++q) {
            if(n_obs[q] && !d_obstacles[q]) return set_error("plan: null obstacle buffer for query %u", q), KPAX_EINVAL;
            kpax_status st = env[q].build(prm[q], d_obstacles[q], n_obs[q], stream);
            if(st != KPAX_OK) return st;
            hq[q].g = env[q].view();
            if(hq[q].occ) {
                st = launch_occupancy(prm[q], hq[q].g, const_cast<uint32_t*>(hq[q].occ), stream);
                if(st != KPAX_OK) return st;
            }
            const uint32_t S = (uint32_t)prm[q].S;
            memcpy(h_ig + (size_t)q * 2 * s_max, h_init + (size_t)q * stride, sizeof(float) * S);
            memcpy(h_ig + (size_t)q * 2 * s_max + S, h_goal + (size_t)q * stride, sizeof(float) * S);
        }
        kpax_status st = upload_descriptors();
        if(st != KPAX_OK) return st;
        KPAX_CUDA(cudaMemcpyAsync(d_ig, h_ig, sizeof(float) * nq * 2 * s_max, cudaMemcpyHostToDevice, stream));
        KPAX_CUDA(cudaMemsetAsync(pool + region_lo, 0, region_hi - region_lo, stream));
        *h_active = nq;
        KPAX_CUDA(cudaMemcpyAsync(d_active, h_active, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        k_begin<<<dim3(1, nq), 128, 0, stream>>>(dq, plans, max_iters, stop);
        KPAX_CHECK_LAUNCH();
        count_launch();
        plans += 1;  // every query of a plan call draws the random stream of this plan index
        begun = true;
        return ensure_graph();
    }

    // Runs graphs until no query is active; `guard` bounds the number of graph launches.  With
    // poll = false all launches are queued first and the stream is synchronised once.
    kpax_status run(uint32_t guard, bool poll = true)
    {
        NvtxRange range("kpax plan iterations");
        for(uint32_t g = 0; g < guard; ++g) {
            KPAX_CUDA(cudaGraphLaunch(graph, stream));
            count_launch(kernels_per_iteration() * (uint64_t)unroll);
            if(!poll) continue;
            KPAX_CUDA(cudaMemcpyAsync(h_active, d_active, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
            KPAX_CUDA(cudaStreamSynchronize(stream));
            if(*h_active == 0u) break;
        }
        return sync_ctl();
    }

    kpax_status sync_ctl()
    {
        KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl) * nq, cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaStreamSynchronize(stream));
        for(uint32_t q = 0; q < nq; ++q) {
            if(h_ctl[q].error & kErrTimeout) return set_error("query %u: a device-side wait gave up", q), KPAX_ETIMEOUT;
            if(h_ctl[q].error & kErrCapacity) return set_error("query %u: tree capacity exceeded", q), KPAX_ECAPACITY;
            if(h_ctl[q].error & kErrProposal)
                return set_error("query %u: a wait of the proposal pass expired", q), KPAX_ETIMEOUT;
        }
        return KPAX_OK;
    }

    kpax_status write_ctl()
    {
        KPAX_CUDA(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(Ctl) * nq, cudaMemcpyHostToDevice, stream));
        return KPAX_OK;
    }

    kpax_status finish(kpax_result* out, double* batch_ms = nullptr)
    {
        k_path<<<dim3(1, nq), 32, 0, stream>>>(dq);
        KPAX_CHECK_LAUNCH();
        count_launch();
        KPAX_CUDA(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(Ctl) * nq, cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaMemcpyAsync(h_path, d_path, sizeof(float) * (size_t)path_total * s_max, cudaMemcpyDeviceToHost, stream));
        KPAX_CUDA(cudaEventRecord(ev1, stream));
        KPAX_CUDA(cudaEventSynchronize(ev1));
        float ms = 0.0f;
        KPAX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        if(batch_ms) *batch_ms = ms;
        for(uint32_t q = 0; out && q < nq; ++q) {
            const Ctl& c = h_ctl[q];
            kpax_result r{};
            r.found = c.goal_idx != kNone;
            r.goal_idx = r.found ? c.goal_idx : 0u;
            r.path_len = c.path_len;
            r.tree_size = c.tree;
            r.iters = c.iters_done;
            r.tree_full = (int32_t)c.full;
            r.h_path = h_path + (size_t)path_off[q] * s_max;
            r.ms = nq == 1 ? ms : (c.t_done_ns > c.t_begin_ns ? (double)(c.t_done_ns - c.t_begin_ns) * 1e-6 : 0.0);
            r.expansions = c.n_exp;
            r.valid_expansions = c.n_valid;
            r.path_cost = c.path_cost;
            out[q] = r;
        }
        return KPAX_OK;
    }

    // Resume every query for n more iterations.
    kpax_status resume(uint32_t n, uint32_t stop_at_goal)
    {
        kpax_status st = sync_ctl();
        if(st != KPAX_OK) return st;
        uint32_t act = 0;
        for(uint32_t q = 0; q < nq; ++q) {
            Ctl& c = h_ctl[q];
            c.max_iters = c.iters_done + n;
            c.stop_at_goal = stop_at_goal;
            c.stop_req = 0;  // a stop the batch stages requested is decided again
            c.done = (c.full || c.error || (stop_at_goal && c.goal_idx != kNone)) ? 1u : 0u;
            act += c.done ? 0u : 1u;
        }
        *h_active = act;
        KPAX_CUDA(cudaMemcpyAsync(d_active, h_active, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
        return write_ctl();
    }

    kpax_status iterate(uint32_t n, uint32_t stop_at_goal)
    {
        kpax_status st = resume(n, stop_at_goal);
        if(st != KPAX_OK) return st;
        if(*h_active == 0u) return sync_ctl();
        if(!stop_at_goal) return run((n + (uint32_t)unroll - 1u) / (uint32_t)unroll, false);
        return run(n / (uint32_t)unroll + 4u);
    }

    // Benchmark iterations: each optionally preceded (outside its events) by a write of
    // flush_bytes, which evicts the 126 MB L2, then the iteration's kernels bracketed by events.
    kpax_status iterate_timed(uint32_t n, uint64_t flush, bool split, kpax_iter_timing* times, uint64_t* totals)
    {
        kpax_status st = sync_ctl();
        if(st != KPAX_OK) return st;
        std::vector<Ctl> c0(h_ctl, h_ctl + nq);
        if((st = resume(n, 0u)) != KPAX_OK) return st;
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
            launch_iteration(&tev[4 * (size_t)i], split);
            KPAX_CHECK_LAUNCH();
            count_launch(kernels_per_iteration());
        }
        KPAX_CUDA(cudaStreamSynchronize(stream));
        Ctl c1 = {};
        if(fused || fused_split) {
            KPAX_CUDA(cudaMemcpyAsync(&c1, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
            KPAX_CUDA(cudaStreamSynchronize(stream));
        }
        for(uint32_t i = 0; i < n; ++i) {
            float a = 0, b = 0, d = 0, t = 0;
            cudaEvent_t* e = &tev[4 * (size_t)i];
            if((fused || fused_split) && split) {  // phase times from the device clock, averaged over the n iterations
                a = (float)((c1.t_front_ns - c0[0].t_front_ns) * 1e-6 / n);
                b = (float)((c1.t_expand_ns - c0[0].t_expand_ns) * 1e-6 / n);
                d = (float)((c1.t_score_ns - c0[0].t_score_ns) * 1e-6 / n);
            } else if(split) {
                KPAX_CUDA(cudaEventElapsedTime(&a, e[0], e[1]));
                KPAX_CUDA(cudaEventElapsedTime(&b, e[1], e[2]));
                KPAX_CUDA(cudaEventElapsedTime(&d, e[2], e[3]));
            }
            KPAX_CUDA(cudaEventElapsedTime(&t, e[0], e[3]));
            if(times) times[i] = kpax_iter_timing{t, a, b, d};
        }
        st = sync_ctl();
        if(totals) {
            totals[0] = totals[1] = totals[2] = totals[3] = 0;
            for(uint32_t q = 0; q < nq; ++q) {
                totals[0] += h_ctl[q].n_exp - c0[q].n_exp;
                totals[1] += h_ctl[q].n_valid - c0[q].n_valid;
                totals[2] += h_ctl[q].n_steps - c0[q].n_steps;
                totals[3] += (uint64_t)(h_ctl[q].tree - c0[q].tree);
            }
        }
        return st;
    }
};

uint32_t plan_guard(const PlanBatch& b, uint32_t iters) { return iters / (uint32_t)b.unroll + 4u; }

}  // namespace

struct kpax_planner {
    PlanBatch b;
    float* d_obs_host = nullptr;
    uint32_t obs_host_cap = 0;
};

struct kpax_batch {
    PlanBatch b;
};

extern "C" {

kpax_status kpax_create(const kpax_config* cfg, kpax_planner** out)
{
    if(!cfg || !out) return set_error("kpax_create: null argument"), KPAX_EINVAL;
    *out = nullptr;
    kpax_planner* pl = new(std::nothrow) kpax_planner();
    if(!pl) return set_error("kpax_create: host allocation failed"), KPAX_ENOMEM;
    kpax_status st = no_throw("kpax_create", [&] { return pl->b.init(cfg, 1); });
    if(st != KPAX_OK) {
        pl->b.release();
        delete pl;
        return st;
    }
    *out = pl;
    return KPAX_OK;
}

kpax_status kpax_destroy(kpax_planner* pl)
{
    if(!pl) return KPAX_OK;
    pl->b.release();
    if(pl->d_obs_host) cudaFree(pl->d_obs_host);
    delete pl;
    return KPAX_OK;
}

void* kpax_planner_stream(kpax_planner* pl) { return pl ? (void*)pl->b.stream : nullptr; }

kpax_status kpax_plan(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs,
                      int32_t save_tree, kpax_result* out)
{
    return no_throw("kpax_plan", [&]() -> kpax_status {
        (void)save_tree;  // the tree always stays on the device; kpax_export_tree copies it out
        if(!pl) return set_error("kpax_plan: null planner"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        kpax_status st = b.begin(h_init, h_goal, 0, &d_obstacles, &n_obs, b.cfg[0].max_iter, 1u);
        if(st != KPAX_OK) return st;
        st = b.run(plan_guard(b, b.cfg[0].max_iter));
        kpax_status st2 = b.finish(out);
        return st != KPAX_OK ? st : st2;
    });
}

kpax_status kpax_plan_host(kpax_planner* pl, const float* h_init, const float* h_goal, const float* h_obstacles, uint32_t n_obs,
                           kpax_result* out)
{
    return no_throw("kpax_plan_host", [&]() -> kpax_status {
        if(!pl || (n_obs && !h_obstacles)) return set_error("kpax_plan_host: null argument"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        if(n_obs > pl->obs_host_cap) {
            if(pl->d_obs_host) cudaFree(pl->d_obs_host), pl->d_obs_host = nullptr;
            KPAX_CUDA(cudaMalloc(&pl->d_obs_host, sizeof(float) * 6 * n_obs));
            pl->obs_host_cap = n_obs;
        }
        KPAX_CUDA(cudaEventRecord(b.ev0, b.stream));
        if(n_obs)
            KPAX_CUDA(cudaMemcpyAsync(pl->d_obs_host, h_obstacles, sizeof(float) * 6 * n_obs, cudaMemcpyHostToDevice, b.stream));
        const float* d = pl->d_obs_host;
        kpax_status st = b.begin(h_init, h_goal, 0, &d, &n_obs, b.cfg[0].max_iter, 1u, false);
        if(st != KPAX_OK) return st;
        st = b.run(plan_guard(b, b.cfg[0].max_iter));
        kpax_status st2 = b.finish(out);
        return st != KPAX_OK ? st : st2;
    });
}

kpax_status kpax_plan_begin(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs)
{
    return no_throw("kpax_plan_begin", [&]() -> kpax_status {
        if(!pl) return set_error("kpax_plan_begin: null planner"), KPAX_EINVAL;
        kpax_status st = pl->b.begin(h_init, h_goal, 0, &d_obstacles, &n_obs, 0u, 0u);
        if(st != KPAX_OK) return st;
        return pl->b.sync_ctl();
    });
}

kpax_status kpax_plan_iterate(kpax_planner* pl, uint32_t n_iters, int32_t stop_at_goal)
{
    return no_throw("kpax_plan_iterate", [&]() -> kpax_status {
        if(!pl || !pl->b.begun) return set_error("kpax_plan_iterate: call kpax_plan_begin first"), KPAX_EINVAL;
        if(!n_iters) return KPAX_OK;
        return pl->b.iterate(n_iters, stop_at_goal ? 1u : 0u);
    });
}

kpax_status kpax_plan_iterate_timed(kpax_planner* pl, uint32_t n_iters, uint64_t flush_bytes, int32_t split,
                                    kpax_iter_timing* h_times, uint64_t* h_totals)
{
    return no_throw("kpax_plan_iterate_timed", [&]() -> kpax_status {
        if(!pl || !pl->b.begun) return set_error("kpax_plan_iterate_timed: call kpax_plan_begin first"), KPAX_EINVAL;
        return pl->b.iterate_timed(n_iters, flush_bytes, split != 0, h_times, h_totals);
    });
}

kpax_status kpax_write_rows_csv(const float* h_rows, uint32_t rows, uint32_t cols, const char* filename, int32_t append)
{
    if((!h_rows && rows) || !cols || !filename) return set_error("kpax_write_rows_csv: bad arguments"), KPAX_EINVAL;
    FILE* f = fopen(filename, append ? "a" : "w");
    if(!f) return set_error("kpax_write_rows_csv: cannot open %s", filename), KPAX_EINVAL;
    char buf[64];
    for(uint32_t i = 0; i < rows; ++i) {
        for(uint32_t j = 0; j < cols; ++j) {  // std::fixed with 6 digits, as writeVectorToCSV (helper.cuh:56-80)
            snprintf(buf, sizeof(buf), "%.6f", (double)h_rows[(size_t)i * cols + j]);
            fputs(buf, f);
            if(j + 1 < cols) fputc(',', f);
        }
        fputc('\n', f);
    }
    const bool ok = fflush(f) == 0;
    fclose(f);
    if(!ok) return set_error("kpax_write_rows_csv: write to %s failed", filename), KPAX_EINVAL;
    return KPAX_OK;
}

kpax_status kpax_write_solution_csv(kpax_planner* pl, const char* filename, int32_t append)
{
    return no_throw("kpax_write_solution_csv", [&]() -> kpax_status {
        if(!pl || !pl->b.begun) return set_error("kpax_write_solution_csv: no plan"), KPAX_EINVAL;
        kpax_result r{};
        kpax_status st = pl->b.finish(&r);
        if(st != KPAX_OK) return st;
        return kpax_write_rows_csv(r.h_path, r.path_len, (uint32_t)pl->b.prm[0].S, filename, append);
    });
}

}  // extern "C"

namespace {

// Text output in the formats of the reference's helpers: rows of comma-separated values, floats
// with std::fixed and 6 digits (writeVectorToCSV, helper.cuh:56-80); one value per line, floats
// with 10 digits (writeValueToCSV, helper.cuh:93-106).
bool write_rows_f(const std::string& path, const float* v, size_t rows, size_t cols, bool append)
{
    FILE* f = fopen(path.c_str(), append ? "a" : "w");
    if(!f) return false;
    for(size_t i = 0; i < rows; ++i)
        for(size_t j = 0; j < cols; ++j) fprintf(f, j + 1 < cols ? "%.6f," : "%.6f\n", (double)v[i * cols + j]);
    return fclose(f) == 0;
}

template <class T>
bool write_rows_i(const std::string& path, const T* v, size_t rows, size_t cols, bool append)
{
    FILE* f = fopen(path.c_str(), append ? "a" : "w");
    if(!f) return false;
    for(size_t i = 0; i < rows; ++i)
        for(size_t j = 0; j < cols; ++j) fprintf(f, j + 1 < cols ? "%lld," : "%lld\n", (long long)v[i * cols + j]);
    return fclose(f) == 0;
}

bool write_value(const std::string& path, long long v, bool append)
{
    FILE* f = fopen(path.c_str(), append ? "a" : "w");
    if(!f) return false;
    fprintf(f, "%lld\n", v);
    return fclose(f) == 0;
}

bool write_value(const std::string& path, double v, bool append)
{
    FILE* f = fopen(path.c_str(), append ? "a" : "w");
    if(!f) return false;
    fprintf(f, "%.10f\n", v);
    return fclose(f) == 0;
}

}  // namespace

extern "C" {

static kpax_status plan_bench_body(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles,
                                   uint32_t n_obs, int32_t bench_itr, const char* out_dir, kpax_result* out)
{
    if(!pl || !out_dir) return set_error("kpax_plan_bench: null argument"), KPAX_EINVAL;
    const auto t0 = std::chrono::steady_clock::now();
    PlanBatch& b = pl->b;
    kpax_status st = b.begin(h_init, h_goal, 0, &d_obstacles, &n_obs, b.cfg[0].max_iter, 1u);
    if(st != KPAX_OK) return st;
    const KParams& p = b.prm[0];
    const uint32_t cap = p.cap, S = (uint32_t)p.S, n1 = (uint32_t)p.num_r1;
    const std::string base = std::string(out_dir) + "/Data/", bi = std::to_string(bench_itr);
    static const char* kDirs[] = {"Samples", "Parents", "TotalCountPerVertex", "ValidCountPerVertex", "Frontier",
                                  "FrontierRepeatCount", "VertexScores", "FrontierSize", "TreeSize", "ExpandedNodes",
                                  "ControlPathToGoal"};
    std::error_code ec;
    for(const char* d : kDirs) std::filesystem::create_directories(base + d + "/" + d + bi, ec);
    std::filesystem::create_directories(base + "ExecutionTime", ec);
    if(ec) return set_error("kpax_plan_bench: cannot create %s: %s", base.c_str(), ec.message().c_str()), KPAX_EINVAL;
    auto file = [&](const char* d, const std::string& name) { return base + d + "/" + d + bi + "/" + name; };
    std::vector<float> rows((size_t)cap * S), scores(n1);
    std::vector<int32_t> parents(cap), counter(n1), valid(n1), r1(cap);
    std::vector<uint8_t> rep(cap), flag(cap);
    uint64_t frontier_size = 1;  // the root, the frontier of the first iteration
    bool ok = true;
    for(uint32_t itr = 1; itr <= b.cfg[0].max_iter; ++itr) {
        if((st = b.iterate(1, 1u)) != KPAX_OK || (st = b.sync_ctl()) != KPAX_OK) return st;
        const Ctl c = b.h_ctl[0];
        if(c.iters_done < itr) break;  // the plan stopped before this iteration (tree full or error)
        uint32_t n = 0;
        std::fill(rows.begin(), rows.end(), 0.0f);
        std::fill(parents.begin(), parents.end(), -1);
        if((st = kpax_export_tree(pl, rows.data(), parents.data(), nullptr, cap, &n)) != KPAX_OK) return st;
        if((st = kpax_export_regions(pl, counter.data(), valid.data(), scores.data(), nullptr)) != KPAX_OK) return st;
        std::fill(rep.begin(), rep.end(), 0);
        if((st = kpax_export_frontier(pl, rep.data(), r1.data(), n)) != KPAX_OK) return st;
        uint64_t next_size = 0;
        for(uint32_t i = 0; i < n; ++i) {  // last iteration's nodes: their repeat as the next count pass sets it
            if(rep[i] == kPending) rep[i] = (uint8_t)(valid[r1[i]] < p.sparse_thr ? p.sparse_repeat : 1u);
            flag[i] = rep[i] != 0;
            next_size += flag[i];
        }
        std::fill(flag.begin() + n, flag.end(), 0);
        // a run's files start fresh with its first iteration (the reference appends to any left over)
        const bool app = itr > 1;
        const std::string k = std::to_string(itr);
        ok = ok && write_rows_f(file("Samples", "samples" + k + ".csv"), rows.data(), cap, S, false);
        ok = ok && write_rows_i(file("Parents", "parents" + k + ".csv"), parents.data(), cap, 1, false);
        ok = ok && write_rows_i(file("TotalCountPerVertex", "totalCountPerVertex.csv"), counter.data(), 1, n1, app);
        ok = ok && write_rows_i(file("ValidCountPerVertex", "validCountPerVertex.csv"), valid.data(), 1, n1, app);
        ok = ok && write_rows_i(file("Frontier", "frontier.csv"), flag.data(), 1, cap, app);
        ok = ok && write_rows_i(file("FrontierRepeatCount", "frontierRepeatCount.csv"), rep.data(), 1, cap, app);
        ok = ok && write_rows_f(file("VertexScores", "vertexScores.csv"), scores.data(), 1, n1, app);
        ok = ok && write_value(file("FrontierSize", "frontierSize.csv"), (long long)frontier_size, app);
        ok = ok && write_value(file("TreeSize", "treeSize.csv"), (long long)c.tree, app);
        ok = ok && write_value(file("ExpandedNodes", "expandedNodes.csv"), (long long)c.n, app);
        if(!ok) return set_error("kpax_plan_bench: cannot write under %s", base.c_str()), KPAX_EINVAL;
        frontier_size = next_size;
        if(c.goal_idx != kNone || c.full || c.error) break;
    }
    if((st = b.finish(out)) != KPAX_OK) return st;
    if(out->found && !write_rows_f(file("ControlPathToGoal", "controlPathToGoal.csv"), out->h_path, out->path_len, S, false))
        return set_error("kpax_plan_bench: cannot write the path under %s", base.c_str()), KPAX_EINVAL;
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if(!write_value(base + "ExecutionTime/executionTime.csv", secs, true))
        return set_error("kpax_plan_bench: cannot write the execution time under %s", base.c_str()), KPAX_EINVAL;
    return KPAX_OK;
}

kpax_status kpax_plan_bench(kpax_planner* pl, const float* h_init, const float* h_goal, const float* d_obstacles,
                            uint32_t n_obs, int32_t bench_itr, const char* out_dir, kpax_result* out)
{
    return no_throw("kpax_plan_bench",
                    [&] { return plan_bench_body(pl, h_init, h_goal, d_obstacles, n_obs, bench_itr, out_dir, out); });
}

kpax_status kpax_plan_result(kpax_planner* pl, kpax_result* out)
{
    return no_throw("kpax_plan_result", [&]() -> kpax_status {
        if(!pl || !pl->b.begun) return set_error("kpax_plan_result: no plan"), KPAX_EINVAL;
        return pl->b.finish(out);
    });
}

static kpax_status export_tree_body(kpax_planner* pl, float* h_rows, int32_t* h_parents, float* h_costs, uint32_t max_rows,
                                    uint32_t* n_rows);

kpax_status kpax_export_tree(kpax_planner* pl, float* h_rows, int32_t* h_parents, float* h_costs, uint32_t max_rows,
                             uint32_t* n_rows)
{
    return no_throw("kpax_export_tree", [&] { return export_tree_body(pl, h_rows, h_parents, h_costs, max_rows, n_rows); });
}

static kpax_status export_tree_body(kpax_planner* pl, float* h_rows, int32_t* h_parents, float* h_costs, uint32_t max_rows,
                                    uint32_t* n_rows)
{
    if(!pl) return set_error("kpax_export_tree: null planner"), KPAX_EINVAL;
    PlanBatch& b = pl->b;
    kpax_status st = b.sync_ctl();
    if(st != KPAX_OK) return st;
    const uint32_t n = std::min(b.h_ctl[0].tree, max_rows);
    if(n_rows) *n_rows = n;
    if(!n) return KPAX_OK;
    const KParams& p = b.prm[0];
    const TreeDev& t = b.hq[0].t;
    if(h_rows) {
        const int planes = p.sd == 12 ? 3 : 2;
        std::vector<float4> buf((size_t)n * (planes + 1));
        std::vector<float> dur(n);
        for(int k = 0; k < planes; ++k)
            KPAX_CUDA(cudaMemcpyAsync(buf.data() + (size_t)k * n, t.s[k], sizeof(float4) * n, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaMemcpyAsync(buf.data() + (size_t)planes * n, t.ctl, sizeof(float4) * n, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaMemcpyAsync(dur.data(), t.dur, sizeof(float) * n, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaStreamSynchronize(b.stream));
        for(uint32_t i = 0; i < n; ++i) {
            float* dst = h_rows + (size_t)i * p.S;
            for(int k = 0; k < p.sd; ++k) dst[k] = ((const float*)&buf[(size_t)(k / 4) * n + i])[k % 4];
            const float* c = (const float*)&buf[(size_t)planes * n + i];
            for(int k = 0; k < p.cd; ++k) dst[p.sd + k] = c[k];
            dst[p.S - 1] = dur[i];
        }
    }
    if(h_parents) KPAX_CUDA(cudaMemcpyAsync(h_parents, t.parent, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, b.stream));
    if(h_costs) KPAX_CUDA(cudaMemcpyAsync(h_costs, t.cost, sizeof(float) * n, cudaMemcpyDeviceToHost, b.stream));
    KPAX_CUDA(cudaStreamSynchronize(b.stream));
    return KPAX_OK;
}

kpax_status kpax_export_regions(kpax_planner* pl, int32_t* h_counter, int32_t* h_valid, float* h_scores, uint32_t* h_r2_bits)
{
    return no_throw("kpax_export_regions", [&]() -> kpax_status {
        if(!pl) return set_error("kpax_export_regions: null planner"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        const KParams& p = b.prm[0];
        const RegDev& rg = b.hq[0].rg;
        if(h_counter) KPAX_CUDA(cudaMemcpyAsync(h_counter, rg.counter, sizeof(int32_t) * p.num_r1, cudaMemcpyDeviceToHost, b.stream));
        if(h_valid) KPAX_CUDA(cudaMemcpyAsync(h_valid, rg.valid, sizeof(int32_t) * p.num_r1, cudaMemcpyDeviceToHost, b.stream));
        if(h_scores) KPAX_CUDA(cudaMemcpyAsync(h_scores, rg.score, sizeof(float) * p.num_r1, cudaMemcpyDeviceToHost, b.stream));
        if(h_r2_bits) KPAX_CUDA(cudaMemcpyAsync(h_r2_bits, rg.cur, sizeof(uint32_t) * p.r2_words, cudaMemcpyDeviceToHost, b.stream));
        kpax_status st = b.sync_ctl();
        if(st != KPAX_OK) return st;
        if(h_scores) {  // stored raw (negative = no valid sample); normalised as region_score does
            const float total = b.h_ctl[0].score_total;
            const bool ready = b.h_ctl[0].scores_ready != 0u;
            for(int r = 0; r < p.num_r1; ++r) {
                const float raw = h_scores[r];
                h_scores[r] = !ready ? 0.0f : (raw < 0.0f ? 1.0f : p.eps + raw / total);
            }
        }
        return KPAX_OK;
    });
}

kpax_status kpax_export_frontier(kpax_planner* pl, uint8_t* h_repeat, int32_t* h_r1, uint32_t max_rows)
{
    return no_throw("kpax_export_frontier", [&]() -> kpax_status {
        if(!pl) return set_error("kpax_export_frontier: null planner"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        kpax_status st = b.sync_ctl();
        if(st != KPAX_OK) return st;
        const uint32_t n = std::min(b.h_ctl[0].tree, max_rows);
        if(b.h_ctl[0].tree_old) {
            k_reactivate<<<(b.h_ctl[0].tree_old + 255) / 256, 256, 0, b.stream>>>(b.dq);
            KPAX_CHECK_LAUNCH();
            count_launch();
        }
        if(n && h_repeat) KPAX_CUDA(cudaMemcpyAsync(h_repeat, b.hq[0].t.rep, n, cudaMemcpyDeviceToHost, b.stream));
        if(n && h_r1) KPAX_CUDA(cudaMemcpyAsync(h_r1, b.hq[0].t.r1, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaStreamSynchronize(b.stream));
        return KPAX_OK;
    });
}

kpax_status kpax_debug_capture(kpax_planner* pl, int32_t enable)
{
    return no_throw("kpax_debug_capture", [&]() -> kpax_status {
        if(!pl) return set_error("kpax_debug_capture: null planner"), KPAX_EINVAL;
        return pl->b.set_capture(enable != 0);
    });
}

kpax_status kpax_export_children(kpax_planner* pl, float* h_rows, uint8_t* h_valid, int32_t* h_r1, int32_t* h_r2,
                                 uint8_t* h_next, int32_t* h_parent, uint32_t max_rows, uint32_t* n_children)
{
    return no_throw("kpax_export_children", [&]() -> kpax_status {
        if(!pl || !pl->b.capture_on) return set_error("kpax_export_children: capture is off"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        kpax_status st = b.sync_ctl();
        if(st != KPAX_OK) return st;
        const uint32_t n = std::min(b.h_ctl[0].n, max_rows);
        if(n_children) *n_children = n;
        if(!n) return KPAX_OK;
        const CaptureDev& c = b.cap;
        if(h_rows) KPAX_CUDA(cudaMemcpyAsync(h_rows, c.rows, sizeof(float) * n * b.prm[0].S, cudaMemcpyDeviceToHost, b.stream));
        if(h_valid) KPAX_CUDA(cudaMemcpyAsync(h_valid, c.valid, n, cudaMemcpyDeviceToHost, b.stream));
        if(h_r1) KPAX_CUDA(cudaMemcpyAsync(h_r1, c.r1, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, b.stream));
        if(h_r2) KPAX_CUDA(cudaMemcpyAsync(h_r2, c.r2, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, b.stream));
        if(h_next) KPAX_CUDA(cudaMemcpyAsync(h_next, c.next, n, cudaMemcpyDeviceToHost, b.stream));
        if(h_parent) KPAX_CUDA(cudaMemcpyAsync(h_parent, c.parent, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaStreamSynchronize(b.stream));
        return KPAX_OK;
    });
}

kpax_status kpax_export_proposal(kpax_planner* pl, float* h_mix, uint32_t max_entries, uint32_t* n_entries)
{
    return no_throw("kpax_export_proposal", [&]() -> kpax_status {
        if(!pl || !pl->b.hq[0].mix) return set_error("kpax_export_proposal: the learned proposal is off"), KPAX_EINVAL;
        PlanBatch& b = pl->b;
        kpax_status st = b.sync_ctl();
        if(st != KPAX_OK) return st;
        const uint32_t n = std::min(b.h_ctl[0].E, max_entries);
        if(n_entries) *n_entries = n;
        if(n && h_mix)
            KPAX_CUDA(cudaMemcpyAsync(h_mix, b.hq[0].mix, sizeof(float) * n * mlp::kMixFloats, cudaMemcpyDeviceToHost, b.stream));
        KPAX_CUDA(cudaStreamSynchronize(b.stream));
        return KPAX_OK;
    });
}

// ---------------------------------------------------------------- batches of queries

kpax_status kpax_batch_create(const kpax_config* cfgs, uint32_t n, kpax_batch** out)
{
    if(!cfgs || !n || !out) return set_error("kpax_batch_create: null argument or empty batch"), KPAX_EINVAL;
    *out = nullptr;
    kpax_batch* b = new(std::nothrow) kpax_batch();
    if(!b) return set_error("kpax_batch_create: host allocation failed"), KPAX_ENOMEM;
    kpax_status st = no_throw("kpax_batch_create", [&] { return b->b.init(cfgs, n); });
    if(st != KPAX_OK) {
        b->b.release();
        delete b;
        return st;
    }
    *out = b;
    return KPAX_OK;
}

kpax_status kpax_batch_destroy(kpax_batch* b)
{
    if(!b) return KPAX_OK;
    b->b.release();
    delete b;
    return KPAX_OK;
}

kpax_status kpax_set_proposal(kpax_planner* pl, kpax_mlp* net, float epsilon)
{
    return no_throw("kpax_set_proposal", [&]() -> kpax_status {
        if(!pl) return set_error("kpax_set_proposal: null planner"), KPAX_EINVAL;
        if(net && pl->b.prm[0].model != KPAX_MODEL_QUADROTOR)
            return set_error("kpax_set_proposal: the proposal network is defined for the quadrotor"), KPAX_EINVAL;
        return pl->b.set_proposal(net, epsilon, nullptr);
    });
}

kpax_status kpax_batch_set_proposal(kpax_batch* bt, kpax_mlp* net, float epsilon, const uint8_t* enable)
{
    return no_throw("kpax_batch_set_proposal", [&]() -> kpax_status {
        if(!bt) return set_error("kpax_batch_set_proposal: null batch"), KPAX_EINVAL;
        return bt->b.set_proposal(net, epsilon, enable);
    });
}

kpax_status kpax_batch_plan(kpax_batch* bt, const float* h_inits, const float* h_goals, uint32_t row_stride,
                            const float* const* d_obstacles, const uint32_t* n_obs, kpax_result* results,
                            kpax_batch_stats* stats)
{
    return no_throw("kpax_batch_plan", [&]() -> kpax_status {
        if(!bt || !d_obstacles || !n_obs) return set_error("kpax_batch_plan: null argument"), KPAX_EINVAL;
        PlanBatch& b = bt->b;
        if(row_stride < b.s_max) return set_error("kpax_batch_plan: row_stride %u < %u", row_stride, b.s_max), KPAX_EINVAL;
        uint32_t max_iter = 0;
        for(const kpax_config& c : b.cfg) max_iter = std::max(max_iter, c.max_iter);
        kpax_status st = b.begin(h_inits, h_goals, row_stride, d_obstacles, n_obs, max_iter, 1u);
        if(st != KPAX_OK) return st;
        // each query stops at its own max_iter
        if((st = b.sync_ctl()) != KPAX_OK) return st;
        for(uint32_t q = 0; q < b.nq; ++q) b.h_ctl[q].max_iters = b.cfg[q].max_iter;
        if((st = b.write_ctl()) != KPAX_OK) return st;
        st = b.run(plan_guard(b, max_iter));
        double ms = 0.0;
        kpax_status st2 = b.finish(results, &ms);
        if(stats) {
            memset(stats, 0, sizeof(*stats));
            stats->ms = ms;
            for(uint32_t q = 0; q < b.nq; ++q) {
                const Ctl& c = b.h_ctl[q];
                stats->iters = std::max(stats->iters, c.iters_done);
                stats->found += c.goal_idx != kNone;
                stats->expansions += c.n_exp;
                stats->valid_expansions += c.n_valid;
                stats->steps += c.n_steps;
            }
        }
        return st != KPAX_OK ? st : st2;
    });
}

}  // extern "C"

namespace {
// Tile 1 of a look-back whose tile 0 never publishes: the expansion's bounded wait runs out after
// spin_limit polls and reports a timeout instead of spinning on.
__global__ void k_test_lookback_timeout(unsigned long long* lb, uint32_t spin_limit, uint32_t* status)
{
    uint32_t excl = 0;
    const bool ok = lb_exclusive(lb, 1u, 1u, excl, spin_limit);
    if(threadIdx.x == 0) *status = ok ? 0u : kErrTimeout;
}
}  // namespace

extern "C" {

kpax_status kpax_test_wait_timeout(uint32_t spin_limit, uint32_t* h_status, void* stream)
{
    return no_throw("kpax_test_wait_timeout", [&]() -> kpax_status {
        if(!h_status || spin_limit == 0 || spin_limit > kSpinLimit)
            return set_error("kpax_test_wait_timeout: need a status pointer and 1 <= spin_limit <= %u", kSpinLimit),
                   KPAX_EINVAL;
        char* mem = nullptr;
        KPAX_CUDA(cudaMalloc(&mem, 64));
        struct Free {
            char* m;
            ~Free() { cudaFree(m); }
        } free_mem{mem};
        cudaStream_t s = (cudaStream_t)stream;
        KPAX_CUDA(cudaMemsetAsync(mem, 0, 64, s));  // status words of tiles 0 and 1: never published
        uint32_t* d_status = reinterpret_cast<uint32_t*>(mem + 32);
        k_test_lookback_timeout<<<1, 32, 0, s>>>(reinterpret_cast<unsigned long long*>(mem), spin_limit, d_status);
        KPAX_CHECK_LAUNCH();
        count_launch(1);
        KPAX_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        KPAX_CUDA(cudaStreamSynchronize(s));
        if(*h_status & kErrTimeout)
            return set_error("kpax_test_wait_timeout: the look-back wait gave up after %u polls", spin_limit), KPAX_ETIMEOUT;
        return KPAX_OK;
    });
}

// ---------------------------------------------------------------- frontier compaction on its own

kpax_status kpax_frontier_compact(const kpax_config* cfg, uint8_t* d_repeat, uint32_t n_nodes, uint32_t budget,
                                  uint32_t* d_entries, kpax_frontier_stats* out, void* stream)
{
    return no_throw("kpax_frontier_compact", [&]() -> kpax_status {
        if(!cfg || !out || (n_nodes && !d_repeat) || (budget && !d_entries))
            return set_error("kpax_frontier_compact: null argument"), KPAX_EINVAL;
        if(n_nodes > (1u << 24)) return set_error("kpax_frontier_compact: %u nodes (at most 2^24)", n_nodes), KPAX_EINVAL;
        KParams p;
        kpax_status st = derive_params(*cfg, &p);
        if(st != KPAX_OK) return st;
        // the count pass takes B = min(budget, cap - tree): a capacity of tree + budget leaves B = budget
        budget = std::min<uint32_t>(budget, 0xFFFFFFFFu - n_nodes);
        p.budget = budget;
        p.cap = n_nodes + budget;
        // one query whose tree is the caller's repeat bytes: region ids 0, region 0 without valid
        // samples (a pending node counts as sparse), no re-activation (tree_old = 0)
        const uint32_t ntiles = std::max<uint32_t>(1, (n_nodes + kTile - 1) / kTile);
        auto al = [](size_t b) { return (b + kAlign - 1) / kAlign * kAlign; };
        const size_t o_ctl = al(sizeof(QueryDev)), o_tiles = o_ctl + al(sizeof(Ctl)), o_small = o_tiles + al(4ull * ntiles),
                     o_r1 = o_small + kAlign, bytes = o_r1 + al(4ull * std::max<uint32_t>(n_nodes, 1));
        char* mem = nullptr;
        KPAX_CUDA(cudaMalloc(&mem, bytes));
        struct Free {
            char* m;
            ~Free() { cudaFree(m); }
        } free_mem{mem};
        cudaStream_t s = (cudaStream_t)stream;
        QueryDev q{};
        q.p = p;
        q.t.rep = d_repeat;
        q.t.r1 = reinterpret_cast<int32_t*>(mem + o_r1);
        q.rg.score = reinterpret_cast<float*>(mem + o_small);
        q.rg.valid = reinterpret_cast<int32_t*>(mem + o_small + 16);
        q.farr = reinterpret_cast<uint32_t*>(mem + o_small + 32);
        uint32_t* d_active = reinterpret_cast<uint32_t*>(mem + o_small + 48);
        q.ctl = reinterpret_cast<Ctl*>(mem + o_ctl);
        q.tiles = reinterpret_cast<uint32_t*>(mem + o_tiles);
        q.entries = d_entries;
        Ctl c{};
        c.tree = n_nodes;
        c.iter = 1u;
        c.score_total = 1.0f;
        c.goal_idx = kNone;
        KPAX_CUDA(cudaMemsetAsync(mem + o_small, 0, bytes - o_small, s));
        KPAX_CUDA(cudaMemcpyAsync(mem, &q, sizeof(q), cudaMemcpyHostToDevice, s));
        KPAX_CUDA(cudaMemcpyAsync(q.ctl, &c, sizeof(c), cudaMemcpyHostToDevice, s));
        const QueryDev* dq = reinterpret_cast<const QueryDev*>(mem);
        const uint32_t gx = std::min<uint32_t>(ntiles, kFrontierCTAs);
        k_frontier_count<<<dim3(gx, 1), kFrontierBS, 0, s>>>(dq, d_active);
        k_frontier_write<<<dim3(gx, 1), kFrontierBS, 0, s>>>(dq);
        KPAX_CHECK_LAUNCH();
        count_launch(2);
        KPAX_CUDA(cudaMemcpyAsync(&c, q.ctl, sizeof(c), cudaMemcpyDeviceToHost, s));
        KPAX_CUDA(cudaStreamSynchronize(s));
        out->R = c.R, out->k = c.k, out->E = c.E, out->n = c.n;
        return KPAX_OK;
    });
}

}  // extern "C"

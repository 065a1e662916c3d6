// kpax_rekino.cu — ReKinoLite, the fork's warp-greedy planner (src/ReKino/ReKinoLite.cu:251-459),
// on the same propagation, collision and draw code as the tree planner.
//
// Each warp keeps one path.  Per iteration its lanes propagate samples_per_thread random
// segments each from the path's last node; the valid one closest to the goal (lowest sample
// index on ties) extends the path, or with probability epsilon_greedy a uniformly chosen valid
// one; when none is valid the path backtracks 1-5 nodes.  Deterministic replacements for the
// reference's races and wraps:
//   * draws come from Philox4x32-10 (sample draws: counter (512 w + j, iteration, 0|1, plan);
//     the warp's selection / backtrack draws: counter (w, iteration, 2, plan));
//   * the winner is the warp with the smallest (iteration, warp id) that reached the goal ball
//     (the reference keeps whichever warp's atomicCAS lands first); a warp stops once a goal was
//     found at an earlier iteration, so the winner does not depend on timing;
//   * a path reaching MAX_PATH_LENGTH nodes restarts from the start state (the reference wraps
//     its depth to 0 and overwrites the start state with the new node).
// The wall-clock give-up (6 s, clock64 in the reference) is a %globaltimer deadline.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "kpax.h"
#include <new>

#include "kpax_internal.h"

using namespace kpax;

namespace {

constexpr int kMaxPath = 200;       // MAX_PATH_LENGTH (ReKinoLite.cuh:20)
constexpr int kMaxSamples = 512;    // samples per warp cap (ReKinoLite.cu:84)

struct RekinoDev {
    KParams p;
    Grid g;
    const float* init;   // S floats
    const float* goal;   // S floats
    float* paths;        // [warps][kMaxPath][S]
    int32_t* lens;       // last path index per warp
    unsigned long long* best;      // (iteration << 32) | warp of the earliest goal, ~0 = none
    unsigned long long* counters;  // samples propagated, valid samples
    uint32_t max_iter, spt, plan;
    float eps_greedy;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Distance of a state's position to the goal position, rounded as the tree planner's cost.
__device__ __forceinline__ float goal_distance3(const float* s, const float* g)
{
    const float dx = __fsub_rn(s[0], g[0]), dy = __fsub_rn(s[1], g[1]), dz = __fsub_rn(s[2], g[2]);
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
}

template <int M>
__global__ void __launch_bounds__(32) k_rekino(const RekinoDev d)
{
    constexpr int SD = ModelDims<M>::SD, CD = ModelDims<M>::CD, S = SD + CD + 1;
    extern __shared__ float s_cand[];  // [spt * 32][S] candidate rows, then [spt * 32] distances
    const KParams& p = d.p;
    const uint32_t w = blockIdx.x, lane = threadIdx.x, spt = d.spt, nsamp = 32u * spt;
    float* s_dist = s_cand + (size_t)nsamp * S;
    float* path = d.paths + (size_t)w * kMaxPath * S;
    if(lane < (uint32_t)S) path[lane] = d.init[lane];
    __syncwarp();
    int depth = 0;
    unsigned long long n_samp = 0, n_valid = 0;
    const unsigned long long t0 = now_ns();
    float g[3] = {d.goal[0], d.goal[1], d.goal[2]};
    for(uint32_t it = 0; it < d.max_iter; ++it) {
        // give-up (ReKinoLite.cu:300-308) and the stop once a goal was reached at an earlier
        // iteration, decided by lane 0 for the whole warp
        bool stop = false;
        if(lane == 0) {
            const unsigned long long found = *reinterpret_cast<volatile unsigned long long*>(d.best);
            stop = (found >> 32) < it || (it % 100u == 0u && now_ns() - t0 > d.timeout_ns);
        }
        if(__shfl_sync(0xffffffffu, stop, 0)) break;
        float cur[SD];
#pragma unroll
        for(int q = 0; q < SD; ++q) cur[q] = path[(size_t)depth * S + q];
        // each lane propagates its samples j = lane * spt + k (ReKinoLite.cu:318-345)
        for(uint32_t k = 0; k < spt; ++k) {
            const uint32_t j = lane * spt + k;
            float u[6], cc[4], rc[4], s[SD];
            child_draws(p, d.plan, it, w * (uint32_t)kMaxSamples + j, u);
            const int steps = draw_controls(p, u, cc);
#pragma unroll
            for(int q = 0; q < SD; ++q) s[q] = cur[q];
            int done = 0;
            const bool valid = propagate<M>(p, d.g, s, cc, steps, done);
            row_controls<M>(cc, rc);
            float* row = s_cand + (size_t)j * S;
#pragma unroll
            for(int q = 0; q < SD; ++q) row[q] = s[q];
#pragma unroll
            for(int q = 0; q < CD; ++q) row[SD + q] = rc[q];
            row[SD + CD] = __fmul_rn(p.h, (float)steps);
            s_dist[j] = valid ? goal_distance3(s, g) : INFINITY;
            n_samp += 1, n_valid += valid ? 1 : 0;
        }
        __syncwarp();
        // greedy choice: smallest distance, lowest index on ties (ReKinoLite.cu:351-362)
        float bd = INFINITY;
        int bj = -1, nv = 0;
        for(uint32_t k = 0; k < spt; ++k) {
            const uint32_t j = lane * spt + k;
            const float dj = s_dist[j];
            if(dj < bd) bd = dj, bj = (int)j;
            nv += dj < INFINITY ? 1 : 0;
        }
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) {
            const float od = __shfl_xor_sync(0xffffffffu, bd, off);
            const int oj = __shfl_xor_sync(0xffffffffu, bj, off);
            if(od < bd || (od == bd && oj >= 0 && (bj < 0 || oj < bj))) bd = od, bj = oj;
        }
        const U4 r = philox(w, it, 2u, d.plan, p.seed_lo, p.seed_hi);
        if(d.eps_greedy > 0.0f && u01(r.x) < d.eps_greedy) {  // epsilon-greedy (ReKinoLite.cu:365-390)
            int incl = nv;  // valid samples of lanes <= this one (sample index order is lane-major)
#pragma unroll
            for(int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, off);
                if((int)lane >= off) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            if(total > 0) {
                const int pick = (int)(u01(r.y) * (float)total);  // the pick-th valid sample
                int own = -1, before = incl - nv;
                if(pick >= before && pick < incl) {
                    int c = before;
                    for(uint32_t k = 0; k < spt; ++k) {
                        const uint32_t j = lane * spt + k;
                        if(s_dist[j] < INFINITY) {
                            if(c == pick) {
                                own = (int)j;
                                break;
                            }
                            ++c;
                        }
                    }
                }
                const unsigned owner = __ballot_sync(0xffffffffu, own >= 0);
                bj = __shfl_sync(0xffffffffu, own, __ffs(owner) - 1);
                bd = s_dist[bj];
            }
        }
        if(bj >= 0) {
            if(depth + 1 >= kMaxPath) {
                depth = 0;  // full path: restart from the start state (the node is dropped)
            } else {
                ++depth;
                if(lane < (uint32_t)S) path[(size_t)depth * S + lane] = s_cand[(size_t)bj * S + lane];
                __syncwarp();
                if(bd < p.goal_thresh) {  // goal ball reached (ReKinoLite.cu:395-399)
                    if(lane == 0) d.lens[w] = depth, atomicMin(d.best, ((unsigned long long)it << 32) | w);
                    break;
                }
            }
        } else if(depth > 0) {  // every sample failed: back up 1-5 nodes (ReKinoLite.cu:425-435)
            depth = max(0, depth - (1 + f2i(u01(r.z) * 5.0f)));
        }
        if(lane == 0) d.lens[w] = depth;
        __syncwarp();
    }
    for(int off = 16; off > 0; off >>= 1) {
        n_samp += __shfl_xor_sync(0xffffffffu, n_samp, off);
        n_valid += __shfl_xor_sync(0xffffffffu, n_valid, off);
    }
    if(lane == 0) atomicAdd(d.counters, n_samp), atomicAdd(d.counters + 1, n_valid);
}

}  // namespace

struct kpax_rekino {
    kpax_config cfg{};
    KParams p{};
    kpax_rekino_params rp{};
    Env env;
    float* d_paths = nullptr;
    int32_t* d_lens = nullptr;
    unsigned long long* d_best = nullptr;  // best key, then 2 counters
    float* d_ig = nullptr;
    float* d_obs = nullptr;
    uint32_t obs_cap = 0;
    std::vector<float> h_path;
    uint32_t plans = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static void rekino_release(kpax_rekino* r)
{
    if(r->stream) cudaStreamSynchronize(r->stream);
    r->env.release();
    void* dev[] = {r->d_paths, r->d_lens, r->d_best, r->d_ig, r->d_obs};
    for(void* q : dev)
        if(q) cudaFree(q);
    if(r->ev0) cudaEventDestroy(r->ev0);
    if(r->ev1) cudaEventDestroy(r->ev1);
    if(r->stream) cudaStreamDestroy(r->stream);
}

extern "C" {

kpax_status kpax_rekino_defaults(kpax_rekino_params* out)
{
    if(!out) return set_error("kpax_rekino_defaults: null output"), KPAX_EINVAL;
    memset(out, 0, sizeof(*out));
    out->num_warps = 512;            // ReKinoLite.cu:11
    out->samples_per_thread = 1;     // :13
    out->epsilon_greedy = 0.0f;      // :14
    out->max_iterations = 20000;     // MAX_ITER_REKINO (config.h:213)
    out->timeout_ms = 6000.0;        // 6-second give-up (:120-122)
    return KPAX_OK;
}

kpax_status kpax_rekino_create(const kpax_config* cfg, const kpax_rekino_params* rp, kpax_rekino** out)
{
    if(!cfg || !rp || !out) return set_error("kpax_rekino_create: null argument"), KPAX_EINVAL;
    *out = nullptr;
    if(rp->num_warps == 0 || rp->num_warps > (1u << 20)) return set_error("kpax_rekino_create: num_warps in [1, 2^20]"), KPAX_EINVAL;
    if(rp->samples_per_thread == 0 || 32u * rp->samples_per_thread > (uint32_t)kMaxSamples)
        return set_error("kpax_rekino_create: samples_per_thread in [1, 16]"), KPAX_EINVAL;
    if(!(rp->epsilon_greedy >= 0.0f && rp->epsilon_greedy <= 1.0f) || !(rp->timeout_ms > 0.0))
        return set_error("kpax_rekino_create: epsilon_greedy in [0,1] and a positive timeout"), KPAX_EINVAL;
    kpax_rekino* r = new(std::nothrow) kpax_rekino();
    if(!r) return set_error("kpax_rekino_create: host allocation failed"), KPAX_ENOMEM;
    r->cfg = *cfg;
    r->rp = *rp;
    kpax_status st = derive_params(*cfg, &r->p);
    auto fail = [&](kpax_status s) {
        rekino_release(r);
        delete r;
        return s;
    };
    if(st != KPAX_OK) return fail(st);
    const size_t S = (size_t)r->p.S;
#define KPAX_RK(call)                                                                            \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if(e_ != cudaSuccess) {                                                                  \
            set_error("kpax_rekino_create: %s", cudaGetErrorString(e_));                         \
            return fail(e_ == cudaErrorMemoryAllocation ? KPAX_ENOMEM : KPAX_ECUDA);             \
        }                                                                                        \
    } while(0)
    KPAX_RK(cudaMalloc(&r->d_paths, sizeof(float) * rp->num_warps * kMaxPath * S));
    KPAX_RK(cudaMalloc(&r->d_lens, sizeof(int32_t) * rp->num_warps));
    KPAX_RK(cudaMalloc(&r->d_best, sizeof(unsigned long long) * 3));
    KPAX_RK(cudaMalloc(&r->d_ig, sizeof(float) * 2 * S));
    KPAX_RK(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
    KPAX_RK(cudaEventCreate(&r->ev0));
    KPAX_RK(cudaEventCreate(&r->ev1));
#undef KPAX_RK
    *out = r;
    return KPAX_OK;
}

kpax_status kpax_rekino_destroy(kpax_rekino* r)
{
    if(!r) return KPAX_OK;
    rekino_release(r);
    delete r;
    return KPAX_OK;
}

static kpax_status rekino_plan_body(kpax_rekino* r, const float* h_init, const float* h_goal, const float* d_obstacles,
                                    uint32_t n_obs, kpax_result* out);

kpax_status kpax_rekino_plan(kpax_rekino* r, const float* h_init, const float* h_goal, const float* d_obstacles, uint32_t n_obs,
                             kpax_result* out)
{
    return no_throw("kpax_rekino_plan", [&] { return rekino_plan_body(r, h_init, h_goal, d_obstacles, n_obs, out); });
}

static kpax_status rekino_plan_body(kpax_rekino* r, const float* h_init, const float* h_goal, const float* d_obstacles,
                                    uint32_t n_obs, kpax_result* out)
{
    if(!r || !h_init || !h_goal || !out || (n_obs && !d_obstacles)) return set_error("kpax_rekino_plan: null argument"), KPAX_EINVAL;
    const KParams& p = r->p;
    const uint32_t S = (uint32_t)p.S, W = r->rp.num_warps, spt = r->rp.samples_per_thread;
    KPAX_CUDA(cudaEventRecord(r->ev0, r->stream));
    kpax_status st = r->env.build(p, d_obstacles, n_obs, r->stream);
    if(st != KPAX_OK) return st;
    std::vector<float> ig(2 * (size_t)S);
    memcpy(ig.data(), h_init, sizeof(float) * S);
    memcpy(ig.data() + S, h_goal, sizeof(float) * S);
    KPAX_CUDA(cudaMemcpyAsync(r->d_ig, ig.data(), sizeof(float) * 2 * S, cudaMemcpyHostToDevice, r->stream));
    const unsigned long long init_best[3] = {~0ull, 0ull, 0ull};
    KPAX_CUDA(cudaMemcpyAsync(r->d_best, init_best, sizeof(init_best), cudaMemcpyHostToDevice, r->stream));
    KPAX_CUDA(cudaMemsetAsync(r->d_lens, 0, sizeof(int32_t) * W, r->stream));
    RekinoDev d{p, r->env.view(), r->d_ig, r->d_ig + S, r->d_paths, r->d_lens, r->d_best, r->d_best + 1,
                r->rp.max_iterations, spt, r->plans, r->rp.epsilon_greedy, (unsigned long long)(r->rp.timeout_ms * 1e6)};
    const size_t smem = sizeof(float) * 32u * spt * (S + 1);
    if(p.model == KPAX_MODEL_DOUBLE_INTEGRATOR) k_rekino<KPAX_MODEL_DOUBLE_INTEGRATOR><<<W, 32, smem, r->stream>>>(d);
    else if(p.model == KPAX_MODEL_DUBINS_AIRPLANE) k_rekino<KPAX_MODEL_DUBINS_AIRPLANE><<<W, 32, smem, r->stream>>>(d);
    else k_rekino<KPAX_MODEL_QUADROTOR><<<W, 32, smem, r->stream>>>(d);
    KPAX_CHECK_LAUNCH();
    count_launch();
    r->plans += 1;
    unsigned long long h_best[3];
    KPAX_CUDA(cudaMemcpyAsync(h_best, r->d_best, sizeof(h_best), cudaMemcpyDeviceToHost, r->stream));
    KPAX_CUDA(cudaStreamSynchronize(r->stream));
    kpax_result res{};
    res.expansions = h_best[1];
    res.valid_expansions = h_best[2];
    if(h_best[0] != ~0ull) {
        const uint32_t win = (uint32_t)(h_best[0] & 0xFFFFFFFFu), iter = (uint32_t)(h_best[0] >> 32);
        int32_t len = 0;
        KPAX_CUDA(cudaMemcpyAsync(&len, r->d_lens + win, sizeof(int32_t), cudaMemcpyDeviceToHost, r->stream));
        KPAX_CUDA(cudaStreamSynchronize(r->stream));
        std::vector<float> rows((size_t)(len + 1) * S);
        KPAX_CUDA(cudaMemcpyAsync(rows.data(), r->d_paths + (size_t)win * kMaxPath * S, sizeof(float) * rows.size(),
                                  cudaMemcpyDeviceToHost, r->stream));
        KPAX_CUDA(cudaStreamSynchronize(r->stream));
        r->h_path.assign(rows.size(), 0.0f);  // goal node first, start state last
        float cost = 0.0f;  // FP32, goal to root, as the planner's path walk
        for(int i = 0; i <= len; ++i) {
            memcpy(r->h_path.data() + (size_t)i * S, rows.data() + (size_t)(len - i) * S, sizeof(float) * S);
            if(i < len) cost += rows[(size_t)(len - i) * S + S - 1];
        }
        res.found = 1;
        res.goal_idx = win;
        res.path_len = (uint32_t)(len + 1);
        res.iters = iter + 1;
        res.tree_size = (uint32_t)(len + 1);
        res.h_path = r->h_path.data();
        res.path_cost = cost;
    } else {
        res.iters = r->rp.max_iterations;
    }
    KPAX_CUDA(cudaEventRecord(r->ev1, r->stream));
    KPAX_CUDA(cudaEventSynchronize(r->ev1));
    float ms = 0.0f;
    KPAX_CUDA(cudaEventElapsedTime(&ms, r->ev0, r->ev1));
    res.ms = ms;
    *out = res;
    return KPAX_OK;
}

}  // extern "C"

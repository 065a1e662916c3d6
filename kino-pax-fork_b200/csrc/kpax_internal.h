// kpax_internal.h — host-side objects shared by the environment, batch and planner units.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include <atomic>
#include <exception>
#include <new>

#include "kpax_device.cuh"
#include "kpax_params.h"

// Error helpers: record the failing call's text and return a status, never exit.
#define KPAX_CUDA(call)                                                                             \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if(e_ != cudaSuccess) {                                                                     \
            kpax::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));     \
            return e_ == cudaErrorMemoryAllocation ? KPAX_ENOMEM : KPAX_ECUDA;                      \
        }                                                                                           \
    } while(0)

#define KPAX_CHECK_LAUNCH() KPAX_CUDA(cudaGetLastError())

namespace kpax {
// An NVTX range over a host call (shown by Nsight Systems; without a tool attached the push and
// pop return at once).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Runs f() inside an NVTX range named `what` and turns a C++ exception (a failed host allocation
// above all) into a status, so nothing thrown crosses the C ABI.
template <class F>
kpax_status no_throw(const char* what, F&& f)
{
    NvtxRange range(what);
    try {
        return f();
    } catch(const std::bad_alloc&) {
        set_error("%s: host allocation failed", what);
        return KPAX_ENOMEM;
    } catch(const std::exception& e) {
        set_error("%s: %s", what, e.what());
        return KPAX_EINVAL;
    }
}
}  // namespace kpax

namespace kpax {

extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Uniform-grid spatial hash over one obstacle set (device buffers, grown on demand).
struct Env {
    float cell = 0.0f, wmin = 0.0f;
    int dim = 0;
    uint32_t n_obs = 0, n_cells = 0, n_ent = 0;
    float4* d_obs = nullptr;  // 2 per obstacle: (min xyz, 0), (max xyz, 0)
    uint32_t* d_off = nullptr;  // n_cells + 1
    uint32_t* d_cursor = nullptr;
    uint32_t* d_ent = nullptr;
    uint32_t* h_total = nullptr;  // pinned
    uint32_t obs_cap = 0, ent_cap = 0;
    bool owned_by_planner = false;
    void* d_live = nullptr;  // scratch of the phased segment batch (grown on demand)
    size_t live_cap = 0;

    Grid view() const { return Grid{d_obs, d_off, d_ent, wmin, 1.0f / cell, dim}; }
    // Build from n x 6 device floats on `stream` (synchronises once to size the entry list).
    kpax_status build(const KParams& p, const float* d_obstacles, uint32_t n, cudaStream_t stream);
    void release();
};

// Batch entry points used by the C ABI (kpax_env.cu).
kpax_status launch_propagate(const KParams& p, const Grid& g, const float* parents, const float* draws, uint32_t stream_id,
                             uint32_t n, float* rows, uint8_t* valid, int32_t* steps, cudaStream_t stream);

// Learned proposal (kpax_learn.cu): occupancy bits of the R1 workspace cells (W1^3 bits, zeroed
// and filled on `stream`) and the packed tensor-core image of a network (null until packed).
kpax_status launch_occupancy(const KParams& p, const Grid& g, uint32_t* d_words, cudaStream_t stream);

}  // namespace kpax

struct kpax_env {
    kpax::KParams params;
    kpax::Env env;
    uint32_t* d_occ = nullptr;  // occupancy bits, computed on first use by the learned proposal
};

namespace kpax {
const uint8_t* mlp_image(const kpax_mlp* n);
}

// kpax_params.h — launch parameters derived once on the host from a kpax_config.
//
// Everything a kernel needs about the dynamics, the checks and the region grid is here,
// precomputed so that device code does only float arithmetic.  The reference evaluates a
// few tests in double because its macros are double literals (C_MIN/C_MAX = +-M_PI,
// DUBINS_AIRPLANE_MIN/MAX_PITCH = +-M_PI/3, config.h:231-232, 280-281); those tests are
// replaced by float thresholds that give the identical verdict for every float input
// (see kpax_config.cpp).
#pragma once
#include <stdint.h>

#include "kpax.h"

namespace kpax {

constexpr int kMaxThr = 15;  // attitude split lengths are limited to 16

struct KParams {
    int model, sd, cd, S;   // state dim, control dim, sample dim (S = sd + cd + 1)
    float h, hh, h6;        // STEP_SIZE, 0.5f*STEP_SIZE, STEP_SIZE/6.0f
    int nsteps, fixed_steps;
    float ws_lo, ws_hi;     // workspace check bounds of the model
    float vmin, vmax;
    float pitch_lo, pitch_hi;  // p < pitch_lo  <=>  (double)p < MIN_PITCH, etc.
    float clo[4], crng[4];     // control ranges in draw order: c = clo + u * crng
    // region grid (Graph.cu:99-205)
    int W1, C1, V1, W2, C2, V2, cdim, vdim, w_only;
    float wmin, wspan, vmin_r, vspan, w1size, v1size;
    float cthr1[kMaxThr];   // attitude R1 index = #{k : c >= cthr1[k]}
    float cthr2[kMaxThr];   // attitude R2 index = #{k : C2*(c - m) >= cthr2[k]}
    int r1_mulW, r1_mulA, r2_mulW, r2_mulA, P, num_r1;
    int compat;             // R1 min corners decoded as initializeRegions_kernel does (w fastest)
    float cmin_tab[kMaxThr + 1];  // (float)(C_MIN + i * C_R1_SIZE), evaluated in double
    uint32_t r2_words;      // ceil(num_r1 * P / 32)
    // spatial hash (spatialHash.cuh:9-13)
    float cell;
    int gdim;
    // planner
    float goal_thresh, eps, vol;
    uint32_t cap, budget, per_entry, root_repeat, sparse_repeat;
    int sparse_thr;
    uint32_t seed_lo, seed_hi;
    // goal-progress pruning (PruneKPAX)
    int prune;
    float prune_goal_bias, prune_expl_bias, prune_scale;
};

// Derive parameters; returns KPAX_OK or KPAX_EINVAL with a message in kpax_last_error().
kpax_status derive_params(const kpax_config& cfg, KParams* out);
void set_error(const char* fmt, ...);

}  // namespace kpax

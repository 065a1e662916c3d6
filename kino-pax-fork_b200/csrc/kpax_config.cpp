// kpax_config.cpp — runtime configuration: presets, validation and derived launch parameters.
//
// The reference fixes all of this at compile time in include/config/config.h; a preset here
// fills the same quantities for one benchmark configuration.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <limits>

#include "kpax_params.h"

namespace kpax {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

static int ipow(int b, int e)
{
    int r = 1;
    while(e-- > 0) r *= b;
    return r;
}

// Total order on floats as unsigned keys (finite values only are searched).
static uint32_t fkey(float f)
{
    uint32_t b;
    memcpy(&b, &f, 4);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
static float kfloat(uint32_t k)
{
    uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

static int d2i_sat(double x)
{
    if(x != x) return 0;
    if(x >= 2147483648.0) return 2147483647;
    if(x <= -2147483648.0) return -2147483647 - 1;
    return (int)x;
}

// Smallest float x with idx(x) >= k for a non-decreasing idx; +inf if none.
template <class F>
static float threshold(F idx, int k)
{
    uint32_t lo = fkey(-std::numeric_limits<float>::max()), hi = fkey(std::numeric_limits<float>::max());
    if(idx(kfloat(hi)) < k) return INFINITY;
    if(idx(kfloat(lo)) >= k) return -INFINITY;
    while(hi - lo > 1) {  // invariant: idx(lo) < k <= idx(hi)
        uint32_t mid = lo + (hi - lo) / 2;
        if(idx(kfloat(mid)) >= k) hi = mid;
        else lo = mid;
    }
    return kfloat(hi);
}

static float ceil_to_float(double d)
{
    float f = (float)d;
    if((double)f < d) f = nextafterf(f, INFINITY);
    return f;
}
static float floor_to_float(double d)
{
    float f = (float)d;
    if((double)f > d) f = nextafterf(f, -INFINITY);
    return f;
}

kpax_status derive_params(const kpax_config& c, KParams* p)
{
    kpax_status st = kpax_config_validate(&c);
    if(st != KPAX_OK) return st;
    memset(p, 0, sizeof(*p));
    p->model = c.model;
    p->sd = c.state_dim;
    p->cd = c.control_dim;
    p->S = c.state_dim + c.control_dim + 1;
    p->h = c.step_size;
    p->hh = 0.5f * c.step_size;
    p->h6 = c.step_size / 6.0f;
    p->nsteps = c.max_propagation_duration;
    p->fixed_steps = c.fixed_steps ? 1 : 0;
    if(c.model == KPAX_MODEL_QUADROTOR) {  // statePropagatorSpatialHash.cu:275
        p->ws_lo = c.w_min, p->ws_hi = c.w_max;
    } else {  // :107, :193 compare against 0 and W_SIZE
        p->ws_lo = 0.0f, p->ws_hi = c.w_size;
    }
    p->vmin = c.v_min, p->vmax = c.v_max;
    p->pitch_lo = ceil_to_float(c.pitch_min);
    p->pitch_hi = floor_to_float(c.pitch_max);
    for(int i = 0; i < 4; ++i) {
        p->clo[i] = c.ctrl_min[i];
        p->crng[i] = c.ctrl_max[i] - c.ctrl_min[i];
    }
    p->W1 = c.w_r1_length, p->C1 = c.c_r1_length, p->V1 = c.v_r1_length;
    p->W2 = c.w_r2_length, p->C2 = c.c_r2_length, p->V2 = c.v_r2_length;
    p->cdim = c.c_dim, p->vdim = c.v_dim;
    p->w_only = (c.v_dim == 1 && c.c_dim == 1);  // Graph.cu:115-118
    p->wmin = c.w_min, p->wspan = c.w_max - c.w_min;
    p->vmin_r = c.v_min, p->vspan = c.v_max - c.v_min;
    p->w1size = (c.w_max - c.w_min) / c.w_r1_length;
    p->v1size = (c.v_max - c.v_min) / c.v_r1_length;
    const double cmin = c.c_min, cspan = c.c_max - c.c_min, c1size = (c.c_max - c.c_min) / c.c_r1_length;
    for(int k = 1; k < p->C1; ++k) {  // Graph.cu:127
        const int L = p->C1;
        p->cthr1[k - 1] = threshold(
          [&](float x) {
              int i = d2i_sat((double)L * ((double)x - cmin) / cspan);
              return i < 0 ? 0 : (i > L - 1 ? L - 1 : i);
          },
          k);
    }
    for(int k = 1; k < p->C2; ++k) {  // Graph.cu:179: t = C_R2_LENGTH * (x - min) (float), t / C_R1_SIZE (double)
        const int L = p->C2;
        p->cthr2[k - 1] = threshold(
          [&](float t) {
              int i = d2i_sat((double)t / c1size);
              return i < 0 ? 0 : (i > L - 1 ? L - 1 : i);
          },
          k);
    }
    p->r1_mulA = ipow(c.v_r1_length, c.v_dim);
    p->r1_mulW = ipow(c.c_r1_length, c.c_dim) * p->r1_mulA;
    p->r2_mulA = ipow(c.v_r2_length, c.v_dim);
    p->r2_mulW = ipow(c.c_r2_length, c.c_dim) * p->r2_mulA;
    p->P = ipow(c.w_r2_length, 3) * p->r2_mulW;
    p->num_r1 = ipow(c.w_r1_length, 3) * p->r1_mulW;
    p->compat = c.region_compat ? 1 : 0;
    for(int i = 0; i < c.c_r1_length; ++i) p->cmin_tab[i] = (float)(c.c_min + i * c1size);  // Graph.cu:82
    p->r2_words = (uint32_t)(((uint64_t)p->num_r1 * (uint64_t)p->P + 31) / 32);
    p->cell = c.hash_cell_size;
    p->gdim = (int)((c.w_max - c.w_min) / c.hash_cell_size) + 1;  // spatialHash.cuh:10
    p->goal_thresh = c.goal_thresh;
    p->eps = c.epsilon;
    p->vol = p->w1size * p->w1size * p->w1size;  // W_R1_VOL
    p->cap = c.max_tree_size;
    p->budget = c.expansions_per_iter;
    p->per_entry = c.children_per_entry;
    p->root_repeat = c.root_repeat;
    p->sparse_repeat = c.sparse_repeat;
    p->sparse_thr = c.sparse_valid_threshold;
    p->seed_lo = (uint32_t)c.seed;
    p->prune = c.prune ? 1 : 0;
    p->prune_goal_bias = c.prune_goal_bias, p->prune_expl_bias = c.prune_exploration_bias;
    p->prune_scale = c.prune_progress_scale;
    p->seed_hi = (uint32_t)(c.seed >> 32);
    return KPAX_OK;
}

}  // namespace kpax

using namespace kpax;

extern "C" {

const char* kpax_last_error(void) { return g_err; }
int32_t kpax_abi_version(void) { return KPAX_ABI_VERSION; }

kpax_status kpax_config_preset(int32_t preset, kpax_config* o)
{
    if(!o) return set_error("kpax_config_preset: null output"), KPAX_EINVAL;
    memset(o, 0, sizeof(*o));
    // shared defaults (config.h:211-263, spatialHash.cuh:9, KPAX.cu:31, 77, 476-479)
    o->max_tree_size = 1u << 20;
    o->max_iter = 300;
    o->goal_thresh = 5.0f;
    o->w_min = 0.0f, o->w_max = 100.0f, o->w_size = 100.0f;
    o->c_min = -M_PI, o->c_max = M_PI;
    o->pitch_min = -M_PI / 3, o->pitch_max = M_PI / 3;
    o->w_r1_length = 8, o->w_r2_length = 2;
    o->region_compat = 1;
    o->epsilon = 1e-2f;
    o->hash_cell_size = 5.0f;
    o->children_per_entry = 32;
    o->root_repeat = 5;
    o->sparse_repeat = 15;
    o->sparse_valid_threshold = 10;
    o->seed = 0x4B504158ull;  // "KPAX"
    o->prune = 0;  // PruneKPAX's defaults (PruneKPAX.cu:34-36) for when it is switched on
    o->prune_goal_bias = 0.7f, o->prune_exploration_bias = 0.3f, o->prune_progress_scale = 10.0f;
    switch(preset) {
        case KPAX_PRESET_DI:  // 6D double integrator: h 0.1, U{1..10} steps, |v|<=1, a in [-1,1]^3
            o->model = KPAX_MODEL_DOUBLE_INTEGRATOR;
            o->state_dim = 6, o->control_dim = 3;
            o->step_size = 0.1f, o->max_propagation_duration = 10, o->fixed_steps = 0;
            o->v_min = -1.0f, o->v_max = 1.0f;
            for(int i = 0; i < 3; ++i) o->ctrl_min[i] = -1.0f, o->ctrl_max[i] = 1.0f;
            o->c_dim = 0, o->v_dim = 3;
            o->c_r1_length = 1, o->v_r1_length = 1, o->c_r2_length = 1, o->v_r2_length = 1;
            o->expansions_per_iter = 1u << 14;
            break;
        case KPAX_PRESET_DUBINS:  // Dubins airplane: h 0.05, 20 steps, v in [0.5,2], a in [-1,1], rates in [-0.5,0.5]
            o->model = KPAX_MODEL_DUBINS_AIRPLANE;
            o->state_dim = 6, o->control_dim = 3;
            o->step_size = 0.05f, o->max_propagation_duration = 20, o->fixed_steps = 1;
            o->v_min = 0.5f, o->v_max = 2.0f;
            o->ctrl_min[0] = -1.0f, o->ctrl_max[0] = 1.0f;  // a
            o->ctrl_min[1] = -0.5f, o->ctrl_max[1] = 0.5f;  // yaw rate
            o->ctrl_min[2] = -0.5f, o->ctrl_max[2] = 0.5f;  // pitch rate
            o->c_dim = 2, o->v_dim = 1;
            o->c_r1_length = 8, o->v_r1_length = 1, o->c_r2_length = 3, o->v_r2_length = 1;
            o->expansions_per_iter = 1u << 16;
            break;
        case KPAX_PRESET_QUAD:  // 12D quadrotor: h 0.02, 25 steps, Zc in [0,2g], torques in [-0.1,0.1]
        case KPAX_PRESET_QUAD_REF:
            o->model = KPAX_MODEL_QUADROTOR;
            o->state_dim = 12, o->control_dim = 4;
            o->v_min = -30.0f, o->v_max = 30.0f;
            o->c_dim = 3, o->v_dim = 3;
            o->c_r1_length = 2, o->v_r1_length = 2, o->c_r2_length = 1, o->v_r2_length = 2;
            if(preset == KPAX_PRESET_QUAD) {
                o->step_size = 0.02f, o->max_propagation_duration = 25, o->fixed_steps = 1;
                o->ctrl_min[0] = 0.0f, o->ctrl_max[0] = 19.62f;
                for(int i = 1; i < 4; ++i) o->ctrl_min[i] = -0.1f, o->ctrl_max[i] = 0.1f;
                o->expansions_per_iter = 1u << 16;
            } else {  // config.h:211-215, 284-291 (torque ranges +-pi rounded to float)
                o->max_tree_size = 400000;
                o->step_size = 0.1f, o->max_propagation_duration = 10, o->fixed_steps = 0;
                o->ctrl_min[0] = 0.0f, o->ctrl_max[0] = 30.0f;
                for(int i = 1; i < 4; ++i) o->ctrl_min[i] = (float)-M_PI, o->ctrl_max[i] = (float)M_PI;
                o->expansions_per_iter = o->max_tree_size;
            }
            break;
        default: return set_error("kpax_config_preset: unknown preset %d", preset), KPAX_EINVAL;
    }
    return KPAX_OK;
}

kpax_status kpax_config_validate(const kpax_config* c)
{
#define KPAX_REQ(cond, ...)                  \
    do {                                     \
        if(!(cond)) {                        \
            set_error(__VA_ARGS__);          \
            return KPAX_EINVAL;              \
        }                                    \
    } while(0)
    KPAX_REQ(c, "null config");
    KPAX_REQ(c->model >= 1 && c->model <= 3, "model %d not in {1,2,3}", c->model);
    const int sd = c->model == KPAX_MODEL_QUADROTOR ? 12 : 6, cd = c->model == KPAX_MODEL_QUADROTOR ? 4 : 3;
    KPAX_REQ(c->state_dim == sd && c->control_dim == cd, "state/control dims %d/%d do not match model %d",
             c->state_dim, c->control_dim, c->model);
    KPAX_REQ(c->max_tree_size >= 2 && c->max_tree_size <= (1u << 28), "max_tree_size %u out of [2, 2^28]",
             c->max_tree_size);
    KPAX_REQ(c->max_iter >= 1, "max_iter must be >= 1");
    KPAX_REQ(c->step_size > 0.0f && isfinite(c->step_size), "step_size must be positive");
    KPAX_REQ(c->max_propagation_duration >= 1 && c->max_propagation_duration <= 100000, "bad max_propagation_duration");
    KPAX_REQ(c->w_max > c->w_min && isfinite(c->w_max) && isfinite(c->w_min), "bad workspace bounds");
    KPAX_REQ(c->v_max > c->v_min, "bad velocity bounds");
    KPAX_REQ(c->c_max > c->c_min, "bad attitude bounds");
    for(int i = 0; i < cd; ++i)
        KPAX_REQ(isfinite(c->ctrl_min[i]) && isfinite(c->ctrl_max[i]) && c->ctrl_max[i] >= c->ctrl_min[i],
                 "bad control range %d", i);
    KPAX_REQ(c->c_dim >= 0 && c->v_dim >= 0 && c->c_dim <= 8 && c->v_dim <= 8 && 3 + c->c_dim + c->v_dim <= sd, "region dims 3+%d+%d exceed state dim %d",
             c->c_dim, c->v_dim, sd);
    KPAX_REQ(c->w_r1_length >= 1 && c->w_r1_length <= 64 && c->w_r2_length >= 1 && c->w_r2_length <= 64, "bad W lengths");
    KPAX_REQ(c->c_r1_length >= 1 && c->c_r1_length <= kMaxThr + 1 && c->c_r2_length >= 1 && c->c_r2_length <= kMaxThr + 1,
             "C lengths must be in [1,16]");
    KPAX_REQ(c->v_r1_length >= 1 && c->v_r1_length <= 64 && c->v_r2_length >= 1 && c->v_r2_length <= 64, "bad V lengths");
    double n1 = pow(c->w_r1_length, 3) * pow(c->c_r1_length, c->c_dim) * pow(c->v_r1_length, c->v_dim);
    double p = pow(c->w_r2_length, 3) * pow(c->c_r2_length, c->c_dim) * pow(c->v_r2_length, c->v_dim);
    KPAX_REQ(n1 <= (double)(1 << 24), "too many R1 regions (%.0f)", n1);
    KPAX_REQ(n1 * p <= 2147483647.0, "too many R2 regions (%.0f)", n1 * p);
    KPAX_REQ(c->hash_cell_size > 0.0f && isfinite(c->hash_cell_size), "bad hash_cell_size");
    double g = floor((c->w_max - c->w_min) / c->hash_cell_size) + 1;
    KPAX_REQ(g <= 1024 && g * g * g <= (double)(1 << 26), "hash grid too fine (%.0f cells per axis)", g);
    KPAX_REQ(c->expansions_per_iter >= 1 && c->expansions_per_iter <= (1u << 26), "bad expansions_per_iter");
    KPAX_REQ(c->children_per_entry >= 1 && c->children_per_entry <= 1024, "bad children_per_entry");
    KPAX_REQ(c->root_repeat >= 1 && c->root_repeat <= 254, "root_repeat in [1,254]");
    KPAX_REQ(c->sparse_repeat >= 1 && c->sparse_repeat <= 254, "sparse_repeat in [1,254]");
    KPAX_REQ(c->epsilon > 0.0f, "epsilon must be positive");
    KPAX_REQ(c->block_size == 0 || c->block_size == 128 || c->block_size == 256 || c->block_size == 448 ||
               c->block_size == 512,
             "block_size must be 0 (default), 128, 256, 448 or 512");
    KPAX_REQ(c->samples_per_thread >= 0 && c->samples_per_thread <= 8, "samples_per_thread in [0,8]");
    KPAX_REQ(!c->prune || (c->prune_progress_scale > 0.0f && isfinite(c->prune_progress_scale) &&
                           isfinite(c->prune_goal_bias) && isfinite(c->prune_exploration_bias)),
             "pruning needs a positive progress scale and finite biases");
    KPAX_REQ(c->unroll_iters >= 0 && c->unroll_iters <= 64, "unroll_iters in [0,64]");
    KPAX_REQ(c->iteration_kernels == 0 || c->iteration_kernels == 1, "iteration_kernels must be 0 or 1");
#undef KPAX_REQ
    return KPAX_OK;
}

kpax_status kpax_config_sizes(const kpax_config* cfg, uint32_t* num_r1, uint32_t* r2_per_r1, uint32_t* sample_dim)
{
    KParams p;
    kpax_status st = derive_params(*cfg, &p);
    if(st != KPAX_OK) return st;
    if(num_r1) *num_r1 = (uint32_t)p.num_r1;
    if(r2_per_r1) *r2_per_r1 = (uint32_t)p.P;
    if(sample_dim) *sample_dim = (uint32_t)p.S;
    return KPAX_OK;
}

}  // extern "C"

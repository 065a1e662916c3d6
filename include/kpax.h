/*
 * kpax.h — C ABI of the B200-native Kino-PAX tree-expansion library (libkpax.so).
 *
 * The reference planner is a C++ class whose configuration is compile-time macros
 * (include/config/config.h) and whose entry point is
 *     void KPAX::plan(float* h_initial, float* h_goal, float* d_obstacles_ptr,
 *                     uint h_obstaclesCount, bool saveTree)          (src/planners/KPAX.cu:51)
 * This header replaces it with plain-C calls: a runtime configuration struct that carries
 * every macro the hot path reads, an opaque planner handle owning the device buffers, and
 * the same plan(init, goal, device obstacles) entry.  Kernel-level entry points expose the
 * individual stages (propagation, collision, region index) for parity tests and the
 * propagation micro-benchmark.
 *
 * Conventions
 *  - Every call returns kpax_status; nothing calls exit() or traps on the device.
 *  - Pointers named d_* are device pointers (cudaMalloc'd by the caller), h_* are host.
 *  - Rows use the reference's sample layout [state | control | duration] with
 *    SAMPLE_DIM = STATE_DIM + CONTROL_DIM + 1 floats (config.h:221).
 *  - Obstacles are n x 6 floats [min x,y,z, max x,y,z] (helper.cu:13-39 CSV layout).
 *  - `stream` arguments are cudaStream_t passed as void* (0 = legacy default stream).
 */
#ifndef KPAX_H_
#define KPAX_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KPAX_ABI_VERSION 3

typedef enum kpax_status {
    KPAX_OK = 0,
    KPAX_EINVAL = 1,     /* bad argument or configuration */
    KPAX_ENOMEM = 2,     /* device or host allocation failed */
    KPAX_ECUDA = 3,      /* a CUDA runtime call failed (kpax_last_error() has the text) */
    KPAX_ETIMEOUT = 4,   /* a bounded device-side wait gave up; results are incomplete */
    KPAX_ECAPACITY = 5,  /* a fixed-size buffer (tree, frontier, path) would overflow */
    KPAX_ENOTFOUND = 6   /* plan finished without reaching the goal (not an error for kpax_plan) */
} kpax_status;

/* Dynamics model ids follow the reference's MODEL macro (config.h:209). */
typedef enum kpax_model {
    KPAX_MODEL_DOUBLE_INTEGRATOR = 1, /* 6D (x,y,z,vx,vy,vz), ctrl (ax,ay,az) */
    KPAX_MODEL_DUBINS_AIRPLANE = 2,   /* 6D (x,y,z,yaw,pitch,v), ctrl stored (yawRate,pitchRate,a) */
    KPAX_MODEL_QUADROTOR = 3          /* 12D (x,y,z,phi,theta,psi,u,v,w,p,q,r), ctrl (Zc,Lc,Mc,Nc) */
} kpax_model;

/* Presets for the benchmark configurations (seeded synthetic environments). */
typedef enum kpax_preset_id {
    KPAX_PRESET_DI = 0,       /* 6D double integrator, h 0.1, steps U{1..10}, R1 8^3, R2 2^3 */
    KPAX_PRESET_DUBINS = 1,   /* Dubins airplane, h 0.05, 20 fixed steps, v in [0.5,2] */
    KPAX_PRESET_QUAD = 2,     /* 12D quadrotor, h 0.02, 25 fixed steps, Zc in [0,2g], torques +-0.1 */
    KPAX_PRESET_QUAD_REF = 3  /* 12D quadrotor exactly as the reference's active block (config.h:209-308) */
} kpax_preset_id;

/*
 * Runtime replacement for the reference's compile-time macros.  Field comments give the macro
 * each one stands for.  kpax_config_preset() fills every field; callers then edit what they need.
 */
typedef struct kpax_config {
    int32_t model;                  /* MODEL */
    int32_t state_dim;              /* STATE_DIM (derived from model; checked) */
    int32_t control_dim;            /* CONTROL_DIM (derived from model; checked) */
    uint32_t max_tree_size;         /* MAX_TREE_SIZE */
    uint32_t max_iter;              /* MAX_ITER */
    float step_size;                /* STEP_SIZE (RK4 step, seconds) */
    int32_t max_propagation_duration; /* MAX_PROPAGATION_DURATION (steps) */
    int32_t fixed_steps;            /* 0: steps = 1 + (int)(u*N) like the reference; 1: always N */
    float goal_thresh;              /* GOAL_THRESH */
    float w_min, w_max, w_size;     /* W_MIN, W_MAX, W_SIZE */
    double c_min, c_max;            /* C_MIN, C_MAX (double literals +-M_PI in the reference) */
    float v_min, v_max;             /* V_MIN, V_MAX */
    float ctrl_min[4], ctrl_max[4]; /* control ranges in the reference's draw order:
                                       DI (A_MIN..A_MAX)x3; Dubins (a, yawRate, pitchRate);
                                       quad (Zc, Lc, Mc, Nc) */
    double pitch_min, pitch_max;    /* DUBINS_AIRPLANE_MIN/MAX_PITCH (double in the reference) */
    int32_t c_dim, v_dim;           /* C_DIM, V_DIM (region split dims; W_DIM is always 3) */
    int32_t w_r1_length, c_r1_length, v_r1_length; /* W/C/V_R1_LENGTH */
    int32_t w_r2_length, c_r2_length, v_r2_length; /* W/C/V_R2_LENGTH */
    int32_t region_compat;          /* 1: R2 min-corner table in the reference's order
                                       (Graph.cu:53-97, bit-exact R2 ids); 0: intended order */
    float epsilon;                  /* EPSILON (score floor) */
    float hash_cell_size;           /* GRID_CELL_SIZE (spatialHash.cuh:9) */
    uint32_t expansions_per_iter;   /* children budget per iteration */
    uint32_t children_per_entry;    /* children per frontier entry (reference: 32, KPAX.cu:31) */
    uint32_t root_repeat;           /* repeat count of the root (reference: 5, KPAX.cu:77) */
    uint32_t sparse_repeat;         /* repeat of a new node in a sparse region (15, KPAX.cu:477) */
    int32_t sparse_valid_threshold; /* region is sparse if valid count < this (10, KPAX.cu:476) */
    uint64_t seed;                  /* Philox4x32-10 key (the reference seeds cuRAND from the clock) */
    int32_t block_size;             /* threads per CTA of the expansion kernel: 0 (= 448), 128, 256, 448, 512 */
    int32_t unroll_iters;           /* planner iterations per captured CUDA graph (0 = default) */
    int32_t samples_per_thread;     /* children per expansion thread, 0 (= 1) .. 8 (grid-stride rounds) */
    /* PruneKPAX goal-progress pruning (PruneKPAX.cu:466-498): an accepted child is kept with
     * probability clamp(exploration_bias + goal_bias * clamp(progress / progress_scale + 1/2, 0, 1),
     * EPSILON, 1), progress = parent's distance to the goal - child's.  0 = off (KPAX). */
    int32_t prune;
    float prune_goal_bias;          /* h_goalBias_ (0.7, PruneKPAX.cu:36) */
    float prune_exploration_bias;   /* h_explorationBias_ (0.3, PruneKPAX.cu:35) */
    float prune_progress_scale;     /* h_progressScale_ (10, PruneKPAX.cu:34) */
    /* 0: a single plan runs each iteration as one persistent launch (frontier passes, expansion
     * and scores separated by bounded grid-wide barriers), or with the learned proposal as two such
     * launches around the tensor-core pass; 1: one launch per stage.  Batches always run their own
     * persistent stages.  Plans are identical either way. */
    int32_t iteration_kernels;
    int32_t reserved[2];
} kpax_config;

/* Result of kpax_plan (the reference exposes these as public fields h_pathToGoal_, h_itr_,
 * h_treeSize_, h_controlPathToGoal_; Planner.cuh:31-43). */
typedef struct kpax_result {
    int32_t found;              /* 1 if a tree node reached the goal ball */
    uint32_t goal_idx;          /* tree index of the goal node (0 = none, as h_pathToGoal_) */
    uint32_t path_len;          /* rows in h_path: goal node first, root last */
    uint32_t tree_size;         /* h_treeSize_ */
    uint32_t iters;             /* h_itr_ */
    int32_t tree_full;          /* 1 if the tree reached max_tree_size */
    const float* h_path;        /* planner-owned host rows (SAMPLE_DIM floats each), valid until next call */
    double ms;                  /* device time of the plan (CUDA events) */
    uint64_t expansions;        /* children propagated (sum of the reference's d_counterArray_) */
    uint64_t valid_expansions;  /* valid children (sum of d_validCounterArray_, KPAX.cu:393) */
    double path_cost;           /* sum of segment durations along the path (column SAMPLE_DIM-1) */
} kpax_result;

typedef struct kpax_planner kpax_planner;
typedef struct kpax_env kpax_env;

/* ---- configuration ---------------------------------------------------------------------- */
kpax_status kpax_config_preset(int32_t preset, kpax_config* out);
kpax_status kpax_config_validate(const kpax_config* cfg);
/* Number of R1 regions, R2 regions per R1, and SAMPLE_DIM for a configuration. */
kpax_status kpax_config_sizes(const kpax_config* cfg, uint32_t* num_r1, uint32_t* r2_per_r1,
                              uint32_t* sample_dim);
const char* kpax_last_error(void);
int32_t kpax_abi_version(void);

/* ---- planner (replaces KPAX::KPAX / KPAX::plan, KPAX.cu:5-115) --------------------------- */
kpax_status kpax_create(const kpax_config* cfg, kpax_planner** out);
kpax_status kpax_destroy(kpax_planner* planner);
/* One full plan.  h_init/h_goal: SAMPLE_DIM host floats (only state dims are read; the goal
 * uses x,y,z).  d_obstacles: caller-owned device buffer of n_obs*6 floats.  Returns KPAX_OK
 * whether or not the goal was reached (see out->found). */
kpax_status kpax_plan(kpax_planner* planner, const float* h_init, const float* h_goal,
                      const float* d_obstacles, uint32_t n_obs, int32_t save_tree,
                      kpax_result* out);
/* Same, with the obstacles in host memory (copied inside the call). */
kpax_status kpax_plan_host(kpax_planner* planner, const float* h_init, const float* h_goal,
                           const float* h_obstacles, uint32_t n_obs, kpax_result* out);
/* Stepwise planning: begin (reset + obstacle grid), then single iterations that never stop
 * at the goal (used by the throughput benchmark), then a synchronising result read. */
kpax_status kpax_plan_begin(kpax_planner* planner, const float* h_init, const float* h_goal,
                            const float* d_obstacles, uint32_t n_obs);
kpax_status kpax_plan_iterate(kpax_planner* planner, uint32_t n_iters, int32_t stop_at_goal);
kpax_status kpax_plan_result(kpax_planner* planner, kpax_result* out);
/* Per-iteration device times (ms) from CUDA events on the planner stream. */
typedef struct kpax_iter_timing {
    float ms_total, ms_frontier, ms_expand, ms_scores;
} kpax_iter_timing;
/* Benchmark entry: runs n_iters iterations without stopping at the goal.  Each is preceded,
 * outside its timed events, by a write of flush_bytes to a scratch buffer (0 = no flush; more
 * than the 126 MB L2 evicts it).  split = 0 records events around each iteration only (its
 * kernels overlap their launches as in a plan; ms_frontier/ms_expand/ms_scores are 0); split != 0
 * also records them between the kernels, which gives the breakdown but serialises the launches.
 * h_times: n_iters entries (may be NULL); h_totals (may be NULL): children propagated, valid
 * children, RK4 steps executed, nodes appended over the n_iters. */
kpax_status kpax_plan_iterate_timed(kpax_planner* planner, uint32_t n_iters, uint64_t flush_bytes, int32_t split,
                                    kpax_iter_timing* h_times, uint64_t* h_totals);
/* The stream all planner work is issued on (cudaStream_t as void*). */
void* kpax_planner_stream(kpax_planner* planner);

/* Tree export in the reference AoS layout (d_treeSamples_, d_treeSamplesParentIdxs_,
 * d_treeSampleCosts_; Planner.cuh:36-38).  Any output pointer may be NULL. */
kpax_status kpax_export_tree(kpax_planner* planner, float* h_rows, int32_t* h_parents,
                             float* h_costs, uint32_t max_rows, uint32_t* n_rows);
/* Region buffers (graph_.d_counterArray_, d_validCounterArray_, d_vertexScoreArray_ and the
 * R2 activation flags as a bitset of ceil(num_r2/32) words; Graph.cuh:25-29). */
kpax_status kpax_export_regions(kpax_planner* planner, int32_t* h_counter, int32_t* h_valid,
                                float* h_scores, uint32_t* h_r2_bits);
/* Per-node frontier repeat counts (0 = not in the frontier) and R1 ids of the live tree. */
kpax_status kpax_export_frontier(kpax_planner* planner, uint8_t* h_repeat, int32_t* h_r1,
                                 uint32_t max_rows);

/* Debug capture: when enabled, every child of the latest iteration is kept (row, validity,
 * R1, R2, frontier flag, parent) for kpax_export_children. */
kpax_status kpax_debug_capture(kpax_planner* planner, int32_t enable);
kpax_status kpax_export_children(kpax_planner* planner, float* h_rows, uint8_t* h_valid,
                                 int32_t* h_r1, int32_t* h_r2, uint8_t* h_next,
                                 int32_t* h_parent, uint32_t max_rows, uint32_t* n_children);

/* ---- batches of independent queries (no counterpart in the reference, which plans one query
 * per KPAX::plan call with a compile-time model) -------------------------------------------- */
typedef struct kpax_batch kpax_batch;
typedef struct kpax_batch_stats {
    double ms;                  /* device time of the whole batch */
    uint32_t iters;             /* iterations of the longest-running query */
    uint32_t found;             /* queries that reached their goal */
    uint64_t expansions, valid_expansions, steps;
} kpax_batch_stats;
/* One configuration per query (models, trees, budgets may differ).  All queries run every
 * iteration stage in the same kernel launches: blocks index a query table. */
kpax_status kpax_batch_create(const kpax_config* cfgs, uint32_t n, kpax_batch** out);
kpax_status kpax_batch_destroy(kpax_batch* batch);
/* h_inits / h_goals: n rows, row_stride floats apart (>= the largest SAMPLE_DIM).
 * d_obstacles[q]: device buffer of n_obs[q] x 6 floats.  results[q].ms is the device time from
 * the batch's start until query q finished (time to solution when results[q].found);
 * results[q].h_path holds path_len rows of query q's own SAMPLE_DIM.  Every query of one call
 * uses the same plan index in its random stream, so a query reproduces exactly what a single
 * planner's plan with the same configuration and plan count gives. */
kpax_status kpax_batch_plan(kpax_batch* batch, const float* h_inits, const float* h_goals,
                            uint32_t row_stride, const float* const* d_obstacles,
                            const uint32_t* n_obs, kpax_result* results, kpax_batch_stats* stats);

/* ---- obstacle environment: uniform-grid spatial hash (spatialHash.cu:9-67) ------------- */
/* Builds a compressed-sparse-row grid (no per-cell cap, deterministic ascending obstacle
 * order inside a cell) from a device obstacle buffer on `stream`. */
kpax_status kpax_env_create(const kpax_config* cfg, const float* d_obstacles, uint32_t n_obs,
                            void* stream, kpax_env** out);
kpax_status kpax_env_destroy(kpax_env* env);
/* Grid statistics: number of cells and of (cell, obstacle) entries. */
kpax_status kpax_env_stats(kpax_env* env, uint32_t* n_cells, uint32_t* n_entries);

/* ---- kernel-level entry points (device pointers) ---------------------------------------- */
/* Propagate n independent segments (statePropagatorSpatialHash.cu:72-308).
 *  d_parents: n x state_dim floats.
 *  d_draws:   n x 5 uniforms in (0,1] in the reference's draw order (controls..., duration;
 *             3-control models ignore column 3), or NULL to draw from Philox4x32-10 keyed by
 *             (cfg->seed, draw_stream) with counter = segment index.
 *  d_rows:    n x SAMPLE_DIM output rows (state after the last executed step, controls,
 *             duration) exactly as the reference writes x1.
 *  d_valid:   n bytes, 1 = collision free and within bounds.  d_steps (optional): executed steps.
 * Batches of 2^18 segments or more run in rounds of up to 2^24 segments, three phases each, whose
 * survivor lists use scratch held by `env` (about 2 x 4 x (1 + control_dim + state_dim) bytes per
 * segment of a round, plus 4 per segment for drawn durations; kept for later calls and freed by
 * kpax_env_destroy), so calls that share an env must be issued in order on one stream. */
kpax_status kpax_propagate_batch(const kpax_config* cfg, kpax_env* env, const float* d_parents,
                                 const float* d_draws, uint32_t draw_stream, uint32_t n,
                                 float* d_rows, uint8_t* d_valid, int32_t* d_steps, void* stream);
/* Allocation-free variant of kpax_propagate_batch; it has no counterpart in the reference.
 * For callers that must not allocate device memory while they run — a planner inside a robot's
 * real-time control cycle, where cudaMalloc can synchronise the device and take unbounded time,
 * or a host application that hands all device memory to its own pool at start-up.  The obstacle
 * grid is built in a fixed array inside the library (about 2.1 MiB, held by every GPU that loads
 * the library until exit) instead of in memory from cudaMalloc; nothing is allocated or freed.
 * Limits: at most 4096 obstacles, 131072 grid cells and 262144 (cell, obstacle) pairs; larger
 * inputs return KPAX_ECAPACITY with a message.  All calls share that one array and each call
 * overwrites it, so calls whose GPU work overlaps (other streams, other host threads) race; issue
 * them one after another on one stream.  A call with obstacles blocks the calling thread once: it
 * waits for `stream` to finish counting the grid entries and reads the count back to the host, to
 * check it against the limit.  Set-up: the first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and keeps it for the life of the process; do not call the entry
 * on a device again after a cudaDeviceReset of it.  Batches of any size run the one-pass propagation kernel (no phase
 * scratch).  Arguments as kpax_propagate_batch, with the obstacles (n_obs x 6 device floats) in
 * place of an environment. */
kpax_status kpax_propagate_batch_noalloc(const kpax_config* cfg, const float* d_obstacles,
                                         uint32_t n_obs, const float* d_parents,
                                         const float* d_draws, uint32_t draw_stream, uint32_t n,
                                         float* d_rows, uint8_t* d_valid, int32_t* d_steps,
                                         void* stream);
/* Broad-phase check of n boxes against the grid (isMotionValidSpatialHash, spatialHash.cu:145-194).
 * d_bbmin/d_bbmax: n x 3 floats.  d_free: n bytes, 1 = no obstacle overlaps the box. */
kpax_status kpax_collide_batch(kpax_env* env, const float* d_bbmin, const float* d_bbmax,
                               uint32_t n, uint8_t* d_free, void* stream);
/* R1 / R2 region ids of n states (getRegion / getSubRegion, Graph.cu:99-205).
 * d_states: n x state_dim floats; d_r2 may be NULL. */
kpax_status kpax_region_batch(const kpax_config* cfg, const float* d_states, uint32_t n,
                              int32_t* d_r1, int32_t* d_r2, void* stream);
/* Frontier compaction of the planner (the entry list of propagateFrontier / updateFrontier,
 * KPAX.cu:310-351 with Planner.cu:52-80) on a caller's repeat counts, through the planner's own
 * kernels.  Node i owns d_repeat[i] consecutive entries (0 = not in the frontier; 255, the
 * planner's mark for a node added in the last iteration, counts as cfg->sparse_repeat).  With R
 * entries in all and a children budget B, each entry gets k = children_per_entry children, or
 * max(1, B / R) when R k > B, and E = min(R, B / k) entries are taken, evenly spaced over the
 * frontier in node order (entry j is virtual entry floor(j R / E)); d_entries (room for B) receives
 * their E node ids and every node with an entry taken gets repeat 0.  At most 2^24 nodes.  Waits
 * for the stream. */
typedef struct kpax_frontier_stats {
    uint32_t R;  /* entries in the frontier */
    uint32_t k;  /* children per entry taken */
    uint32_t E;  /* entries taken */
    uint32_t n;  /* children: E * k */
} kpax_frontier_stats;
kpax_status kpax_frontier_compact(const kpax_config* cfg, uint8_t* d_repeat, uint32_t n_nodes,
                                  uint32_t budget, uint32_t* d_entries, kpax_frontier_stats* out,
                                  void* stream);
/* Test hook of the bounded device waits: one warp runs the expansion's look-back wait
 * (tile 1 waiting for tile 0, which nothing publishes) with a limit of spin_limit polls
 * (1 .. 2^22); it gives up, the kernel stores a timeout status and returns, and the call returns
 * KPAX_ETIMEOUT with *h_status = 1.  The context stays usable. */
kpax_status kpax_test_wait_timeout(uint32_t spin_limit, uint32_t* h_status, void* stream);
/* Test hook: for each x, writes (sin, cos) of the propagation kernels' sine/cosine and
 * (sin, cos) of CUDA's sincosf, 4 floats per input, so tests can bound their difference. */
kpax_status kpax_test_sincos(const float* d_x, uint32_t n, float* d_out, void* stream);
/* FP32 issue rate of this GPU: an FMA-chain kernel (8 independent chains per thread, 2048 threads
 * per SM, iters FMAs per chain) timed with CUDA events on `stream` after one warm-up launch;
 * *h_tflops = 16 x iters x threads / time.  The denominator of the propagation roofline. */
kpax_status kpax_fp32_peak(uint32_t iters, double* h_tflops, double* h_ms, void* stream);
/* Number of propagation kernels (and other library kernels) launched since load; the
 * benchmark reports it as evidence that the device path ran. */
uint64_t kpax_kernel_launches(void);

/* ---- ReKinoLite (src/ReKino/ReKinoLite.cu, include/ReKino/ReKinoLite.cuh) ----------------
 * The fork's warp-greedy planner on the same propagation and collision code: every warp extends
 * one path by the valid sample closest to the goal among samples_per_thread x 32 propagated from
 * its last node (a random valid one with probability epsilon_greedy), backing up 1-5 nodes when
 * none is valid, up to 200 nodes.  The result's goal_idx is the winning warp (the earliest
 * iteration, then the lowest warp id), iters its iteration + 1, path_len / h_path its path (goal
 * first), expansions / valid_expansions the samples propagated by all warps. */
typedef struct kpax_rekino_params {
    uint32_t num_warps;          /* h_numWarps_ (512, ReKinoLite.cu:11) */
    uint32_t samples_per_thread; /* h_samplesPerThread_ (1), at most 16 (512 samples per warp) */
    float epsilon_greedy;        /* h_epsilonGreedy_ (0) */
    uint32_t max_iterations;     /* MAX_ITER_REKINO (20000, config.h:213) */
    double timeout_ms;           /* give-up time (6 s, ReKinoLite.cu:120-122) */
    uint32_t reserved[4];
} kpax_rekino_params;
typedef struct kpax_rekino kpax_rekino;
kpax_status kpax_rekino_defaults(kpax_rekino_params* out);
kpax_status kpax_rekino_create(const kpax_config* cfg, const kpax_rekino_params* params, kpax_rekino** out);
kpax_status kpax_rekino_destroy(kpax_rekino* planner);
/* One plan: h_init / h_goal SAMPLE_DIM host floats, d_obstacles n_obs x 6 device floats. */
kpax_status kpax_rekino_plan(kpax_rekino* planner, const float* h_init, const float* h_goal,
                             const float* d_obstacles, uint32_t n_obs, kpax_result* out);

/* ---- environment input (readObstaclesFromCSV, helper.cu:13-39) ----------------------------
 * Every float of the file, read as the reference reads it: line by line, a float taken off the
 * line by stream extraction and one comma skipped after it; the first token that does not read as
 * a float ends its line.  Up to `capacity` floats go to h_values (NULL to count only) and the number
 * read to *n_values; the obstacles are the first n_values / 6 rows (the reference's numObstacles,
 * workspaceDim 3; a trailing partial row is read but is not an obstacle).  KPAX_EINVAL when the
 * file cannot be opened, where the reference exits the process. */
kpax_status kpax_read_obstacles_csv(const char* filename, float* h_values, uint64_t capacity, uint64_t* n_values);

/* ---- solution output (copyAndWriteVectorToCSV / writeVectorToCSV, helper.cuh:56-93) ------
 * Rows of `cols` floats as CSV, each value printed "%.6f" (std::fixed, setprecision 6) and
 * separated by commas, one row per line; append = 1 appends as the reference's append mode. */
kpax_status kpax_write_rows_csv(const float* h_rows, uint32_t rows, uint32_t cols,
                                const char* filename, int32_t append);
/* The last plan's solution (KPAX.cu:621-627, controlPathToGoal.csv): SAMPLE_DIM columns, the goal
 * node first and the root last (every row; the reference copies h_itr_ rows, which can drop the root).  No file
 * content is written when no path was found (an empty file unless appending). */
kpax_status kpax_write_solution_csv(kpax_planner* planner, const char* filename, int32_t append);
/* planBench (KPAX.cu:243-300) with the reference's per-iteration dumps (writeDeviceVectorsToCSV,
 * KPAX.cu:545-633, and writeExecutionTimeToCSV, 635-643): plans like kpax_plan, one iteration at a
 * time, and after each iteration writes under out_dir/Data/<Name>/<Name><bench_itr>/ the tree rows
 * (samples<itr>.csv: MAX_TREE_SIZE rows of SAMPLE_DIM, unused rows 0), parents (parents<itr>.csv,
 * unused -1), one row per iteration of the region counters, valid counters, frontier flags,
 * frontier repeat counts and region scores, one value per iteration of the frontier size, tree
 * size and children expanded, the solution rows when found (controlPathToGoal.csv), and the
 * run's seconds to Data/ExecutionTime/executionTime.csv.  A run's files start fresh at its first
 * iteration (the reference appends to whatever a previous run left).  Debug output: every
 * iteration copies the whole tree to the host. */
kpax_status kpax_plan_bench(kpax_planner* planner, const float* h_init, const float* h_goal,
                            const float* d_obstacles, uint32_t n_obs, int32_t bench_itr,
                            const char* out_dir, kpax_result* out);

/* ---- learned proposal (no counterpart in the reference) ----------------------------------
 * The reference draws every control and duration uniformly (statePropagatorSpatialHash.cu,
 * propagateAndCheck).  A proposal network reshapes those draws for the quadrotor: an MLP
 * 51 -> 256 -> 256 -> 88 (SiLU) maps (state, goal - state, occupancy of the 3x3x3 R1 workspace
 * cells around the state) to an 8-component Gaussian mixture over the logits of the five draw
 * uniforms (4 controls, duration).  A fraction epsilon of the draws stays uniform and every
 * segment is still propagated and collision-checked exactly.
 * Layouts: features n x 64 floats (51 used), network outputs n x 96 floats (88 used), mixture
 * records n x 88 floats (the outputs with biases: component k's logit at 11k, its 5 means at
 * 11k+1.., its 5 raw log-sigmas at 11k+6.., sigma = exp(-2 + 5 tanh(raw / 5))), logit targets
 * n x 5. */
typedef struct kpax_mlp kpax_mlp;
#define KPAX_MLP_FEATURES 64
#define KPAX_MLP_OUTPUTS 96
#define KPAX_MLP_MIX 88
#define KPAX_MLP_HIDDEN 256

/* A network with buffers for training batches of up to max_batch rows; parameters start at 0. */
kpax_status kpax_mlp_create(uint32_t max_batch, kpax_mlp** out);
kpax_status kpax_mlp_destroy(kpax_mlp* net);
/* Number of FP32 parameters (W1[256][64], b1, W2[256][256], b2, W3[96][256], b3). */
uint32_t kpax_mlp_num_params(void);
/* Sets the FP32 parameters, clears the Adam state and packs the BF16 inference image. */
kpax_status kpax_mlp_set_params(kpax_mlp* net, const float* h_params, void* stream);
kpax_status kpax_mlp_get_params(kpax_mlp* net, float* h_params, void* stream);
/* Weights of the five target dimensions in the loss (default 1; 0 drops a dimension, e.g. the
 * duration of fixed-step models). */
kpax_status kpax_mlp_set_loss_mask(kpax_mlp* net, const float* h_mask5, void* stream);
/* Re-packs the BF16 inference image from the FP32 parameters (after training). */
kpax_status kpax_mlp_pack(kpax_mlp* net, void* stream);
/* FP32 forward pass (training kernels): d_x n x 64 -> d_out n x 96. */
kpax_status kpax_mlp_forward(kpax_mlp* net, const float* d_x, uint32_t n, float* d_out, void* stream);
/* Mean loss (h_loss, synchronises) and its gradient (d_grad, num_params floats; may be NULL)
 * of n rows of features d_x and logit targets d_y. */
kpax_status kpax_mlp_loss_grad(kpax_mlp* net, const float* d_x, const float* d_y, uint32_t n,
                               float* h_loss, float* d_grad, void* stream);
/* One Adam step (beta 0.9/0.999, eps 1e-8) on the rows d_idx[0..batch) of (d_x, d_y).
 * h_loss (may be NULL: no synchronisation) receives the batch's mean loss. */
kpax_status kpax_mlp_train_step(kpax_mlp* net, const float* d_x, const float* d_y,
                                const uint32_t* d_idx, uint32_t batch, float lr, float* h_loss,
                                void* stream);
/* Adam moments (num_params floats each, may be NULL) and step count. */
kpax_status kpax_mlp_adam_state(kpax_mlp* net, float* h_m, float* h_v, uint64_t* step,
                                void* stream);
/* Occupancy bits of the env's R1 workspace cells (W1^3 bits, cell (x,y,z) at bit
 * (z*W1 + y)*W1 + x): blocked when >= 32 of a 4x4x4 point lattice lie inside obstacles. */
kpax_status kpax_env_occupancy(kpax_env* env, uint32_t* d_words, void* stream);
/* Features of n states (row stride `stride` floats) with goals d_goals (n x 3). */
kpax_status kpax_mlp_features(kpax_env* env, const float* d_states, uint32_t stride,
                              const float* d_goals, uint32_t n, float* d_x, void* stream);
/* Tensor-core (BF16, FP32 accumulate) forward pass of n states to mixture records d_mix.
 * Optional dumps: d_out (n x 96 outputs), d_h1 / d_h2 (n x 256 BF16 hidden activations).
 * Synchronises `stream`; KPAX_ETIMEOUT if a pipeline wait expired. */
kpax_status kpax_mlp_propose(kpax_mlp* net, kpax_env* env, const float* d_states, uint32_t stride,
                             const float* d_goals, uint32_t n, float* d_mix, float* d_out,
                             uint16_t* d_h1, uint16_t* d_h2, void* stream);
/* Device time (CUDA events on `stream`) of the tensor-core kernel of the last kpax_mlp_propose. */
float kpax_mlp_last_propose_ms(const kpax_mlp* net);
/* Turns the learned proposal on (net != NULL) or off for the planner's quadrotor plans.  The
 * packed image is copied, so the network may be trained further or destroyed afterwards. */
kpax_status kpax_set_proposal(kpax_planner* planner, kpax_mlp* net, float epsilon);
/* Mixture records (88 outputs each) of the frontier entries of the last iteration; child c of
 * that iteration drew from record c / k with k = children / entries. */
kpax_status kpax_export_proposal(kpax_planner* planner, float* h_mix, uint32_t max_entries,
                                 uint32_t* n_entries);
/* The same for the quadrotor queries of a batch; enable: one byte per query (NULL = all). */
kpax_status kpax_batch_set_proposal(kpax_batch* batch, kpax_mlp* net, float epsilon,
                                    const uint8_t* enable);

#ifdef __cplusplus
}
#endif

#endif /* KPAX_H_ */

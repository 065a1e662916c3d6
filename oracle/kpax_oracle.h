/*
 * kpax_oracle.h — CPU restatement of the Kino-PAX tree-expansion iteration.
 *
 * TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load liboracle.so, and only as the checker or the timed CPU baseline; the library in
 * kino-pax-fork_b200/ never calls it.
 *
 * Pinning: the FP32 propagation, collision and region functions are checked bit-exactly
 * against the reference's own routines compiled for the host (oracle/_ref, built from
 * src/statePropagator/*.cu, src/collisionCheck/*.cu, spatialHash.cu:145-194 and
 * Graph.cu:99-205 by oracle/Makefile) and against the golden vectors in tests/golden/.
 * The reference has no tests or known-answer vectors of its own.
 *
 * Semantics that the reference leaves undefined are fixed here and followed by the CUDA path:
 *  - random numbers: Philox4x32-10 (Salmon et al., SC'11), u = ((x >> 8) + 1) * 2^-24 in (0,1];
 *  - float->int conversion saturates and maps NaN to 0 (the reference's device behaviour);
 *  - a state with a non-finite component after a step ends the segment as invalid (the
 *    reference's NaN comparisons let it pass);
 *  - R2 "first visit" tests read a snapshot taken at the start of the iteration (the
 *    reference's read-then-exchange is racy);
 *  - the goal node is the lowest tree index that reached the goal ball (the reference's
 *    concurrent path writes race);
 *  - children per iteration are clamped to the budget and to the free tree capacity (the reference
 *    can write past MAX_TREE_SIZE);
 *  - region scores use a fixed-order float sum (the reference's block reductions are
 *    mis-sized and its total is never reset, so its sum is undefined).
 */
#ifndef KPAX_ORACLE_H_
#define KPAX_ORACLE_H_

#include <stdint.h>
#include "kpax.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 block and the (0,1] uniform mapping. */
void ko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float ko_u01(uint32_t x);
/* The six uniforms of one child: [c0 c1 c2 c3 | duration | frontier draw].
 * ctr = {index, iter, 0|1, stream}; key = seed. */
void ko_child_draws(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index, float u[6]);
/* Re-activation draw of tree node `index` in iteration `iter`. */
float ko_reactivate_draw(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index);
float ko_prune_draw(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index);

/* Sizes derived from a configuration (same meaning as kpax_config_sizes). */
int ko_sizes(const kpax_config* cfg, uint32_t* num_r1, uint32_t* r2_per_r1, uint32_t* sample_dim);

/* ---- collision ---- */
typedef struct ko_env ko_env;
ko_env* ko_env_create(const kpax_config* cfg, const float* obs, uint32_t n);
void ko_env_destroy(ko_env* env);
/* CSR grid: cells, entries; copies of the offsets (cells+1) and entries if the pointers are set. */
void ko_env_grid(const ko_env* env, uint32_t* n_cells, uint32_t* n_entries, uint32_t* offsets,
                 uint32_t* entries);
/* 1 = the box overlaps no obstacle (isBroadPhaseValid over the cells of the box). */
int ko_collide_hash(const ko_env* env, const float bbmin[3], const float bbmax[3]);
int ko_collide_brute(const float* obs, uint32_t n, const float bbmin[3], const float bbmax[3]);
/* Signed separation of a box from the nearest obstacle (<= 0: overlap; touching counts as free). */
float ko_separation(const float* obs, uint32_t n, const float bbmin[3], const float bbmax[3]);

/* ---- propagation ---- */
typedef struct ko_seg_diag {
    float margin;       /* smallest |value - bound| over all checks and steps executed */
    int32_t nonfinite;  /* 1 if the segment stopped on a non-finite state */
    int32_t fail_kind;  /* 0 valid, 1 velocity/pitch, 2 workspace, 3 collision, 4 non-finite */
} ko_seg_diag;
/* One segment in FP32 with the reference's operation order.  u: 6 uniforms (see above). */
int ko_propagate(const kpax_config* cfg, const ko_env* env, const float* x0, const float* u,
                 float* row, int32_t* steps_done, ko_seg_diag* diag);
/* Batch: draws (n x 6) or NULL for Philox (ko_child_draws(seed, stream, 0, i)). */
void ko_propagate_batch(const kpax_config* cfg, const ko_env* env, const float* parents,
                        const float* draws, uint32_t stream, uint32_t n, float* rows,
                        uint8_t* valid, int32_t* steps, ko_seg_diag* diag, int nthreads);
/* FP64 integration of the same segment for error reports.  mode 0: the model's discrete
 * update exactly as written, in double; mode 1: classical RK4 of the continuous ODE (for the
 * double integrator this differs from the reference's update x += h(5v + 2ah)/6).  Integrates `steps` steps
 * with no checks; writes state_dim doubles. */
void ko_integrate_f64(const kpax_config* cfg, const double* x0, const float* ctrl, int steps,
                      int mode, double* out);
/* Map six uniforms to the row's controls (row layout) and the step count. */
int ko_controls(const kpax_config* cfg, const float* u, float* ctrl_row, int32_t* steps);

/* ---- regions (Graph.cu:53-205) ---- */
int ko_table_cols(const kpax_config* cfg);
void ko_region_table(const kpax_config* cfg, float* table);
int ko_region_r1(const kpax_config* cfg, const float* state);
int ko_region_r2(const kpax_config* cfg, const float* table, const float* state, int r1);

/* ---- scores (Graph.cu:233-358, fixed-order restatement) ---- */
void ko_scores(const kpax_config* cfg, const int32_t* counter, const int32_t* valid,
               const uint32_t* r2_bits, float* scores);
float ko_faccept(const kpax_config* cfg, uint32_t iter, uint32_t tree_after);

/* ---- whole plan (KPAX.cu:51-115, 303-543) ---- */
typedef struct ko_plan_out {
    /* caller-allocated (max_tree_size rows etc.); any may be NULL */
    float* rows;        /* tree rows, sample_dim floats each */
    int32_t* parents;
    float* costs;
    int32_t* r1;
    uint8_t* repeat;    /* frontier repeat count per node at the end (255 = pending new node) */
    int32_t* counter;   /* num_r1 */
    int32_t* valid;     /* num_r1 */
    float* scores;      /* num_r1 */
    uint32_t* r2_bits;  /* ceil(num_r2 / 32) words */
    float* path;        /* (max_iter + 1) rows */
    uint32_t* iter_children;  /* per iteration: children propagated */
    uint32_t* iter_appended;  /* per iteration: nodes appended */
    /* results */
    kpax_result result;
} ko_plan_out;
/* Frontier compaction on its own (kpax_frontier_compact): repeat bytes in place (255 = pending,
 * resolved as a node of a region without valid samples), entries[0..E), stats = {R, k, E, n}. */
void ko_frontier_compact(const kpax_config* cfg, uint8_t* rep, uint32_t n, uint32_t budget, uint32_t* entries,
                         uint32_t stats[4]);
int ko_plan(const kpax_config* cfg, const float* init, const float* goal, const float* obs,
            uint32_t n_obs, uint32_t plan_idx, uint32_t max_iters, int stop_at_goal,
            ko_plan_out* out);

/* ReKinoLite restatement (see kpax_oracle.c). */
int ko_rekino(const kpax_config* cfg, const float* init, const float* goal, const float* obs, uint32_t n_obs,
              uint32_t num_warps, uint32_t spt, float eps, uint32_t max_iter, uint32_t plan_idx,
              float* out_path, int32_t* out_len, int32_t* out_warp, int32_t* out_iter);

#ifdef __cplusplus
}
#endif
#endif

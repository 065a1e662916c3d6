/*
 * C entry points around the reference's own host-compiled propagation, collision and region
 * routines (oracle/_ref; TEST INFRASTRUCTURE and CPU BASELINE only — never the product path).
 *
 * The reference functions themselves are compiled unmodified from the reference tree:
 *   src/statePropagator/statePropagatorSpatialHash.cu  (propagateAndCheck*SpatialHash)
 *   src/statePropagator/statePropagator.cu             (brute-force propagateAndCheck*, ode)
 *   src/collisionCheck/collisionCheck.cu               (isBroadPhaseValid, isMotionValid)
 *   spatialHash.cu:145-194 and Graph.cu:99-205         (extracted by extract.py)
 *   helper.cu:13-39 (readObstaclesFromCSV)             (extracted by extract.py)
 * This file only adds what the reference implements as kernels or host code that cannot be
 * compiled for the CPU: the grid build (spatialHash.cu:9-67, run serially in obstacle order),
 * the region min-corner table (initializeRegions_kernel, Graph.cu:53-97) and the per-child
 * body of propagateFrontier_kernel1 (KPAX.cu:381-396) as an OpenMP loop.
 */
#include "statePropagator/statePropagatorSpatialHash.cuh"
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <vector>
#include <algorithm>
#include <omp.h>

int getRegion(float* coord);
int getSubRegion(float* coord, int r1, float* minRegion);
std::vector<float> readObstaclesFromCSV(const std::string& filename, int& numObstacles, int workspaceDim);

namespace {
std::vector<int> g_starts(GRID_SIZE), g_counts(GRID_SIZE), g_idx(GRID_SIZE * MAX_OBSTACLES_PER_CELL);
std::vector<float> g_obs;
int g_nobs = 0;
std::vector<float> g_minRegion;

SpatialHashGrid grid_view()
{
    SpatialHashGrid g;
    g.cellStarts = g_starts.data();
    g.cellCounts = g_counts.data();
    g.obstacleIndices = g_idx.data();
    return g;
}

/* initializeRegions_kernel (Graph.cu:53-97) evaluated for every R1 id on the host. */
void build_min_table()
{
    g_minRegion.assign((size_t)NUM_R1_REGIONS * STATE_DIM, 0.0f);
    for(int tid = 0; tid < NUM_R1_REGIONS; ++tid) {
        float* m = &g_minRegion[(size_t)tid * STATE_DIM];
        int wRegion = tid % (W_R1_LENGTH * W_R1_LENGTH * W_R1_LENGTH);
        int idx[8];
        int t = wRegion;
        for(int i = W_DIM - 1; i >= 0; --i) { idx[i] = t % W_R1_LENGTH; t /= W_R1_LENGTH; }
        for(int i = 0; i < W_DIM; ++i) m[i] = W_MIN + idx[i] * W_R1_SIZE;
        int aRegion = (tid / (W_R1_LENGTH * W_R1_LENGTH * W_R1_LENGTH)) % (C_R1_LENGTH * C_R1_LENGTH);
        t = aRegion;
        for(int i = C_DIM - 1; i >= 0; --i) { idx[i] = t % C_R1_LENGTH; t /= C_R1_LENGTH; }
        for(int i = 0; i < C_DIM; ++i) m[W_DIM + i] = C_MIN + idx[i] * C_R1_SIZE;
        int vRegion = (tid / (W_R1_LENGTH * W_R1_LENGTH * W_R1_LENGTH * C_R1_LENGTH * C_R1_LENGTH)) % V_R1_LENGTH;
        t = vRegion;
        for(int i = V_DIM - 1; i >= 0; --i) { idx[i] = t % V_R1_LENGTH; t /= V_R1_LENGTH; }
        for(int i = 0; i < V_DIM; ++i) m[W_DIM + C_DIM + i] = V_MIN + idx[i] * V_R1_SIZE;
    }
}

/* Replay buffer for one child: controls in draw order, duration, then the frontier draw. */
int fill_replay(const float* d6, float* r)
{
    int k = 0;
    for(int i = 0; i < CONTROL_DIM; ++i) r[k++] = d6[i];
    r[k++] = d6[4];
    r[k++] = d6[5];
    return k;
}
}  // namespace

extern "C" {

int kref_info(int what)
{
    switch(what) {
        case 0: return MODEL;
        case 1: return STATE_DIM;
        case 2: return CONTROL_DIM;
        case 3: return SAMPLE_DIM;
        case 4: return GRID_SIZE;
        case 5: return MAX_OBSTACLES_PER_CELL;
        case 6: return NUM_R1_REGIONS;
        case 7: return NUM_R2_PER_R1;
        case 8: return MAX_PROPAGATION_DURATION;
        case 9: return GRID_DIM_X;
        default: return -1;
    }
}

/* Serial restatement of initSpatialHashGrid + buildSpatialHashGrid (spatialHash.cu:9-67).
 * Returns the number of cells whose 16-slot list overflowed (entries dropped). */
int kref_set_obstacles(const float* obs, int n)
{
    g_obs.assign(obs, obs + (size_t)n * 2 * W_DIM);
    g_nobs = n;
    for(int c = 0; c < GRID_SIZE; ++c) { g_starts[c] = c * MAX_OBSTACLES_PER_CELL; g_counts[c] = 0; }
    std::fill(g_idx.begin(), g_idx.end(), 0);
    for(int o = 0; o < n; ++o) {
        const float* b = &g_obs[(size_t)o * 2 * W_DIM];
        int x0, y0, z0, x1, y1, z1;
        worldToGrid(b[0], b[1], b[2], x0, y0, z0);
        worldToGrid(b[3], b[4], b[5], x1, y1, z1);
        for(int gz = z0; gz <= z1; gz++)
            for(int gy = y0; gy <= y1; gy++)
                for(int gx = x0; gx <= x1; gx++) {
                    int cell = gridToIndex(gx, gy, gz);
                    int pos = g_counts[cell]++;
                    if(pos < MAX_OBSTACLES_PER_CELL) g_idx[cell * MAX_OBSTACLES_PER_CELL + pos] = o;
                }
    }
    int overflow = 0;
    for(int c = 0; c < GRID_SIZE; ++c) overflow += g_counts[c] > MAX_OBSTACLES_PER_CELL;
    if(g_minRegion.empty()) build_min_table();
    return overflow;
}

/* Number of entries the reference grid holds for a cell (its count, possibly > 16). */
int kref_cell_count(int cell) { return g_counts[cell]; }

/* Propagate n segments with the reference's model function selected by MODEL.
 * x0: n x STATE_DIM; draws: n x 6 (controls in draw order in columns 0..3, duration in 4).
 * use_hash: 1 = propagateAndCheckSpatialHash (spatial-hash collision, with the 16-slot cap),
 *           0 = propagateAndCheck (brute force over all obstacles). */
void kref_propagate(const float* x0, const float* draws, int n, int use_hash, float* rows,
                    unsigned char* valid, int nthreads)
{
    SpatialHashGrid g = grid_view();
    float* obs = g_obs.data();
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(dynamic, 64)
    for(int i = 0; i < n; ++i) {
        float p[STATE_DIM], r[8];
        memcpy(p, x0 + (size_t)i * STATE_DIM, sizeof(p));
        fill_replay(draws + (size_t)i * 6, r);
        curandState st = {r, 0};
        bool ok = use_hash ? propagateAndCheckSpatialHash(p, rows + (size_t)i * SAMPLE_DIM, &st, g, obs, g_nobs)
                           : propagateAndCheck(p, rows + (size_t)i * SAMPLE_DIM, &st, obs, g_nobs);
        valid[i] = ok ? 1 : 0;
    }
}

/* getRegion / getSubRegion of n states with the reference's min-corner table. */
void kref_region(const float* states, int stride, int n, int* r1, int* r2)
{
    if(g_minRegion.empty()) build_min_table();
    for(int i = 0; i < n; ++i) {
        float s[SAMPLE_DIM];
        memset(s, 0, sizeof(s));
        memcpy(s, states + (size_t)i * stride, sizeof(float) * STATE_DIM);
        int a = getRegion(s);
        r1[i] = a;
        if(r2) r2[i] = getSubRegion(s, a, g_minRegion.data());
    }
}

/* The reference's min-corner table (NUM_R1_REGIONS x STATE_DIM floats). */
void kref_min_table(float* out)
{
    if(g_minRegion.empty()) build_min_table();
    memcpy(out, g_minRegion.data(), g_minRegion.size() * sizeof(float));
}

/* isMotionValidSpatialHash / isMotionValid on one step box. */
int kref_collide(const float* bbmin, const float* bbmax, int use_hash)
{
    float lo[3] = {bbmin[0], bbmin[1], bbmin[2]}, hi[3] = {bbmax[0], bbmax[1], bbmax[2]};
    if(use_hash) return isMotionValidSpatialHash(lo, hi, lo, hi, grid_view(), g_obs.data()) ? 1 : 0;
    return isMotionValid(lo, hi, lo, hi, g_obs.data(), g_nobs) ? 1 : 0;
}

/* kref_collide over n boxes (n x 3 floats each side), OpenMP over the boxes. */
void kref_collide_batch(const float* bbmin, const float* bbmax, int n, int use_hash, uint8_t* out, int nthreads)
{
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for(int i = 0; i < n; ++i) out[i] = (uint8_t)kref_collide(bbmin + 3 * (size_t)i, bbmax + 3 * (size_t)i, use_hash);
}

#if MODEL == 3
/* The quadrotor right-hand side (statePropagator.cu:325-370). */
void kref_ode(float* xdot, const float* x0, const float* h, const float* ctrl, int itr)
{
    float a[STATE_DIM], b[STATE_DIM];
    memcpy(a, x0, sizeof(a));
    if(h) memcpy(b, h, sizeof(b));
    ode(xdot, a, h ? b : nullptr, ctrl[0], ctrl[1], ctrl[2], ctrl[3], itr);
}
#endif

/* Per-child body of propagateFrontier_kernel1 (KPAX.cu:381-396) over n children, OpenMP.
 * Child c expands parents[c / per_parent]; draws: n x 6 (controls, duration, frontier draw).
 * scores: NUM_R1_REGIONS floats; r2flags: NUM_R2_REGIONS ints (read and set like the kernel);
 * counter/valid_counter: NUM_R1_REGIONS ints.  Returns the number of valid children. */
long long kref_expand(const float* parents, int per_parent, const float* draws, int n, const float* scores,
                      int* r2flags, int* counter, int* valid_counter, unsigned char* fnext, float* rows, int nthreads)
{
    if(g_minRegion.empty()) build_min_table();
    SpatialHashGrid g = grid_view();
    float* obs = g_obs.data();
    float* minRegion = g_minRegion.data();
    long long nvalid = 0;
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(dynamic, 64) reduction(+ : nvalid)
    for(int c = 0; c < n; ++c) {
        float p[STATE_DIM], r[8];
        memcpy(p, parents + (size_t)(c / per_parent) * STATE_DIM, sizeof(p));
        fill_replay(draws + (size_t)c * 6, r);
        curandState st = {r, 0};
        float* x1 = rows + (size_t)c * SAMPLE_DIM;
        bool valid = propagateAndCheckSpatialHash(p, x1, &st, g, obs, g_nobs);
        int v = getRegion(x1);
        int sv = getSubRegion(x1, v, minRegion);
#pragma omp atomic
        counter[v] += 1;
        fnext[c] = 0;
        if(valid) {
            nvalid += 1;
#pragma omp atomic
            valid_counter[v] += 1;
            int flag;
#pragma omp atomic read
            flag = r2flags[sv];
            if(curand_uniform(&st) < scores[v] || !flag) fnext[c] = 1;
            if(flag == 0) {
#pragma omp atomic write
                r2flags[sv] = 1;
            }
        }
    }
    return nvalid;
}

int kref_max_threads(void) { return omp_get_max_threads(); }

/* readObstaclesFromCSV (helper.cu:13-39) on a file that exists (it exits the process otherwise):
 * returns the number of floats read and copies up to `cap` of them; *n_obstacles as it sets. */
int kref_read_obstacles_csv(const char* path, float* out, int cap, int* n_obstacles)
{
    FILE* f = fopen(path, "r");
    if(!f) return -1;
    fclose(f);
    int n = 0;
    const std::vector<float> v = readObstaclesFromCSV(path, n, 3);
    memcpy(out, v.data(), sizeof(float) * std::min<size_t>(v.size(), (size_t)cap));
    *n_obstacles = n;
    return (int)v.size();
}

}  // extern "C"

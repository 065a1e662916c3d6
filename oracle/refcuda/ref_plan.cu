// ref_plan.cu — harness of the reference's own CUDA planner (TEST INFRASTRUCTURE).
//
// Links the reference's KPAX planner, compiled unmodified from its sources for sm_100a
// (src/planners/KPAX.cu, Planner.cu, src/graphs/Graph.cu, src/collisionCheck/*.cu,
// src/statePropagator/statePropagator*.cu, src/helper/helper.cu) with one configuration header
// from cfg/, and times whole plans through its public entry point
//     KPAX::plan(float* h_initial, float* h_goal, float* d_obstacles_ptr, uint n, bool)
// (KPAX.cu:51-115), as the reference's example drivers do (examples/gpu/main.cu).  The valid
// expansions of a plan are the reference's own counter, the sum of graph_.d_validCounterArray_
// (incremented once per valid child, KPAX.cu:393; reset by plan, KPAX.cu:71).
//
// Guards (both checked before any device work of the planner runs):
//  - capacity: MAX_ITER is kref_iteration_bound() (see kref_cuda_common.h), evaluated by the
//    reference before each iteration.  It sums the frontier's repeat counts R (the quantity
//    propagateFrontier scans, KPAX.cu:316-321) and ends the plan before an iteration whose frontier
//    has more entries than the tree has free slots.  That is the one case in which the reference
//    writes past its buffers: propIterations rounds down to 0 and is forced to 1
//    (KPAX.cu:325-333), so R children are appended into fewer free slots (updateFrontier_kernel,
//    KPAX.cu:461) and repeatInd fills R entries (Planner.cu:68-80).  With R <= free slots the
//    branch of KPAX.cu:323-341 runs as designed (propIterations = min(free / R, 32) children per
//    entry) and stays inside every buffer; its clear of frontier[tid] by thread index
//    (KPAX.cu:411) reaches index propIterations * R + 31 < MAX_TREE_SIZE once the tree holds 32
//    nodes, which the guard also requires whenever that branch would run.
//  - hash grid: a cell's obstacle count keeps growing past its 16 slots (spatialHash.cu:41-48)
//    and isMotionValidSpatialHash reads `count` slots from the cell's start
//    (spatialHash.cu:166-173), i.e. into the following cells' slots.  The harness recounts the
//    cells on the host with the reference's own worldToGrid / gridToIndex and refuses a scene in
//    which such a read would pass the end of the slot array; it zeroes the slot array once, so a
//    slot that no build wrote reads as obstacle 0 rather than uninitialised memory.
//
// Usage: kref_cuda_<cfg> <obstacles.csv> <queries.txt> <out.json> <workdir> <iteration cap> [repeats]
//   queries.txt: one query per line, "sx sy sz gx gy gz" (the other state components 0).
//   The planner writes its CSV side files (Data/...) under <workdir> (created if missing).
#include <stdint.h>
#include <sys/stat.h>
#include <unistd.h>

#include <chrono>
#include <climits>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include <thrust/reduce.h>

#include "collisionCheck/spatialHash.cuh"
#include "planners/KPAX.cuh"

namespace {

constexpr int kPathRows = 1 << 14;  // MAX_ITER at construction: rows of the path buffers

KPAX* g_planner = nullptr;
bool g_planning = false;
uint32_t g_cap = 0;
bool g_guard_stop = false;
bool g_stopped = false;  // the last evaluation ended the loop
double g_hook_s = 0.0;

struct HookRec {
    double t0, t1;       // host clock around the hook
    uint32_t R;          // frontier repeat total before the next iteration
    uint32_t tree;       // h_treeSize_
    long long valid;     // sum of the valid counters so far
    long long children;  // sum of the sample counters so far (one per child, KPAX.cu:390)
};
std::vector<HookRec> g_recs;

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int kref_iteration_bound(void)
{
    if(!g_planning || !g_planner) return kPathRows;
    KPAX& pl = *g_planner;
    const double t0 = now_s();
    const uint32_t R = thrust::reduce(pl.d_activeFrontierRepeatCount_.begin(), pl.d_activeFrontierRepeatCount_.end(), 0u);
    const long long valid = thrust::reduce(pl.graph_.d_validCounterArray_.begin(), pl.graph_.d_validCounterArray_.end(), 0LL);
    const long long children = thrust::reduce(pl.graph_.d_counterArray_.begin(), pl.graph_.d_counterArray_.end(), 0LL);
    const uint64_t free_slots = (uint64_t)(MAX_TREE_SIZE - pl.h_treeSize_);
    const bool full_expansion = (uint64_t)R * pl.h_activeBlockSize_ <= free_slots;  // propagateFrontier_kernel1
    const bool fits = full_expansion || ((uint64_t)R <= free_slots && pl.h_treeSize_ >= 32);
    const double t1 = now_s();
    g_recs.push_back({t0, t1, R, pl.h_treeSize_, valid, children});
    g_hook_s += t1 - t0;
    g_guard_stop = !fits;
    g_stopped = !fits || pl.h_itr_ >= g_cap;
    return g_stopped ? 0 : INT_MAX;
}

static void fail(const char* out, const std::string& why)
{
    std::ofstream f(out);
    f << "{\"unavailable\": \"" << why << "\"}\n";
    fprintf(stderr, "%s\n", why.c_str());
}

static bool cuda_ok(const char* out, cudaError_t e, const char* what)
{
    if(e == cudaSuccess) return true;
    fail(out, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

int main(int argc, char** argv)
{
    if(argc < 6) {
        fprintf(stderr, "usage: %s obstacles.csv queries.txt out.json workdir iteration_cap [repeats]\n", argv[0]);
        return 2;
    }
    // the output path is resolved before the planner's work directory is entered
    std::string out_path = argv[3];
    if(!out_path.empty() && out_path[0] != '/') {
        char cwd[4096];
        if(getcwd(cwd, sizeof(cwd))) out_path = std::string(cwd) + "/" + out_path;
    }
    const char* out = out_path.c_str();
    const uint32_t cap = (uint32_t)atoi(argv[5]);
    const int repeats = argc > 6 ? atoi(argv[6]) : 1;
    if(cap < 1 || cap > kPathRows - 2) {
        fail(out, "iteration cap out of range");
        return 2;
    }
    // queries
    std::vector<std::vector<float>> queries;
    {
        std::ifstream qf(argv[2]);
        std::string line;
        while(std::getline(qf, line)) {
            std::istringstream ss(line);
            std::vector<float> q(6);
            bool ok = true;
            for(int k = 0; k < 6; ++k) ok = ok && static_cast<bool>(ss >> q[k]);
            if(ok) queries.push_back(q);
        }
    }
    if(queries.empty()) {
        fail(out, "no queries");
        return 2;
    }
    // obstacles through the reference's own reader (helper.cu:13-39)
    int n_obs = 0;
    std::vector<float> obs = readObstaclesFromCSV(argv[1], n_obs, W_DIM);
    // hash-grid guard, on the host with the reference's cell mapping (spatialHash.cu:26-38)
    std::vector<int> counts(GRID_SIZE, 0);
    for(int o = 0; o < n_obs; ++o) {
        int x0, y0, z0, x1, y1, z1;
        worldToGrid(obs[6 * o + 0], obs[6 * o + 1], obs[6 * o + 2], x0, y0, z0);
        worldToGrid(obs[6 * o + 3], obs[6 * o + 4], obs[6 * o + 5], x1, y1, z1);
        for(int gz = z0; gz <= z1; ++gz)
            for(int gy = y0; gy <= y1; ++gy)
                for(int gx = x0; gx <= x1; ++gx) ++counts[gridToIndex(gx, gy, gz)];
    }
    long long worst_end = 0;
    int overflowing = 0, max_count = 0;
    for(int c = 0; c < GRID_SIZE; ++c) {
        worst_end = std::max(worst_end, (long long)c * MAX_OBSTACLES_PER_CELL + counts[c]);
        overflowing += counts[c] > MAX_OBSTACLES_PER_CELL;
        max_count = std::max(max_count, counts[c]);
    }
    if(worst_end > (long long)GRID_SIZE * MAX_OBSTACLES_PER_CELL) {
        fail(out, "scene refused: a hash-cell query of the reference would read past its slot array");
        return 0;
    }
    mkdir(argv[4], 0755);
    if(chdir(argv[4]) != 0) {
        fail(out, "cannot enter the work directory");
        return 2;
    }

    float* d_obs = nullptr;
    if(!cuda_ok(out, cudaMalloc(&d_obs, sizeof(float) * obs.size() + 16), "cudaMalloc")) return 1;
    if(!cuda_ok(out, cudaMemcpy(d_obs, obs.data(), sizeof(float) * obs.size(), cudaMemcpyHostToDevice), "copy"))
        return 1;

    KPAX planner;
    {
        SpatialHashGrid hg;
        if(!cuda_ok(out, cudaMemcpy(&hg, planner.d_spatialHashGrid_, sizeof(hg), cudaMemcpyDeviceToHost), "grid"))
            return 1;
        if(!cuda_ok(out, cudaMemset(hg.obstacleIndices, 0, sizeof(int) * GRID_SIZE * MAX_OBSTACLES_PER_CELL), "zero"))
            return 1;
    }
    if(!cuda_ok(out, cudaDeviceSynchronize(), "setup")) return 1;
    g_planner = &planner;
    g_cap = cap;

    std::ostringstream js;
    js << "{\"config\": {\"model\": " << MODEL << ", \"max_tree_size\": " << MAX_TREE_SIZE << ", \"step_size\": " << STEP_SIZE
       << ", \"max_propagation_duration\": " << MAX_PROPAGATION_DURATION << ", \"iteration_cap\": " << cap
       << ", \"num_r1\": " << NUM_R1_REGIONS << ", \"obstacles\": " << n_obs << ", \"grid_cells_over_16\": " << overflowing
       << ", \"grid_max_count\": " << max_count << "},\n \"plans\": [";
    bool first = true;
    std::vector<int> parents;
    for(int rep = 0; rep < repeats; ++rep)
        for(const auto& q : queries) {
            float h_init[SAMPLE_DIM] = {0}, h_goal[SAMPLE_DIM] = {0};
            for(int k = 0; k < 3; ++k) h_init[k] = q[k], h_goal[k] = q[3 + k];
            g_recs.clear();
            g_guard_stop = g_stopped = false;
            g_hook_s = 0.0;
            g_planning = true;
            const double t0 = now_s();
            planner.plan(h_init, h_goal, d_obs, (uint)n_obs, false);
            const double t1 = now_s();
            g_planning = false;
            if(!cuda_ok(out, cudaDeviceSynchronize(), "plan")) return 1;
            const long long valid =
              thrust::reduce(planner.graph_.d_validCounterArray_.begin(), planner.graph_.d_validCounterArray_.end(), 0LL);
            const long long children =
              thrust::reduce(planner.graph_.d_counterArray_.begin(), planner.graph_.d_counterArray_.end(), 0LL);
            // path: parent walk from the goal node (the reference copies h_itr_ rows, KPAX.cu:102)
            const int goal = planner.h_pathToGoal_;
            int path_len = 0;
            double path_cost = 0.0;
            if(goal != 0) {
                parents.resize(planner.h_treeSize_);
                cudaMemcpy(parents.data(), planner.d_treeSamplesParentIdxs_ptr_, sizeof(int) * parents.size(),
                           cudaMemcpyDeviceToHost);
                for(int node = goal; node >= 0 && path_len <= (int)planner.h_treeSize_; node = parents[node]) {
                    ++path_len;
                    if(parents[node] >= 0) {
                        float d = 0.0f;
                        cudaMemcpy(&d, planner.d_treeSamples_ptr_ + (size_t)node * SAMPLE_DIM + SAMPLE_DIM - 1, sizeof(float),
                                   cudaMemcpyDeviceToHost);
                        path_cost += d;
                    }
                }
            }
            // per iteration: children and valid children (the reference's counters), host seconds
            std::ostringstream it;
            const size_t nrec = g_recs.size();
            const size_t n_it = g_stopped && nrec ? nrec - 1 : nrec;
            for(size_t i = 0; i < n_it; ++i) {
                const double te = i + 1 < nrec ? g_recs[i + 1].t0 : t1;
                const long long ve = i + 1 < nrec ? g_recs[i + 1].valid : valid;
                const long long ce = i + 1 < nrec ? g_recs[i + 1].children : children;
                it << (i ? "," : "") << "[" << (ce - g_recs[i].children) << "," << (ve - g_recs[i].valid) << ","
                   << (te - g_recs[i].t1) << "]";
            }
            js << (first ? "\n  " : ",\n  ") << "{\"start\": [" << q[0] << "," << q[1] << "," << q[2] << "], \"goal\": [" << q[3]
               << "," << q[4] << "," << q[5] << "], \"found\": " << (goal != 0 ? 1 : 0) << ", \"iters\": " << planner.h_itr_
               << ", \"tree_size\": " << planner.h_treeSize_ << ", \"children\": " << children << ", \"valid\": " << valid
               << ", \"wall_s\": " << (t1 - t0) << ", \"guard_s\": " << g_hook_s << ", \"capacity_stop\": " << (g_guard_stop ? 1 : 0)
               << ", \"path_len\": " << path_len << ", \"path_cost\": " << path_cost << ", \"iterations\": [" << it.str() << "]}";
            first = false;
        }
    js << "\n]}\n";
    g_planner = nullptr;
    std::ofstream f(out);
    f << js.str();
    cudaFree(d_obs);
    return 0;
}

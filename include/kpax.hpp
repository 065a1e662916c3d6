/*
 * kpax.hpp — header-only C++ mirror of the reference planner class over the C ABI (kpax.h).
 *
 * Same entry point and public result fields as the reference's KPAX / Planner classes
 * (include/planners/KPAX.cuh:6-65, include/planners/Planner.cuh:19-69):
 *     KPAX planner(cfg);
 *     planner.plan(h_initial, h_goal, d_obstacles_ptr, h_obstaclesCount, saveTree);
 *     planner.h_pathToGoal_, planner.h_itr_, planner.h_treeSize_, planner.h_controlPathToGoal_
 * The reference reads its configuration from compile-time macros; here it is a kpax_config
 * (defaulting to the quadrotor preset).  Errors raise std::runtime_error with the library's
 * message instead of going unreported.
 */
#ifndef KPAX_HPP_
#define KPAX_HPP_

#include <stdexcept>
#include <string>
#include <vector>

#include "kpax.h"

class KPAX {
public:
    explicit KPAX(int preset = KPAX_PRESET_QUAD) { init(make_preset(preset)); }
    explicit KPAX(const kpax_config& cfg) { init(cfg); }
    ~KPAX() { kpax_destroy(handle_); }
    KPAX(const KPAX&) = delete;
    KPAX& operator=(const KPAX&) = delete;

    /* KPAX::plan (src/planners/KPAX.cu:51-115): h_initial / h_goal hold SAMPLE_DIM host floats,
     * d_obstacles_ptr is a device buffer of h_obstaclesCount x 6 floats. */
    void plan(float* h_initial, float* h_goal, float* d_obstacles_ptr, unsigned h_obstaclesCount, bool saveTree = false)
    {
        check(kpax_plan(handle_, h_initial, h_goal, d_obstacles_ptr, h_obstaclesCount, saveTree ? 1 : 0, &result_));
        publish();
    }

    /* KPAX::planBench (src/planners/KPAX.cu:243-300): the plan with the per-iteration CSV dumps of
     * writeDeviceVectorsToCSV under out_dir/Data (the reference writes under the working directory). */
    void planBench(float* h_initial, float* h_goal, float* d_obstacles_ptr, unsigned h_obstaclesCount, int benchItr,
                   const char* out_dir = ".")
    {
        check(kpax_plan_bench(handle_, h_initial, h_goal, d_obstacles_ptr, h_obstaclesCount, benchItr, out_dir, &result_));
        publish();
    }

    const kpax_result& result() const { return result_; }
    kpax_planner* handle() const { return handle_; }
    unsigned sampleDim() const { return sample_dim_; }

    /* public fields of the reference (Planner.cuh:31-43) */
    unsigned h_treeSize_ = 0, h_itr_ = 0;
    int h_pathToGoal_ = 0;
    float h_costToGoal_ = 0.0f;
    float* h_controlPathToGoal_ = nullptr; /* path rows, goal first, result().path_len of them */

private:
    void publish()
    {
        h_treeSize_ = result_.tree_size;
        h_itr_ = result_.iters;
        h_pathToGoal_ = (int)result_.goal_idx;
        h_costToGoal_ = (float)result_.path_cost;
        path_.assign(result_.h_path, result_.h_path + (size_t)result_.path_len * sample_dim_);
        h_controlPathToGoal_ = path_.data();
    }
    static kpax_config make_preset(int preset)
    {
        kpax_config c;
        check(kpax_config_preset(preset, &c));
        return c;
    }
    static void check(kpax_status s)
    {
        if(s != KPAX_OK) throw std::runtime_error(std::string("kpax: ") + kpax_last_error());
    }
    void init(const kpax_config& cfg)
    {
        uint32_t n1 = 0, p = 0;
        check(kpax_config_sizes(&cfg, &n1, &p, &sample_dim_));
        check(kpax_create(&cfg, &handle_));
    }

    kpax_planner* handle_ = nullptr;
    kpax_result result_{};
    uint32_t sample_dim_ = 0;
    std::vector<float> path_;
};

/* readObstaclesFromCSV (src/helper/helper.cu:13-39) with the reference's signature: every float of
 * the file, numObstacles = floats / (2 * workspaceDim).  Throws std::runtime_error where the
 * reference exits (the file cannot be opened). */
inline std::vector<float> readObstaclesFromCSV(const std::string& filename, int& numObstacles, int workspaceDim)
{
    auto check = [](kpax_status s) {
        if(s != KPAX_OK) throw std::runtime_error(std::string("kpax: ") + kpax_last_error());
    };
    uint64_t n = 0, m = 0;
    check(kpax_read_obstacles_csv(filename.c_str(), nullptr, 0, &n));
    std::vector<float> v(n);
    check(kpax_read_obstacles_csv(filename.c_str(), v.data(), n, &m));
    v.resize(m < n ? m : n);
    numObstacles = (int)(v.size() / (2 * (size_t)workspaceDim));
    return v;
}

#endif /* KPAX_HPP_ */

"""Whole plans of the Dubins and quadrotor planners judged as distributions over a fixed seed set.

For these models the CUDA path matches the oracle per child within the propagation tolerance
(teacher-forced iterations in test_gpu_plan.py), so whole plans may part ways where a state lands
within rounding of a region boundary or a verdict within rounding of contact.  Over 16 seeded
queries (scene, start/goal pair, plan index) the success count and the path-cost distribution of
the solved plans must agree with the oracle's: success counts within 2 of 16; of the solved plans'
path costs (sums of segment durations), the means within 25 %, the medians within 25 % or one
segment, and the two-sample Kolmogorov-Smirnov distance at most 0.35; and at least 12 of the 16
outcomes (found, path cost, iterations) identical."""
import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

pytestmark = pytest.mark.gpu

SEEDS = range(16)


def small(preset: int):
    cfg = kpax.preset(preset)
    cfg.expansions_per_iter = 1 << 12
    cfg.max_tree_size = 1 << 17
    cfg.max_iter = 100
    return cfg


def dubins_query(seed: int, obs: np.ndarray, lo: float = 8.0, hi: float = 12.0):
    """Start and goal in the forest's free space, lo..hi apart, the start heading for the goal at 1 m/s."""
    rng = np.random.default_rng(seed)
    while True:
        a, b = rng.uniform(10.0, 90.0, 3), rng.uniform(10.0, 90.0, 3)
        if lo <= np.linalg.norm(a - b) <= hi and not any(E._covers(o, a) or E._covers(o, b) for o in obs):
            break
    s, g = np.zeros(6, np.float32), np.zeros(6, np.float32)
    s[:3], g[:3] = a, b
    s[3], s[5] = np.arctan2(b[1] - a[1], b[0] - a[0]), 1.0
    return s, g


def queries(model: str):
    if model == "dubins":
        obs, _, _ = E.dubins_scene()
        return [(obs, *dubins_query(seed, obs)) for seed in SEEDS]
    # quadrotor: building scenes of 100-300 boxes (windowed wall included), start and goal 6-10 m apart
    return [E.learned_family(100 + seed, obs_range=(100, 300), min_sep=6.0, max_sep=10.0) for seed in SEEDS]


@pytest.mark.parametrize("model", ["dubins", "quad"])
def test_success_and_path_cost_distributions_match_oracle(cuda, model):
    import torch

    cfg = small(kpax.PRESET_DUBINS if model == "dubins" else kpax.PRESET_QUAD)
    pl = kpax.KPAX(cfg)  # plan i of this planner draws from plan index i, as the oracle's plan_idx = i
    gpu, ora = [], []
    for i, (obs, s, g) in enumerate(queries(model)):
        d_obs = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
        r = pl.plan(s, g, d_obs.data_ptr(), obs.shape[0])
        gpu.append((int(r.found), float(r.path_cost) if r.found else None, int(r.iters)))
        o = O.plan(cfg, s, g, obs, plan_idx=i)
        ora.append((int(o["found"]), float(o["path_cost"]) if o["found"] else None, int(o["iters"])))
        if r.found:  # a solved plan's path reaches the goal ball from the start
            p = pl.h_controlPathToGoal_
            assert np.linalg.norm(p[0, :3] - g[:3]) < cfg.goal_thresh
            assert np.array_equal(p[-1, :3], s[:3])
    same = sum(a == b for a, b in zip(gpu, ora))
    print(f"{model}: gpu {gpu}\n{model}: oracle {ora}\n{model}: identical outcomes {same}/{len(gpu)}")
    # on a B200 all 16 outcomes (found, path cost, iterations) are identical for both models
    assert same >= 12, same
    n_gpu, n_ora = sum(x[0] for x in gpu), sum(x[0] for x in ora)
    assert n_ora >= len(ora) // 2, "the seed set should be mostly solvable"
    assert abs(n_gpu - n_ora) <= 2, (n_gpu, n_ora)
    a, b = np.sort([x[1] for x in gpu if x[0]]), np.sort([x[1] for x in ora if x[0]])
    seg = cfg.step_size * cfg.max_propagation_duration  # one full segment's duration
    assert abs(np.mean(a) - np.mean(b)) <= 0.25 * np.mean(b), (np.mean(a), np.mean(b))
    assert abs(np.median(a) - np.median(b)) <= max(0.25 * np.median(b), seg), (np.median(a), np.median(b))
    # two-sample Kolmogorov-Smirnov distance of the path costs
    x = np.union1d(a, b)
    ks = np.max(np.abs(np.searchsorted(a, x, "right") / a.size - np.searchsorted(b, x, "right") / b.size))
    assert ks <= 0.35, ks


def test_benchmark_configuration_plans_match_oracle(cuda):
    """Whole plans at the 12D quadrotor benchmark configuration itself — 2^16 children per
    iteration, a 2^20-node tree, the 1000-box building scene with its windowed wall, 25 fixed RK4
    steps of 0.02 s — on 12 seeded start/goal pairs in the scene's free space, 6-12 m apart (30
    iterations per plan).  Every outcome (found, path cost, iterations, tree size) must equal the
    oracle's plan with the same plan index, and most queries must be solved."""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter = 30
    obs, _, _ = E.quad_scene()
    qs = E.free_queries(obs, 12, seed=11, min_sep=6.0, max_sep=12.0)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    pl = kpax.KPAX(cfg)
    gpu, ora = [], []
    for i, q in enumerate(qs):
        s, g = np.zeros(12, np.float32), np.zeros(12, np.float32)
        s[:3], g[:3] = q[:3], q[3:]
        r = pl.plan(s, g, d_obs.data_ptr(), obs.shape[0])
        gpu.append((int(r.found), float(r.path_cost) if r.found else None, int(r.iters), int(r.tree_size)))
        o = O.plan(cfg, s, g, obs, plan_idx=i)
        ora.append((int(o["found"]), float(o["path_cost"]) if o["found"] else None, int(o["iters"]), int(o["tree_size"])))
        if r.found:
            p = pl.h_controlPathToGoal_
            assert np.linalg.norm(p[0, :3] - g[:3]) < cfg.goal_thresh
            assert np.array_equal(p[-1, :3], s[:3])
    same = sum(a == b for a, b in zip(gpu, ora))
    print(f"gpu {gpu}\noracle {ora}\nidentical outcomes {same}/{len(gpu)}")
    assert sum(x[0] for x in ora) >= len(ora) // 2, "the query set should be mostly solvable"
    # children within rounding of a region boundary or of contact may part the trees (FP32 states
    # within 1e-5 of the oracle's); allow one of the twelve to differ
    assert same >= len(gpu) - 1, same

"""Whole-plan parity of the CUDA planner with the CPU oracle.

Double integrator: every buffer (tree rows, parents, costs, region counters, scores, R2 bits,
frontier repeats, path) is bit-exact.  Dubins / quadrotor: each iteration is checked child by
child against the oracle re-run on the GPU's own tree ("teacher forcing"): parent assignment,
draws, step counts and region ids exact, states within the propagation tolerance, verdicts exact
except near-boundary segments (listed)."""
import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
NEAR_TOL = 1e-4


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def small_di(fast: bool = False):
    cfg = kpax.preset(kpax.PRESET_DI)
    cfg.max_tree_size = 1 << 15
    cfg.expansions_per_iter = 1 << 12
    cfg.max_iter = 60
    if fast:  # moves up to ~5 m per segment so the goal is reachable before the tree fills
        cfg.v_min, cfg.v_max = -5.0, 5.0
        for i in range(3):
            cfg.ctrl_min[i], cfg.ctrl_max[i] = -4.0, 4.0
    return cfg


def gpu_plan(torch, cfg, start, goal, obs, planner=None):
    pl = planner or kpax.KPAX(cfg)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    r = pl.plan(start, goal, d_obs.data_ptr(), obs.shape[0])
    out = {f: getattr(r, f) for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full", "expansions",
                                        "valid_expansions", "path_cost")}
    rows, parents, costs = pl.export_tree()
    counter, valid, scores, r2 = pl.export_regions()
    rep, r1 = pl.export_frontier(r.tree_size)
    out.update(rows=rows, parents=parents, costs=costs, counter=counter, valid=valid, scores=scores, r2_bits=r2, repeat=rep,
               r1=r1, path=pl.h_controlPathToGoal_.copy())
    return out, pl


def assert_plans_equal(g, o):
    for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full", "expansions", "valid_expansions"):
        assert g[f] == o[f], (f, g[f], o[f])
    assert np.array_equal(bits(g["rows"]), bits(o["rows"]))
    assert np.array_equal(g["parents"], o["parents"])
    assert np.array_equal(bits(g["costs"]), bits(o["costs"]))
    assert np.array_equal(g["r1"], o["r1"])
    assert np.array_equal(g["repeat"], o["repeat"])
    assert np.array_equal(g["counter"], o["counter"]) and np.array_equal(g["valid"], o["valid"])
    assert np.array_equal(bits(g["scores"]), bits(o["scores"]))
    assert np.array_equal(g["r2_bits"], o["r2_bits"])
    assert np.array_equal(bits(g["path"]), bits(o["path"]))


def test_di_plan_bit_exact_until_tree_full(cuda):
    import torch

    cfg = small_di()
    obs, s, goal = E.di_scene()
    g, _ = gpu_plan(torch, cfg, s, goal, obs)
    o = O.plan(cfg, s, goal, obs, plan_idx=0)
    assert g["tree_full"] == 1 and g["tree_size"] == cfg.max_tree_size
    assert_plans_equal(g, o)


def test_di_plan_bit_exact_goal_found(cuda, tmp_path):
    import torch

    cfg = small_di(fast=True)
    obs, s, _ = E.di_scene()
    goal = np.array([40, 40, 40, 0, 0, 0], np.float32)
    g, pl = gpu_plan(torch, cfg, s, goal, obs)
    o = O.plan(cfg, s, goal, obs, plan_idx=0)
    assert g["found"] == 1
    assert_plans_equal(g, o)
    # the path walks parent links from the goal node to the root (KPAX.cu:482-501)
    path = g["path"]
    assert np.linalg.norm(path[0, :3] - goal[:3]) < cfg.goal_thresh
    assert np.array_equal(path[-1, :6], s[:6])
    # the solution file: controlPathToGoal.csv rows (goal first, root last), "%.6f" values
    f = tmp_path / "controlPathToGoal.csv"
    pl.write_solution_csv(f)
    want = "".join(",".join(f"{float(v):.6f}" for v in r) + "\n" for r in path)
    assert f.read_text() == want
    # a second plan on the same planner draws a new random stream (plan index 1)
    g2, _ = gpu_plan(torch, cfg, s, goal, obs, planner=pl)
    o2 = O.plan(cfg, s, goal, obs, plan_idx=1)
    assert_plans_equal(g2, o2)


@pytest.mark.parametrize("fast", [False, True])
def test_di_plan_with_pruning_bit_exact(cuda, fast):
    """PruneKPAX's goal-progress pruning (PruneKPAX.cu:466-498) as a frontier policy on the same
    kernels: whole plans equal the oracle's bit for bit, and pruning removes children."""
    import torch

    cfg = small_di(fast=fast)
    cfg.prune = 1
    obs, s, goal = E.di_scene()
    if fast:
        goal = np.array([40, 40, 40, 0, 0, 0], np.float32)
    g, _ = gpu_plan(torch, cfg, s, goal, obs)
    o = O.plan(cfg, s, goal, obs, plan_idx=0)
    assert_plans_equal(g, o)
    cfg.prune = 0
    plain = O.plan(cfg, s, goal, obs, plan_idx=0)
    assert (g["tree_size"] < plain["tree_size"]) or (g["iters"] != plain["iters"])


def test_plan_host_matches_device_obstacles(cuda):
    import torch

    cfg = small_di(fast=True)
    obs, s, _ = E.di_scene()
    goal = np.array([40, 40, 40, 0, 0, 0], np.float32)
    a = kpax.KPAX(cfg).plan_host(s, goal, obs)
    g, _ = gpu_plan(torch, cfg, s, goal, obs)
    assert (a.found, a.goal_idx, a.tree_size, a.iters, a.valid_expansions) == (g["found"], g["goal_idx"], g["tree_size"],
                                                                               g["iters"], g["valid_expansions"])


def test_plan_without_obstacles_and_with_tiny_tree(cuda):
    import torch

    cfg = small_di()
    cfg.max_tree_size = 300
    s = np.array([5, 5, 5, 0, 0, 0], np.float32)
    goal = np.array([95, 95, 95, 0, 0, 0], np.float32)
    empty = np.zeros((0, 6), np.float32)
    g, _ = gpu_plan(torch, cfg, s, goal, empty)
    o = O.plan(cfg, s, goal, empty, plan_idx=0)
    assert g["tree_full"] == 1 and g["tree_size"] == 300
    assert_plans_equal(g, o)


def expected_parents(rep_after, tree, cfg):
    """Frontier entries of the next iteration from the exported repeat counts (Planner.cu:68-80):
    with R entries and E taken, entry j is virtual entry floor(j*R/E); k children each."""
    rep = rep_after[:tree].astype(np.int64)
    R = int(rep.sum())
    if R == 0:
        return np.zeros(0, np.int64)
    B = min(cfg.expansions_per_iter, cfg.max_tree_size - tree)
    k = cfg.children_per_entry
    if R * k > B:
        k = max(1, B // R)
    E = min(R, B // k)
    v = (np.arange(E, dtype=np.int64) * R) // E
    node = np.searchsorted(np.cumsum(rep), v, side="right")
    return np.repeat(node, k)


@pytest.mark.parametrize("preset,scene", [(kpax.PRESET_QUAD, E.quad_scene), (kpax.PRESET_DUBINS, E.dubins_scene)])
def test_iterations_teacher_forced(cuda, preset, scene):
    import torch

    cfg = kpax.preset(preset)
    cfg.unroll_iters = 1
    obs, s, goal = scene()
    n1, P, S = kpax.sizes(cfg)
    sd = cfg.state_dim
    pl = kpax.KPAX(cfg)
    pl.debug_capture(True)
    d_obs = torch.from_numpy(obs).cuda()
    pl.begin(s, goal, d_obs.data_ptr(), obs.shape[0])
    table = O.region_table(cfg)
    flips_total = 0
    for it in range(1, 5):
        rows, parents, _ = pl.export_tree()
        counter0, valid0, scores0, bits0 = pl.export_regions()
        rep, _ = pl.export_frontier(rows.shape[0])
        # pending repeat counts resolve against the counters as they stand (KPAX.cu:476-479)
        rep = rep.astype(np.int64)
        pend = rep == 255
        r1_tree = O.regions(cfg, rows)[0]
        rep[pend] = np.where(valid0[r1_tree[pend]] < cfg.sparse_valid_threshold, cfg.sparse_repeat, 1)
        want_par = expected_parents(rep, rows.shape[0], cfg)
        pl.iterate(1)
        c_rows, c_valid, c_r1, c_r2, c_next, c_par = pl.export_children()
        assert np.array_equal(c_par, want_par), f"iteration {it}: parent assignment differs"
        n = c_par.size
        draws = np.stack([O.child_draws(cfg.seed, 0, it, n)]).reshape(n, 6)
        o_rows, o_valid, o_steps, margin, nonfin, kind = O.propagate(cfg, obs, rows[c_par, :sd], draws, nthreads=8)
        assert np.array_equal(bits(c_rows[:, sd:]), bits(o_rows[:, sd:]))  # controls + duration exact
        flips = np.where(c_valid != o_valid)[0]
        assert np.all(margin[flips] < NEAR_TOL), [(int(i), float(margin[i])) for i in flips if margin[i] >= NEAR_TOL]
        flips_total += flips.size
        same = np.setdiff1d(np.arange(n), flips)
        err = np.abs(c_rows[same, :sd].astype(np.float64) - o_rows[same, :sd]) / np.maximum(np.abs(o_rows[same, :sd]), 1.0)
        far = margin[same] >= NEAR_TOL
        assert err[far].max(initial=0.0) <= REL_TOL, err[far].max()
        # regions of the GPU's own child states are bit-exact
        g1, g2 = O.regions(cfg, c_rows)
        assert np.array_equal(g1, c_r1) and np.array_equal(g2, c_r2)
        # frontier mark with the scores and the R2 snapshot at the start of the iteration
        seen = (bits0[c_r2 >> 5] >> (c_r2 & 31)) & 1
        want_next = (c_valid == 1) & ((draws[:, 5] < scores0[c_r1]) | (seen == 0))
        assert np.array_equal(c_next.astype(bool), want_next)
        counter1, valid1, scores1, bits1 = pl.export_regions()
        assert np.array_equal(counter1 - counter0, np.bincount(c_r1, minlength=n1))
        assert np.array_equal(valid1 - valid0, np.bincount(c_r1[c_valid == 1], minlength=n1))
        assert np.array_equal(bits(scores1), bits(O.scores(cfg, counter1, valid1, bits1)))
        # appended children are exactly the marked ones, in child order
        rows2, parents2, costs2 = pl.export_tree()
        new = np.where(c_next)[0]
        t0 = rows.shape[0]
        assert rows2.shape[0] == t0 + new.size
        assert np.array_equal(bits(rows2[t0:]), bits(c_rows[new]))
        assert np.array_equal(parents2[t0:], c_par[new])
        d = rows2[t0:, :3] - goal[:3]
        assert np.array_equal(bits(costs2[t0:]), bits(np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])))
    print(f"near-boundary verdict flips over 4 iterations: {flips_total}")


def test_quad_plan_invariants(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter = 40
    obs, s, goal = E.quad_scene()
    g, _ = gpu_plan(torch, cfg, s, goal, obs)
    t = g["tree_size"]
    assert g["counter"].sum() == g["expansions"] and g["valid"].sum() == g["valid_expansions"]
    assert np.all(g["parents"][1:] < np.arange(1, t)) and g["parents"][0] == -1
    rows = g["rows"]
    assert np.all((rows[:, :3] >= 0) & (rows[:, :3] <= 100))
    assert np.all(np.isfinite(rows))
    r1, _ = O.regions(cfg, rows)
    assert np.array_equal(r1, g["r1"])
    if g["found"]:
        p = g["path"]
        assert np.linalg.norm(p[0, :3] - goal[:3]) < cfg.goal_thresh
        assert np.array_equal(p[-1, :12], s[:12])
    print({k: g[k] for k in ("found", "iters", "tree_size", "expansions", "valid_expansions")})

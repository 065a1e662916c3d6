"""Host-side logic of the learned proposal's data pipeline and of the autotuner's cache, on the CPU:
tree depths, hindsight relabelling, solution-path pairs, logit targets, summaries of evaluations,
parameter files, and cache keys / lookups."""
import json
import math

import numpy as np
import pytest

import kpax
import kpax_autotune as T
import kpax_learn as L


def chain_tree(n: int, branch_every: int = 0):
    """Rows of a small tree: node i's parent is i - 1 (a chain), or the root every `branch_every`."""
    parents = np.arange(-1, n - 1, dtype=np.int32)
    if branch_every:
        parents[branch_every::branch_every] = 0
    rows = np.zeros((n, 17), np.float32)
    rows[:, 0] = np.arange(n, dtype=np.float32)  # x grows with the index
    rows[:, 12:16] = np.arange(4 * n, dtype=np.float32).reshape(n, 4) / (4 * n)
    return rows, parents


def test_depths_of_chains_and_branches():
    _, par = chain_tree(7)
    assert np.array_equal(L.depths(par), np.arange(7))
    _, par = chain_tree(7, branch_every=3)  # 0-1-2, 0-3-4-5, 0-6
    assert np.array_equal(L.depths(par), [0, 1, 2, 1, 2, 3, 1])
    assert np.array_equal(L.depths(np.array([-1], np.int32)), [0])


@pytest.mark.parametrize("select", ["weighted", "far", "goal"])
def test_hindsight_pairs_are_tree_edges(select):
    rows, par = chain_tree(40, branch_every=9)
    rng = np.random.default_rng(0)
    goal = np.array([30.0, 0.0, 0.0], np.float32)
    x, g, y = L.hindsight_pairs(rows, par, 500, rng, select=select, goal=goal)
    assert x.shape == (500, 12) and g.shape == (500, 3) and y.shape == (500, 4)
    # every pair is (parent state, child controls) of one edge of the tree
    child = np.rint(y[:, 0] * 40).astype(int)  # rows[i, 12] = i / 40 in chain_tree(40)
    assert np.all(child >= 1) and np.array_equal(x[:, 0], rows[par[child], 0])
    if select == "goal":
        assert np.all(g == goal)
    else:  # the goal is a node on the edge's branch, at or below the child
        assert np.all(g[:, 0] >= rows[child, 0])


def test_hindsight_ray_goals_lie_on_the_ray():
    rows, par = chain_tree(30)
    x, g, _ = L.hindsight_pairs(rows, par, 200, np.random.default_rng(1), ray=True)
    dist = np.linalg.norm(g - x[:, :3], axis=1)
    assert np.all((dist >= 10.0 - 1e-3) & (dist <= 150.0 + 1e-3))
    assert np.allclose(g[:, 1:], 0.0) and np.all(g[:, 0] > x[:, 0])


def test_solution_pairs_walk_to_the_root():
    rows, par = chain_tree(6)
    goal = np.array([9.0, 8.0, 7.0, 0, 0, 0], np.float32)
    x, g, y = L.solution_pairs(rows, par, 5, goal)
    assert x.shape == (5, 12) and np.array_equal(x[:, 0], [4, 3, 2, 1, 0])
    assert np.all(g == goal[:3]) and np.array_equal(y, rows[[5, 4, 3, 2, 1], 12:16])
    assert L.solution_pairs(rows, par, 0, goal)[0].shape == (0, 12)


def test_logit_targets_invert_the_control_map():
    cfg = L.quad_config()
    u = np.array([[0.5, 0.25, 0.75, 0.5], [1e-9, 1.0, 0.5, 0.5]])
    lo, hi = np.array(cfg.ctrl_min[:4]), np.array(cfg.ctrl_max[:4])
    y = L.logit_targets((lo + u * (hi - lo)).astype(np.float32), cfg)
    assert y.shape == (2, 5) and np.all(y[:, 4] == 0)
    assert np.allclose(y[0, :4], [0.0, math.log(1 / 3), math.log(3), 0.0], atol=1e-5)
    edge = math.log(L.U_CLAMP / (1 - L.U_CLAMP))  # draws at the ends are clamped to [U_CLAMP, 1 - U_CLAMP]
    assert np.all(np.isfinite(y)) and y[1, 0] == pytest.approx(edge, rel=1e-5) and y[1, 1] == pytest.approx(-edge, rel=1e-5)
    assert L.loss_mask(cfg) == [1.0, 1.0, 1.0, 1.0, 0.0]  # fixed-step model: no duration term


def test_summary_counts_unsolved_plans_as_infinite():
    res = [{"found": 1, "ms": 2.0, "valid": 10}, {"found": 0, "ms": 8.0, "valid": 30}, {"found": 1, "ms": 4.0, "valid": 20}]
    s = L.summarize(res)
    assert s["n"] == 3 and s["success"] == pytest.approx(2 / 3)
    assert s["p50_ms"] == 4.0 and s["p95_ms"] == math.inf and s["p50_ms_solved"] == 3.0
    assert s["valid_per_s"] == pytest.approx(60 / 14e-3)


def test_parameter_files_round_trip(tmp_path):
    w = L.init_params(3)
    assert w.dtype == np.float32 and w.size == L.NUM_PARAMS and np.all(np.isfinite(w))
    L.save_params(tmp_path / "w.npz", w, {"rounds": [1, 2]})
    w2, meta = L.load_params(tmp_path / "w.npz")
    assert np.array_equal(w, w2) and meta == {"rounds": [1, 2]}


def test_autotune_cache_keys_and_lookup(tmp_path, monkeypatch):
    cfg = kpax.preset(kpax.PRESET_QUAD)
    assert T.obs_bucket(0) == 0 and T.obs_bucket(1000) == 9 and T.obs_bucket(1024) == 10
    key = T.workload_key(cfg, 1000)
    assert key == "model3|exp65536|obs2^9"
    monkeypatch.setattr(T, "gpu_key", lambda: "TestGPU|sm100|148SM")
    path = tmp_path / "cache.json"
    assert T.tuned(cfg, 1000, path)[1] is None  # nothing cached yet
    best = {"block_size": 256, "samples_per_thread": 2, "hash_cell_size": 10.0}
    T.store("TestGPU|sm100|148SM", key, best, [{"ms_per_iter": 0.1, **best}], path)
    tcfg, got = T.tuned(cfg, 1000, path)
    assert got == best and (tcfg.block_size, tcfg.samples_per_thread, tcfg.hash_cell_size) == (256, 2, 10.0)
    assert T.tuned(cfg, 5000, path)[1] is None  # another obstacle bucket is not covered
    assert json.loads(path.read_text())["TestGPU|sm100|148SM"][key]["best"] == best

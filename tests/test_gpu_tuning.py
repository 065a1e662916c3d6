"""Launch parameters the autotuner searches (expansion block size, samples per thread, hash cell
size, iterations per graph) must not change a plan: every combination expands the identical tree,
and the double integrator still matches the CPU oracle bit for bit."""
import numpy as np
import pytest

import kpax
import kpax_autotune as T
import kpax_envs as E
import oracle as O

pytestmark = pytest.mark.gpu

COMBOS = [
    {"block_size": 128, "samples_per_thread": 1, "hash_cell_size": 2.5},
    {"block_size": 256, "samples_per_thread": 2, "hash_cell_size": 10.0},
    {"block_size": 512, "samples_per_thread": 3, "hash_cell_size": 5.0, "unroll_iters": 3},
    {"block_size": 448, "samples_per_thread": 8, "hash_cell_size": 7.0},
]


def plan_rows(torch, cfg, obs, s, g):
    pl = kpax.KPAX(cfg)
    d = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    r = pl.plan(s, g, d.data_ptr(), obs.shape[0])
    rows, parents, costs = pl.export_tree()
    return r, rows, parents


@pytest.mark.parametrize("preset,scene", [(kpax.PRESET_QUAD, E.quad_scene), (kpax.PRESET_DUBINS, E.dubins_scene)])
def test_tuning_parameters_leave_plans_unchanged(cuda, preset, scene):
    import torch

    cfg = kpax.preset(preset)
    cfg.max_iter = 12
    obs, s, g = scene()
    r0, rows0, par0 = plan_rows(torch, cfg, obs, s, g)
    for params in COMBOS:
        r, rows, par = plan_rows(torch, T.apply(cfg, params), obs, s, g)
        assert (r.tree_size, r.valid_expansions, r.iters) == (r0.tree_size, r0.valid_expansions, r0.iters), params
        assert np.array_equal(rows.view(np.uint32), rows0.view(np.uint32)) and np.array_equal(par, par0), params


def test_tuned_double_integrator_matches_oracle(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_DI)
    cfg.max_tree_size = 1 << 15
    cfg.expansions_per_iter = 1 << 12
    cfg.max_iter = 40
    obs, s, g = E.di_scene()
    tcfg = T.apply(cfg, {"block_size": 128, "samples_per_thread": 4, "hash_cell_size": 2.5})
    r, rows, par = plan_rows(torch, tcfg, obs, s, g)
    o = O.plan(cfg, s, g, obs, plan_idx=0)
    assert r.tree_size == o["tree_size"] and r.valid_expansions == o["valid_expansions"]
    assert np.array_equal(rows.view(np.uint32), np.ascontiguousarray(o["rows"], np.float32).view(np.uint32))
    assert np.array_equal(par, o["parents"])


@pytest.mark.parametrize("split", [False, True])
def test_timed_iterations_expand_the_same_tree(cuda, split):
    """The benchmark's timed path (direct launches, with or without events between the chained
    kernels, an L2-evicting write before each iteration) expands the tree the captured plan loop
    expands for the same iterations."""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter = 10
    obs, s, g = E.quad_scene()
    d = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    ref = kpax.KPAX(cfg)
    ref.begin(s, g, d.data_ptr(), obs.shape[0])
    ref.iterate(cfg.max_iter)
    rows0, par0, _ = ref.export_tree()
    pl = kpax.KPAX(cfg)
    pl.begin(s, g, d.data_ptr(), obs.shape[0])
    times, tot = pl.iterate_timed(cfg.max_iter, 1 << 20, split=split)
    rows, par, _ = pl.export_tree()
    assert times.shape == (cfg.max_iter, 4) and np.all(times[:, 0] > 0)
    assert np.all(times[:, 1:] > 0) if split else np.all(times[:, 1:] == 0)
    assert tot["appended"] == rows.shape[0] - 1
    assert np.array_equal(rows.view(np.uint32), rows0.view(np.uint32)) and np.array_equal(par, par0)
    ref.close()
    pl.close()

"""Batched planning (many independent queries per kernel launch) against single plans.

A query planned inside a mixed batch (double integrator, Dubins and quadrotor queries with their
own obstacles, trees and budgets) must give exactly the tree and result of the same query planned
alone: the kernels, draws and append order do not depend on the other queries."""
import numpy as np
import pytest

import kpax
import kpax_envs as E

pytestmark = pytest.mark.gpu


def _queries():
    qs = []
    di = kpax.preset(kpax.PRESET_DI)
    di.max_tree_size, di.expansions_per_iter, di.max_iter = 1 << 14, 1 << 11, 40
    di.v_min, di.v_max = -5.0, 5.0
    for i in range(3):
        di.ctrl_min[i], di.ctrl_max[i] = -4.0, 4.0
    obs, s, _ = E.di_scene()
    qs.append((di, obs, s, np.array([40, 40, 40, 0, 0, 0], np.float32)))
    di2 = kpax.preset(kpax.PRESET_DI)
    di2.max_tree_size, di2.expansions_per_iter, di2.max_iter, di2.seed = 1 << 13, 1 << 10, 30, 7
    qs.append((di2, obs, s, np.array([95, 95, 95, 0, 0, 0], np.float32)))
    du = kpax.preset(kpax.PRESET_DUBINS)
    du.max_tree_size, du.expansions_per_iter, du.max_iter = 1 << 16, 1 << 13, 12
    dobs, ds, dg = E.dubins_scene()
    qs.append((du, dobs, ds, dg))
    qu = kpax.preset(kpax.PRESET_QUAD)
    qu.max_tree_size, qu.expansions_per_iter, qu.max_iter = 1 << 16, 1 << 13, 10
    qobs, qs_, qg = E.quad_scene(n_total=300)
    qs.append((qu, qobs, qs_, qg))
    qu2 = kpax.preset(kpax.PRESET_QUAD)
    qu2.max_tree_size, qu2.expansions_per_iter, qu2.max_iter, qu2.seed = 1 << 15, 1 << 12, 8, 11
    qs.append((qu2, np.zeros((0, 6), np.float32), qs_, qg))
    return qs


def test_batch_matches_single_plans(cuda):
    import torch

    qs = _queries()
    d_obs = [torch.from_numpy(np.ascontiguousarray(o, np.float32)).cuda() if o.size else None for _, o, _, _ in qs]
    ptrs = [d.data_ptr() if d is not None else 0 for d in d_obs]
    batch = kpax.Batch([c for c, _, _, _ in qs])
    res, stats = batch.plan([s for _, _, s, _ in qs], [g for _, _, _, g in qs], ptrs, [o.shape[0] for _, o, _, _ in qs])
    assert stats["found"] == sum(r["found"] for r in res)
    assert stats["valid_expansions"] == sum(r["valid_expansions"] for r in res)
    for q, (cfg, obs, s, g) in enumerate(qs):
        pl = kpax.KPAX(cfg)
        r = pl.plan(s, g, ptrs[q], obs.shape[0])
        single = {f: getattr(r, f) for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full",
                                              "expansions", "valid_expansions")}
        assert {f: res[q][f] for f in single} == single, (q, single, res[q])
        if r.path_len:
            assert np.array_equal(res[q]["path"].view(np.uint32), pl.h_controlPathToGoal_.view(np.uint32))
        assert res[q]["ms"] > 0.0
        pl.close()
    assert res[0]["found"] == 1  # the fast double integrator reaches its goal
    batch.close()


def test_second_batch_plan_uses_a_new_random_stream(cuda):
    import torch

    cfg, obs, s, g = _queries()[0]
    d_obs = torch.from_numpy(obs).cuda()
    batch = kpax.Batch([cfg, cfg])
    r1, _ = batch.plan([s, s], [g, g], [d_obs.data_ptr()] * 2, [obs.shape[0]] * 2)
    r2, _ = batch.plan([s, s], [g, g], [d_obs.data_ptr()] * 2, [obs.shape[0]] * 2)
    assert r1[0]["tree_size"] == r1[1]["tree_size"]  # same config and plan index: same plan
    pl = kpax.KPAX(cfg)
    pl.plan(s, g, d_obs.data_ptr(), obs.shape[0])
    second = pl.plan(s, g, d_obs.data_ptr(), obs.shape[0])  # plan index 1
    assert (second.tree_size, second.iters, second.valid_expansions) == (r2[0]["tree_size"], r2[0]["iters"],
                                                                          r2[0]["valid_expansions"])
    batch.close()

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


@pytest.mark.parametrize("block", [0, 256])
def test_persistent_stages_over_many_uneven_queries(cuda, block):
    """24 queries of uneven size in one batch (the stages run as persistent launches over all
    queries' work, with per-query offsets): trees from 2^10 to 2^16 nodes, some filling before
    their goal, some reaching it in a few iterations (at least the fast double integrator added last),
    some planning with no obstacles.  Every query must give its single plan, at the default
    expansion tiles and at the 256-child tiles the batch expansion runs at four or five CTAs per SM."""
    import torch

    rng = np.random.default_rng(5)
    dobs, ds, dg = E.dubins_scene()
    qobs, qs_, qg = E.quad_scene(n_total=300)
    obs0, s0, _ = E.di_scene()
    qs = []
    for i in range(24):
        kind = i % 3
        if kind == 0:
            c = kpax.preset(kpax.PRESET_DI)
            c.max_tree_size = int(2 ** rng.integers(10, 15))
            c.expansions_per_iter = min(c.max_tree_size, 1 << 11)
            c.max_iter, c.seed = 25, 100 + i
            c.v_min, c.v_max = -5.0, 5.0
            for k in range(3):
                c.ctrl_min[k], c.ctrl_max[k] = -4.0, 4.0
            goal = np.array([rng.uniform(20, 60), rng.uniform(20, 60), rng.uniform(20, 60), 0, 0, 0], np.float32)
            qs.append((c, obs0 if i % 2 else np.zeros((0, 6), np.float32), s0, goal))
        elif kind == 1:
            c = kpax.preset(kpax.PRESET_DUBINS)
            c.max_tree_size = int(2 ** rng.integers(12, 17))
            c.expansions_per_iter = min(c.max_tree_size, 1 << 12)
            c.max_iter, c.seed = 10, 200 + i
            qs.append((c, dobs, ds, dg))
        else:
            c = kpax.preset(kpax.PRESET_QUAD)
            c.max_tree_size = int(2 ** rng.integers(12, 17))
            c.expansions_per_iter = min(c.max_tree_size, 1 << 12)
            c.max_iter, c.seed = 8, 300 + i
            qs.append((c, qobs, qs_, qg))
    qs.append(_queries()[0])  # the fast double integrator that reaches its goal in a few iterations
    if block:  # the batch expansion's 256-child tiles (four or five CTAs per SM)
        for c, _, _, _ in qs:
            c.block_size = block
    d_obs = [torch.from_numpy(np.ascontiguousarray(o, np.float32)).cuda() if o.size else None for _, o, _, _ in qs]
    ptrs = [d.data_ptr() if d is not None else 0 for d in d_obs]
    batch = kpax.Batch([c for c, _, _, _ in qs])
    res, stats = batch.plan([s for _, _, s, _ in qs], [g for _, _, _, g in qs], ptrs, [o.shape[0] for _, o, _, _ in qs])
    full = found = 0
    for q, (cfg, obs, s, g) in enumerate(qs):
        pl = kpax.KPAX(cfg)
        r = pl.plan(s, g, ptrs[q], obs.shape[0])
        single = {f: getattr(r, f) for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full",
                                              "expansions", "valid_expansions", "path_cost")}
        assert {f: res[q][f] for f in single} == single, (q, single, {f: res[q][f] for f in single})
        full += int(r.tree_full)
        found += int(r.found)
        pl.close()
    assert full >= 1 and found >= 1, (full, found)  # both early exits are exercised
    assert stats["found"] == found
    batch.close()


def test_learned_proposal_in_a_batch_matches_single_plans(cuda):
    """With the learned proposal on, a batch runs one proposal launch over the entries of all its
    quadrotor queries (tiles shared by every CTA); each query's records, and so its plan, equal
    those of the query planned alone."""
    import torch

    import kpax_learn as L

    net = L.load_network(L.DEFAULT_WEIGHTS)
    qobs, s, g = E.quad_scene(n_total=300)
    qs = []
    for i, (budget, cap, iters) in enumerate(((1 << 13, 1 << 16, 8), (1 << 11, 1 << 15, 10), (1 << 12, 1 << 16, 6))):
        c = kpax.preset(kpax.PRESET_QUAD)
        c.max_tree_size, c.expansions_per_iter, c.max_iter, c.seed = cap, budget, iters, 21 + i
        qs.append((c, qobs if i != 1 else np.zeros((0, 6), np.float32), s, g))
    qs.append(_queries()[0])  # a double integrator query beside them
    d_obs = [torch.from_numpy(np.ascontiguousarray(o, np.float32)).cuda() if o.size else None for _, o, _, _ in qs]
    ptrs = [d.data_ptr() if d is not None else 0 for d in d_obs]
    batch = kpax.Batch([c for c, _, _, _ in qs])
    batch.set_proposal(net, 0.3)
    res, _ = batch.plan([s for _, _, s, _ in qs], [g for _, _, _, g in qs], ptrs, [o.shape[0] for _, o, _, _ in qs])
    for q, (cfg, obs, s_, g_) in enumerate(qs):
        pl = kpax.KPAX(cfg)
        if cfg.model == kpax.MODEL_QUADROTOR:
            pl.set_proposal(net, 0.3)
        r = pl.plan(s_, g_, ptrs[q], obs.shape[0])
        single = {f: getattr(r, f) for f in ("found", "goal_idx", "tree_size", "iters", "expansions", "valid_expansions")}
        assert {f: res[q][f] for f in single} == single, (q, single, res[q])
        pl.close()
    batch.close()


def test_plans_do_not_depend_on_the_tile_size(cuda):
    """Every model's step spells out its roundings, so a query's plan is the same whichever
    kernel expands it: batches at 448- and 256-child tiles (one and four or five CTAs per SM) and
    single plans at 128-child tiles give the same trees."""
    import torch

    qs = _queries()
    d_obs = [torch.from_numpy(np.ascontiguousarray(o, np.float32)).cuda() if o.size else None for _, o, _, _ in qs]
    ptrs = [d.data_ptr() if d is not None else 0 for d in d_obs]
    fields = ("found", "goal_idx", "tree_size", "iters", "expansions", "valid_expansions", "path_cost")
    out = []
    for block in (448, 256):
        cfgs = []
        for c, _, _, _ in qs:
            c.block_size = block
            cfgs.append(c)
        batch = kpax.Batch(cfgs)
        res, _ = batch.plan([s for _, _, s, _ in qs], [g for _, _, _, g in qs], ptrs, [o.shape[0] for _, o, _, _ in qs])
        out.append([{f: r[f] for f in fields} for r in res])
        batch.close()
    assert out[0] == out[1]
    for q, (cfg, obs, s, g) in enumerate(qs):
        cfg.block_size = 128
        pl = kpax.KPAX(cfg)
        r = pl.plan(s, g, ptrs[q], obs.shape[0])
        assert {f: getattr(r, f) for f in fields} == out[0][q], q
        pl.close()

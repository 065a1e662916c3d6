"""The fused iteration kernel (k_iterate: frontier count, entry list, expansion and region scores of
one iteration in one persistent launch, separated by bounded grid-wide barriers) against the
per-stage kernels (k_frontier_count, k_frontier_write, k_expand, k_scores): the same plan, bit for
bit — tree rows, parents, costs, region counters, scores, R2 bits, frontier repeats and path — for
every model, for block sizes with one and several CTAs per SM, for budgets that take several
expansion rounds per CTA, for a tree that fills, and with goal-progress pruning."""
from pathlib import Path

import numpy as np
import pytest

import kpax
import kpax_envs as E

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).parent / "golden"


def run(torch, cfg, obs, s, g, kernels, net=None):
    c = cfg.copy()
    c.iteration_kernels = kernels
    pl = kpax.KPAX(c)
    if net is not None:
        pl.set_proposal(net, 0.3)
    d = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    l0 = kpax.kernel_launches()
    r = pl.plan(s, g, d.data_ptr(), obs.shape[0])
    launches = kpax.kernel_launches() - l0
    res = (r.found, r.goal_idx, r.path_len, r.tree_size, r.iters, r.tree_full, r.expansions, r.valid_expansions,
           r.path_cost)
    path = pl.h_controlPathToGoal_.copy()
    rows, parents, costs = pl.export_tree()
    counter, valid, scores, bits = pl.export_regions()
    rep, r1 = pl.export_frontier(res[3])
    out = {"res": res, "rows": rows.view(np.uint32), "parents": parents, "costs": costs.view(np.uint32), "rep": rep,
           "r1": r1, "path": path.view(np.uint32), "counter": counter, "valid": valid, "scores": scores.view(np.uint32),
           "r2_bits": bits, "launches": launches}
    pl.close()
    return out


def same(a, b):
    for k in a:
        if k == "launches":
            continue
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], (k, a[k], b[k])


CASES = {
    "di": (kpax.PRESET_DI, E.di_scene, {"max_tree_size": 1 << 15, "expansions_per_iter": 1 << 12, "max_iter": 40}),
    "dubins": (kpax.PRESET_DUBINS, E.dubins_scene, {"max_iter": 14}),
    "quad": (kpax.PRESET_QUAD, E.quad_scene, {"max_iter": 14}),
    "quad_bs128": (kpax.PRESET_QUAD, E.quad_scene, {"max_iter": 10, "block_size": 128}),
    "quad_bs256_spt2": (kpax.PRESET_QUAD, E.quad_scene, {"max_iter": 10, "block_size": 256, "samples_per_thread": 2}),
    "quad_rounds": (kpax.PRESET_QUAD, E.quad_scene, {"max_iter": 8, "expansions_per_iter": 1 << 18}),
    "dubins_fills": (kpax.PRESET_DUBINS, E.dubins_scene, {"max_iter": 40, "max_tree_size": 1 << 16,
                                                          "expansions_per_iter": 1 << 14}),
    "di_pruned": (kpax.PRESET_DI, E.di_scene, {"max_tree_size": 1 << 15, "expansions_per_iter": 1 << 12, "max_iter": 40,
                                               "prune": 1}),
    "quad_ref_block": (kpax.PRESET_QUAD_REF, None, {"max_iter": 12}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fused_iteration_equals_per_stage_kernels(cuda, name):
    import torch

    preset, scene, edits = CASES[name]
    cfg = kpax.preset(preset)
    for k, v in edits.items():
        setattr(cfg, k, v)
    if scene is None:  # the reference's own quadrotor block on its quadTrees scene
        obs = np.load(GOLDEN / "quad_quadTrees.npz")["obstacles"]
        s = np.zeros(cfg.sample_dim, np.float32)
        g = np.zeros(cfg.sample_dim, np.float32)
        s[:3], g[:3] = (10, 8, 5), (80, 95, 90)
    else:
        obs, s, g = scene()
    fused = run(torch, cfg, obs, s, g, 0)
    staged = run(torch, cfg, obs, s, g, 1)
    same(fused, staged)
    # the fused path launched one kernel per iteration (plus the plan's begin and path kernels)
    iters = fused["res"][4]
    assert fused["launches"] < staged["launches"], (fused["launches"], staged["launches"])
    assert fused["res"][3] > 1 and iters >= 1


@pytest.mark.parametrize("block", [0, 128])
def test_fused_parts_around_the_proposal_pass_equal_per_stage_kernels(cuda, block):
    """With the learned proposal a single plan runs the fused iteration in two launches around the
    tensor-core pass (frontier count and entry list; expansion and scores): the same plan, bit for
    bit, as the per-stage kernels with the same pass between them, in three launches per
    iteration instead of five."""
    import torch

    import kpax_learn as L

    net = L.load_network(L.DEFAULT_WEIGHTS)
    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter, cfg.max_tree_size, cfg.expansions_per_iter = 12, 1 << 18, 1 << 13
    if block:
        cfg.block_size = block
    obs, s, g = E.quad_scene(n_total=300)
    fused = run(torch, cfg, obs, s, g, 0, net)
    staged = run(torch, cfg, obs, s, g, 1, net)
    same(fused, staged)
    iters = fused["res"][4]
    assert iters >= 2 and fused["launches"] < staged["launches"], (iters, fused["launches"], staged["launches"])


def test_fused_timed_iterations_report_phase_times(cuda):
    """With the fused kernel the split timing comes from the device clock: every phase positive,
    their sum within the event time of the launch, and the tree the same as the per-stage path's."""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter = 10
    obs, s, g = E.quad_scene()
    d = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    trees = []
    for kernels in (0, 1):
        c = cfg.copy()
        c.iteration_kernels = kernels
        pl = kpax.KPAX(c)
        pl.begin(s, g, d.data_ptr(), obs.shape[0])
        times, tot = pl.iterate_timed(8, 1 << 20, split=True)
        rows, par, _ = pl.export_tree()
        trees.append((rows.view(np.uint32), par, tot["valid"], tot["steps"]))
        if kernels == 0:
            assert np.all(times[:, 1:] > 0)
            assert float(times[:, 1:].sum(axis=1).mean()) <= float(times[:, 0].mean()) * 1.05
        pl.close()
    assert np.array_equal(trees[0][0], trees[1][0]) and np.array_equal(trees[0][1], trees[1][1])
    assert trees[0][2:] == trees[1][2:]

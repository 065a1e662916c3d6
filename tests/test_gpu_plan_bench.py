"""planBench's per-iteration dumps (KPAX.cu:243-300, writeDeviceVectorsToCSV 545-633): the
directory layout and file names of the reference, one file of MAX_TREE_SIZE tree rows and parents
per iteration, one row per iteration of the region and frontier buffers, one value per iteration
of the frontier size, tree size and children expanded, and the same plan as kpax_plan."""
import numpy as np
import pytest

import kpax
import kpax_envs as E

pytestmark = pytest.mark.gpu


def small_di():
    cfg = kpax.preset(kpax.PRESET_DI)
    cfg.max_tree_size = 1 << 12
    cfg.expansions_per_iter = 1 << 9
    cfg.max_iter = 6
    return cfg


def test_plan_bench_dumps(cuda, tmp_path):
    import torch

    cfg = small_di()
    obs, s, g = E.di_scene()
    d_obs = torch.from_numpy(obs).cuda()
    n1, _, S = kpax.sizes(cfg)
    cap = cfg.max_tree_size
    pl = kpax.KPAX(cfg)
    r = pl.planBench(s, g, d_obs.data_ptr(), obs.shape[0], 3, tmp_path)
    rows_now, par_now, _ = pl.export_tree()
    ref = kpax.KPAX(cfg)
    r0 = ref.plan(s, g, d_obs.data_ptr(), obs.shape[0])
    rows0, par0, _ = ref.export_tree()
    assert (r.iters, r.tree_size, r.found) == (r0.iters, r0.tree_size, r0.found)
    assert np.array_equal(rows_now.view(np.uint32), rows0.view(np.uint32)) and np.array_equal(par_now, par0)

    data = tmp_path / "Data"
    d = lambda name: data / name / f"{name}3"  # noqa: E731
    its = r.iters
    assert sorted(p.name for p in d("Samples").iterdir()) == sorted(f"samples{k}.csv" for k in range(1, its + 1))
    last = np.loadtxt(d("Samples") / f"samples{its}.csv", delimiter=",", ndmin=2)
    assert last.shape == (cap, S)
    assert np.allclose(last[: r.tree_size], rows0, atol=5.1e-7 * np.maximum(1, np.abs(rows0)).max(), rtol=0)
    assert not last[r.tree_size:].any()
    parents = np.loadtxt(d("Parents") / f"parents{its}.csv", dtype=np.int64)
    assert parents.shape == (cap,) and np.array_equal(parents[: r.tree_size], par0) and np.all(parents[r.tree_size:] == -1)

    counter = np.loadtxt(d("TotalCountPerVertex") / "totalCountPerVertex.csv", delimiter=",", dtype=np.int64, ndmin=2)
    valid = np.loadtxt(d("ValidCountPerVertex") / "validCountPerVertex.csv", delimiter=",", dtype=np.int64, ndmin=2)
    scores = np.loadtxt(d("VertexScores") / "vertexScores.csv", delimiter=",", ndmin=2)
    frontier = np.loadtxt(d("Frontier") / "frontier.csv", delimiter=",", dtype=np.int64, ndmin=2)
    repeat = np.loadtxt(d("FrontierRepeatCount") / "frontierRepeatCount.csv", delimiter=",", dtype=np.int64, ndmin=2)
    assert counter.shape == valid.shape == scores.shape == (its, n1)
    assert frontier.shape == repeat.shape == (its, cap)
    c_end, v_end, s_end, _ = ref.export_regions()
    assert np.array_equal(counter[-1], c_end) and np.array_equal(valid[-1], v_end)
    assert np.allclose(scores[-1], s_end, atol=5.1e-7, rtol=0)
    assert np.all(np.diff(counter.sum(axis=1)) > 0)  # counters accumulate over the iterations
    assert np.array_equal(frontier, (repeat > 0).astype(np.int64)) and np.all(repeat < 255)

    tree = np.loadtxt(d("TreeSize") / "treeSize.csv", dtype=np.int64, ndmin=1)
    fsize = np.loadtxt(d("FrontierSize") / "frontierSize.csv", dtype=np.int64, ndmin=1)
    expanded = np.loadtxt(d("ExpandedNodes") / "expandedNodes.csv", dtype=np.int64, ndmin=1)
    assert tree.shape == fsize.shape == expanded.shape == (its,)
    assert tree[-1] == r.tree_size and np.all(np.diff(tree) >= 0)
    assert fsize[0] == 1 and np.array_equal(fsize[1:], frontier[:-1].sum(axis=1))
    assert counter[0].sum() == expanded[0] and np.array_equal(np.diff(counter.sum(axis=1)), expanded[1:])
    assert (d("ControlPathToGoal") / "controlPathToGoal.csv").exists() == bool(r.found)
    secs = np.loadtxt(data / "ExecutionTime" / "executionTime.csv", ndmin=1)
    assert secs.shape == (1,) and secs[0] > 0

    # a second run with the same index starts its per-run files afresh
    r2 = pl.planBench(s, g, d_obs.data_ptr(), obs.shape[0], 3, tmp_path)
    again = np.loadtxt(d("TotalCountPerVertex") / "totalCountPerVertex.csv", delimiter=",", dtype=np.int64, ndmin=2)
    assert again.shape == (r2.iters, n1)
    assert np.loadtxt(data / "ExecutionTime" / "executionTime.csv", ndmin=1).shape == (2,)
    pl.close()
    ref.close()

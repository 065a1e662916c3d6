"""ReKinoLite (src/ReKino/ReKinoLite.cu) on the library's kernels against the oracle restatement.

Double integrator: the winning warp, its iteration and its whole path are bit-exact (greedy and
epsilon-greedy, one and several samples per thread).  Quadrotor: the path starts at the start
state, ends in the goal ball, and every segment is the FP64 integration of its parent with the
row's controls (within the FP32-vs-FP64 tolerance)."""
import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spt,eps", [(1, 0.0), (2, 0.3)])
def test_di_rekino_bit_exact(cuda, spt, eps):
    import torch

    cfg = kpax.preset(kpax.PRESET_DI)
    obs, s, _ = E.di_scene()
    g = np.array([30, 30, 30, 0, 0, 0], np.float32)
    d_obs = torch.from_numpy(obs).cuda()
    rk = kpax.ReKinoLite(cfg, num_warps=64, samples_per_thread=spt, epsilon_greedy=eps, max_iterations=2000)
    r, path = rk.plan(s, g, d_obs.data_ptr(), obs.shape[0])
    o = O.rekino(cfg, s, g, obs, num_warps=64, spt=spt, eps=eps, max_iter=2000)
    assert r.found == 1 and o["found"] == 1
    assert (r.goal_idx, r.iters - 1) == (o["warp"], o["iter"])
    assert np.array_equal(path[::-1].view(np.uint32), o["path"].view(np.uint32))
    assert np.linalg.norm(path[0, :3] - g[:3]) < cfg.goal_thresh
    assert r.expansions >= 64 * 32 * spt * (o["iter"] + 1) // 64  # every warp ran at least the winner's iterations
    # a second planner object draws the same streams (plan index 0)
    r2, path2 = kpax.ReKinoLite(cfg, num_warps=64, samples_per_thread=spt, epsilon_greedy=eps,
                                max_iterations=2000).plan(s, g, d_obs.data_ptr(), obs.shape[0])
    assert np.array_equal(path2.view(np.uint32), path.view(np.uint32))


def test_quad_rekino_path_is_a_valid_trajectory(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs, s, _ = E.quad_scene()
    g = s.copy()
    g[:3] = (14.0, 12.0, 12.0)
    d_obs = torch.from_numpy(obs).cuda()
    rk = kpax.ReKinoLite(cfg, num_warps=256, max_iterations=4000)
    r, path = rk.plan(s, g, d_obs.data_ptr(), obs.shape[0])
    assert r.found == 1, "ReKinoLite did not reach a goal 9 m away"
    rows = path[::-1]
    assert np.array_equal(rows[0, :12], s[:12])
    assert np.linalg.norm(rows[-1, :3] - g[:3]) < cfg.goal_thresh
    for a, b in zip(rows[:-1], rows[1:]):
        steps = int(round(float(b[16]) / cfg.step_size))
        x = O.integrate_f64(cfg, a[:12], b[12:], steps, mode=0)
        assert np.all(np.abs(x - b[:12]) <= 1e-4 * np.maximum(np.abs(x), 1.0))
    print({"iters": r.iters, "path_len": r.path_len, "ms": r.ms, "samples": r.expansions})


def test_give_up_deadline_stops_every_warp(cuda):
    """The 6-second give-up of ReKinoLite (ReKinoLite.cu:120-124, 300-313) is a %globaltimer
    deadline checked every 100 iterations: with a 0.1 ms deadline and a goal no state can reach
    (outside the workspace, which every propagated state must stay in), every warp stops at the
    first check past the deadline: a whole number of 100-iteration rounds of 32 samples per warp,
    at least one round each and far below the 20000 iterations, and the plan ends in milliseconds.
    (A warp whose first 100 iterations take less than the deadline checks again 100 iterations
    later, so the count is not pinned to exactly one round.)"""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs, s, g = E.quad_scene()
    g = g.copy()
    g[:3] = (500.0, 500.0, 500.0)
    d_obs = torch.from_numpy(obs).cuda()
    rk = kpax.ReKinoLite(cfg, num_warps=64, timeout_ms=0.1, max_iterations=20000)
    r, path = rk.plan(s, g, d_obs.data_ptr(), obs.shape[0])
    assert r.found == 0 and path.shape[0] == 0
    rounds, rem = divmod(r.expansions, 100 * 32)
    assert rem == 0 and 64 <= rounds <= 64 * 20, r.expansions  # every warp: 1 to 20 rounds of 100
    assert r.ms < 500.0, r.ms

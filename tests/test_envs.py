"""Seeded scene generators of the benchmark configurations (CPU): every family is deterministic in
its seed and has the properties its configuration states (box sizes and bounds, free start and
goal, the windowed wall's openings, start-goal separations, batch mixes)."""
import numpy as np
import pytest

import kpax
import kpax_envs as E


def covers_any(obs, p):
    return any(E._covers(b, p) for b in obs)


@pytest.mark.parametrize("make", [lambda s: E.random_boxes(50, s), lambda s: E.forest(200, s), lambda s: E.building(300, s),
                                  lambda s: E.learned_family(s)[0]])
def test_generators_are_deterministic_in_the_seed(make):
    a, b, c = make(5), make(5), make(6)
    assert a.dtype == np.float32 and np.array_equal(a, b) and not np.array_equal(a, c)


def test_random_boxes_sizes_and_avoidance():
    p = np.array([50.0, 50.0, 50.0], np.float32)
    obs = E.random_boxes(400, 3, avoid=(p,))
    side = obs[:, 3:] - obs[:, :3]
    centre = (obs[:, 3:] + obs[:, :3]) / 2
    assert obs.shape == (400, 6) and np.all(side >= 5 - 1e-4) and np.all(side <= 15 + 1e-4)
    assert np.all((centre >= 0) & (centre <= 100)) and not covers_any(obs, p)


def test_benchmark_scenes_leave_start_and_goal_free():
    for scene, n in ((E.di_scene, 20), (E.dubins_scene, None), (E.quad_scene, 1000)):
        obs, s, g = scene()
        if n is not None:
            assert obs.shape[0] == n
        assert not covers_any(obs, s[:3]) and not covers_any(obs, g[:3])


def test_forest_columns():
    obs = E.forest(200, 1)
    fp, h = obs[:, 3:5] - obs[:, :2], obs[:, 5]
    assert np.all(obs[:, 2] == 0) and np.all((h >= 20) & (h <= 100)) and np.all((fp >= 2 - 1e-4) & (fp <= 6 + 1e-4))


def test_windowed_wall_has_four_open_windows():
    wall = E.wall_with_windows()
    assert np.all(wall[:, 0] == E.WALL_X - E.WALL_T / 2) and np.all(wall[:, 3] == E.WALL_X + E.WALL_T / 2)
    for cy, cz in E.WINDOW_CENTRES:  # a window's centre is open, a point just outside it is wall
        assert not covers_any(wall, [E.WALL_X, cy, cz])
        assert covers_any(wall, [E.WALL_X, cy + E.WINDOW / 2 + 0.5, cz])
    # the wall spans the workspace in y and z except for the windows: its area is 100^2 - 4 * 6^2
    area = np.sum((wall[:, 4] - wall[:, 1]) * (wall[:, 5] - wall[:, 2]))
    assert area == pytest.approx(100 * 100 - 4 * E.WINDOW ** 2)


def test_building_keeps_the_window_tunnels_open():
    obs = E.building(1000, 2)
    extra = obs[len(E.wall_with_windows()):]
    for cy, cz in E.WINDOW_CENTRES:  # the 8 m long passage through each window is free of random boxes
        for x in np.linspace(E.WALL_X - 4, E.WALL_X + 4, 9):
            assert not covers_any(extra, [x, cy, cz])


@pytest.mark.parametrize("sep", [(6.0, 12.0), (25.0, 45.0)])
def test_learned_family_separation_and_obstacle_range(sep):
    for seed in range(20):
        obs, s, g = E.learned_family(1000 + seed, obs_range=(100, 300), min_sep=sep[0], max_sep=sep[1])
        assert 100 <= obs.shape[0] <= 300 and s.shape == (12,) and g.shape == (12,)
        assert sep[0] <= np.linalg.norm(s[:3] - g[:3]) <= sep[1]
        assert abs(s[0] - E.WALL_X) > 2 and abs(g[0] - E.WALL_X) > 2
        assert not covers_any(obs, s[:3]) and not covers_any(obs, g[:3])


def test_batch_queries_mix_and_ranges():
    qs = E.batch_queries(200, seed=4)
    models = np.array([q["model"] for q in qs])
    counts = {m: int((models == m).sum()) for m in (kpax.MODEL_DOUBLE_INTEGRATOR, kpax.MODEL_DUBINS_AIRPLANE,
                                                    kpax.MODEL_QUADROTOR)}
    assert sum(counts.values()) == 200 and counts[kpax.MODEL_DOUBLE_INTEGRATOR] == 80
    for q in qs:
        assert 10 <= q["n_obs"] <= 5000 and (1 << 14) <= q["tree"] <= (1 << 20)
        assert q["obstacles"].shape == (q["n_obs"], 6)
        assert np.linalg.norm(q["start"][:3] - q["goal"][:3]) >= 50
        assert not covers_any(q["obstacles"], q["start"][:3]) and not covers_any(q["obstacles"], q["goal"][:3])

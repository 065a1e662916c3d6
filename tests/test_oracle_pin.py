"""Pins the CPU oracle to the reference: bit-exact against the reference's own routines compiled
for the host (oracle/_ref) and against the committed golden vectors made from them."""
from pathlib import Path

import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden"
PRESETS = {"di": kpax.PRESET_DI, "dubins": kpax.PRESET_DUBINS, "quad": kpax.PRESET_QUAD}
SCENES = {"di": E.di_scene, "dubins": E.dubins_scene, "quad": E.quad_scene}


def ref_available(model: int) -> bool:
    try:
        O.RefLib(model)
        return True
    except (FileNotFoundError, OSError):
        return False


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


# Random123 known-answer vectors for Philox4x32-10.
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0], [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert list(O.philox(ctr, key)) == want


def test_uniforms_in_half_open_unit_interval():
    u = O.child_draws(123, 0, 1, 4096)
    assert u.min() > 0.0 and u.max() <= 1.0
    # exactly representable on the 2^-24 grid
    assert np.all((u.astype(np.float64) * 2**24) == np.round(u.astype(np.float64) * 2**24))
    assert abs(float(u.mean()) - 0.5) < 0.01


# the benchmark scenes per model, and the quadrotor in the reference's own obstacle files
GOLDEN_SETS = {**PRESETS, "quad_quadTrees": kpax.PRESET_QUAD, "quad_quadHouse": kpax.PRESET_QUAD,
               "quad_quadPillars": kpax.PRESET_QUAD}


@pytest.mark.parametrize("name", list(GOLDEN_SETS))
def test_golden_vectors_reproduced(name):
    """The oracle reproduces the reference's outputs stored in tests/golden (bit-exact)."""
    g = np.load(GOLDEN / f"{name}.npz")
    cfg = kpax.preset(GOLDEN_SETS[name])
    rows, valid, steps, margin, nonfinite, kind = O.propagate(cfg, g["obstacles"], g["parents"], g["draws"])
    assert np.array_equal(bits(rows), bits(g["rows"]))
    assert np.array_equal(valid, g["valid"])
    assert np.array_equal(valid, g["valid_brute"])  # no cell overflows in these scenes
    r1, r2 = O.regions(cfg, g["rows"])
    assert np.array_equal(r1, g["r1"]) and np.array_equal(r2, g["r2"])
    # a duration draw of exactly 1 runs N + 1 steps where steps are drawn
    if not cfg.fixed_steps:
        assert steps[0] <= cfg.max_propagation_duration + 1
        assert g["rows"][0, -1] == np.float32(cfg.step_size) * (cfg.max_propagation_duration + 1)


@pytest.mark.parametrize("name", list(PRESETS))
def test_propagation_matches_reference(name):
    cfg = kpax.preset(PRESETS[name])
    if not ref_available(cfg.model):
        pytest.skip("reference tree not present")
    ref = O.RefLib(cfg.model)
    obs, _, _ = SCENES[name]()
    ref.set_obstacles(obs)
    n = 3000
    par = E.sample_states(cfg.model, n, 31, cfg.v_min, cfg.v_max)
    par[:50, :3] += np.float32(200.0)  # far outside the workspace
    d = E.uniform_draws(n, 32)
    d[50:60, :] = 1.0
    if cfg.fixed_steps:
        d[:, 4] = np.float32((cfg.max_propagation_duration - 0.5) / cfg.max_propagation_duration)
    rr, rv = ref.propagate(par, d, use_hash=True)
    _, bv = ref.propagate(par, d, use_hash=False)
    orow, oval, *_ = O.propagate(cfg, obs, par, d)
    assert np.array_equal(bits(rr), bits(orow))
    assert np.array_equal(rv, oval) and np.array_equal(bv, oval)


@pytest.mark.parametrize("name", list(PRESETS))
def test_regions_match_reference(name):
    cfg = kpax.preset(PRESETS[name])
    if not ref_available(cfg.model):
        pytest.skip("reference tree not present")
    ref = O.RefLib(cfg.model)
    rng = np.random.default_rng(5)
    n = 5000
    s = E.sample_states(cfg.model, n, 6, cfg.v_min, cfg.v_max)
    # out-of-range and boundary coordinates (moderate magnitudes: the host build's float->int
    # conversion of huge values differs from the device's saturation)
    s[: n // 4] = rng.uniform(-150, 250, (n // 4, s.shape[1])).astype(np.float32)
    s[n // 4 : n // 4 + 64, :3] = np.float32(100.0)
    s[n // 4 + 64 : n // 4 + 128, :3] = np.float32(0.0)
    s[n // 4 + 128 : n // 4 + 192, 3:6] = np.float32(np.pi)
    r1, r2 = ref.regions(s)
    o1, o2 = O.regions(cfg, s)
    assert np.array_equal(r1, o1) and np.array_equal(r2, o2)
    t_ref = ref.min_table()
    t_o = O.region_table(cfg)
    assert np.array_equal(bits(t_ref[:, : t_o.shape[1]]), bits(t_o))


def test_collision_hash_equals_brute_force():
    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs, _, _ = E.quad_scene()
    env = O.OEnv(cfg, obs)
    rng = np.random.default_rng(9)
    n = 4000
    lo = rng.uniform(-5, 105, (n, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0, 3, (n, 3))).astype(np.float32)
    # boxes that touch an obstacle face exactly: touching is free (collisionCheck.cu:7)
    k = 200
    lo[:k] = obs[:k, 3:]
    hi[:k] = obs[:k, 3:] + 1.0
    assert np.array_equal(env.collide(lo, hi), O.collide_brute(obs, lo, hi))
    assert np.all(O.collide_brute(obs[:1], lo[:1], hi[:1]) == 1)


def test_reference_cell_overflow_is_listed_separately():
    """The reference drops entries past 16 per 5 m cell; the oracle keeps them all.  Segments
    whose reference verdict differs from the brute-force verdict must touch an overflowing cell."""
    cfg = kpax.preset(kpax.PRESET_DI)
    if not ref_available(cfg.model):
        pytest.skip("reference tree not present")
    ref = O.RefLib(cfg.model)
    obs = E.random_boxes(3000, 4)
    overflow = ref.set_obstacles(obs)
    assert overflow > 0
    rng = np.random.default_rng(3)
    n = 3000
    lo = rng.uniform(0, 99, (n, 3)).astype(np.float32)
    hi = (lo + 0.5).astype(np.float32)
    hv = ref.collide(lo, hi, use_hash=True)
    bv = ref.collide(lo, hi, use_hash=False)
    ov = O.OEnv(cfg, obs).collide(lo, hi)
    assert np.array_equal(ov, bv)
    diff = np.where(hv != bv)[0]
    cells = lambda x: np.clip((x / 5.0).astype(int), 0, 20)
    for i in diff:  # every disagreement involves a cell with more than 16 entries
        a, b = cells(lo[i]), cells(hi[i])
        counts = [ref.L.kref_cell_count(int(x + 21 * (y + 21 * z))) for z in range(a[2], b[2] + 1)
                  for y in range(a[1], b[1] + 1) for x in range(a[0], b[0] + 1)]
        assert max(counts) > 16


def test_oracle_pruning_removes_children():
    """With PruneKPAX's pruning on, accepted children are dropped with the goal-progress
    probability; off, the plan is the plain one (PruneKPAX.cu:466-498)."""
    import kpax
    import kpax_envs as E

    cfg = kpax.preset(kpax.PRESET_DI)
    cfg.max_tree_size = 1 << 13
    cfg.expansions_per_iter = 1 << 10
    cfg.max_iter = 10
    obs, s, g = E.di_scene()
    plain = O.plan(cfg, s, g, obs, plan_idx=0, stop_at_goal=False)
    cfg.prune = 1
    pruned = O.plan(cfg, s, g, obs, plan_idx=0, stop_at_goal=False)
    assert pruned["tree_size"] < plain["tree_size"]
    # the first iteration's children (same draws) differ only by the pruning
    assert pruned["expansions"] > 0 and pruned["valid_expansions"] > 0


def test_oracle_rekino_path():
    """The ReKinoLite restatement: a path from the start state into the goal ball, the same on a
    second run, and each row the propagation of its parent with the row's draws' controls."""
    import kpax
    import kpax_envs as E

    cfg = kpax.preset(kpax.PRESET_DI)
    obs, s, _ = E.di_scene()
    g = np.array([30, 30, 30, 0, 0, 0], np.float32)
    a = O.rekino(cfg, s, g, obs, num_warps=16, max_iter=800)
    b = O.rekino(cfg, s, g, obs, num_warps=16, max_iter=800)
    assert a["found"] and a["warp"] == b["warp"] and np.array_equal(a["path"], b["path"])
    assert np.array_equal(a["path"][0, :6], s[:6]) and np.linalg.norm(a["path"][-1, :3] - g[:3]) < cfg.goal_thresh


def test_obstacle_csv_reader(tmp_path):
    """readObstaclesFromCSV (helper.cu:13-39): comma-separated floats, any number per line, six per
    obstacle; the written form reads back exactly at float32."""
    import kpax_envs as E

    text = "50.7722,37.8436,0.0,53.37019999999999,39.3436,20.0\n1,2,3,\n4,5,6\n"
    (tmp_path / "a.csv").write_text(text)
    obs = E.read_obstacles_csv(tmp_path / "a.csv")
    want = np.array([[50.7722, 37.8436, 0.0, 53.37019999999999, 39.3436, 20.0], [1, 2, 3, 4, 5, 6]], np.float32)
    assert obs.dtype == np.float32 and np.array_equal(obs, want)
    g = np.load(GOLDEN / "quad_quadTrees.npz")
    E.write_obstacles_csv(tmp_path / "b.csv", g["obstacles"])
    back = E.read_obstacles_csv(tmp_path / "b.csv")
    assert back.shape == (158, 6) and np.allclose(back, g["obstacles"], atol=5e-7 * 100, rtol=0)

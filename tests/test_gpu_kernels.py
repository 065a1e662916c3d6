"""Parity of the sm_100a kernels with the reference (golden vectors) and the CPU oracle.

Bars: double-integrator segments, control draws, step counts, region ids, collision verdicts and
the obstacle grid are bit-exact.  Dubins and quadrotor states use the accurate device trig with
fused multiply-adds and must match the reference's FP32 RK4 within REL_TOL relative error
(|gpu - ref| <= REL_TOL * max(|ref|, 1)).  A segment whose validity differs is accepted only when
its smallest check margin (oracle) is below NEAR_TOL, and is listed."""
from pathlib import Path

import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
PRESETS = {"di": kpax.PRESET_DI, "dubins": kpax.PRESET_DUBINS, "quad": kpax.PRESET_QUAD}
SCENES = {"di": E.di_scene, "dubins": E.dubins_scene, "quad": E.quad_scene}
REL_TOL = 1e-5
NEAR_TOL = 1e-4


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_propagate(torch, cfg, obs, parents, draws=None, stream_id=0):
    n = parents.shape[0]
    S = cfg.state_dim + cfg.control_dim + 1
    d_obs = dev(torch, obs.astype(np.float32))
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    d_par = dev(torch, parents.astype(np.float32))
    d_draw = dev(torch, np.ascontiguousarray(draws[:, :5], np.float32)) if draws is not None else None
    rows = torch.zeros((n, S), dtype=torch.float32, device="cuda")
    valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
    steps = torch.zeros(n, dtype=torch.int32, device="cuda")
    kpax.propagate_batch(cfg, env, d_par.data_ptr(), d_draw.data_ptr() if d_draw is not None else None, stream_id, n,
                         rows.data_ptr(), valid.data_ptr(), steps.data_ptr())
    torch.cuda.synchronize()
    return rows.cpu().numpy(), valid.cpu().numpy(), steps.cpu().numpy(), env


def compare_segments(cfg, rows, valid, ref_rows, ref_valid, margin, label):
    """Returns the list of accepted near-boundary disagreements."""
    sd, cd = cfg.state_dim, cfg.control_dim
    # controls and duration come from the draws: bit-exact for every model
    assert np.array_equal(bits(rows[:, sd:]), bits(ref_rows[:, sd:])), f"{label}: control/duration columns differ"
    flips = np.where(valid != ref_valid)[0]
    near = [int(i) for i in flips if margin[i] < NEAR_TOL]
    assert len(near) == len(flips), f"{label}: verdict differs on segments with margin >= {NEAR_TOL}: " \
                                    f"{[(int(i), float(margin[i])) for i in flips if margin[i] >= NEAR_TOL][:5]}"
    same = np.setdiff1d(np.arange(rows.shape[0]), flips)
    a, b = rows[same, :sd].astype(np.float64), ref_rows[same, :sd].astype(np.float64)
    # segments that stopped on a check compare their last state only when both stopped at the same step;
    # a near-boundary margin can move the stop by one step without changing the verdict
    err = np.abs(a - b) / np.maximum(np.abs(b), 1.0)
    row_err = err.max(axis=1)
    bad = np.where((row_err > REL_TOL) & (margin[same] >= NEAR_TOL))[0]
    assert bad.size == 0, f"{label}: {bad.size} rows beyond {REL_TOL}: worst {row_err.max():.3g}"
    return near, float(row_err.max()) if row_err.size else 0.0


# the benchmark scenes per model, and the quadrotor in the reference's own obstacle files
GOLDEN_SETS = {**PRESETS, "quad_quadTrees": kpax.PRESET_QUAD, "quad_quadHouse": kpax.PRESET_QUAD,
               "quad_quadPillars": kpax.PRESET_QUAD}


@pytest.mark.parametrize("name", list(GOLDEN_SETS))
def test_propagate_matches_reference_golden(cuda, name):
    import torch

    g = np.load(GOLDEN / f"{name}.npz")
    cfg = kpax.preset(GOLDEN_SETS[name])
    rows, valid, steps, env = gpu_propagate(torch, cfg, g["obstacles"], g["parents"], g["draws"])
    orow, oval, ostep, margin, nonfinite, kind = O.propagate(cfg, g["obstacles"], g["parents"], g["draws"])
    assert np.array_equal(bits(orow), bits(g["rows"]))  # oracle pinned to the reference
    if cfg.model == kpax.MODEL_DOUBLE_INTEGRATOR:
        assert np.array_equal(bits(rows), bits(g["rows"]))
        assert np.array_equal(valid, g["valid"])
        assert np.array_equal(steps, ostep)
    else:
        near, worst = compare_segments(cfg, rows, valid, g["rows"], g["valid"], margin, name)
        print(f"{name}: worst relative state error {worst:.3g}; near-boundary verdict flips {near}")


@pytest.mark.parametrize("name", list(PRESETS))
def test_propagate_philox_draws_match_oracle(cuda, name):
    import torch

    cfg = kpax.preset(PRESETS[name])
    obs, _, _ = SCENES[name]()
    n = 8192
    par = E.sample_states(cfg.model, n, 77, cfg.v_min, cfg.v_max)
    rows, valid, steps, env = gpu_propagate(torch, cfg, obs, par, None, stream_id=5)
    orow, oval, ostep, margin, nonfinite, kind = O.propagate(cfg, obs, par, None, stream=5, nthreads=8)
    if cfg.model == kpax.MODEL_DOUBLE_INTEGRATOR:
        assert np.array_equal(bits(rows), bits(orow)) and np.array_equal(valid, oval) and np.array_equal(steps, ostep)
    else:
        near, worst = compare_segments(cfg, rows, valid, orow, oval, margin, name)
        print(f"{name}: worst relative state error {worst:.3g}; near-boundary flips {len(near)} of {n}")
        assert len(near) <= n // 1000


@pytest.mark.parametrize("name", list(PRESETS))
@pytest.mark.parametrize("compat", [1, 0])
def test_regions_bit_exact(cuda, name, compat):
    import torch

    cfg = kpax.preset(PRESETS[name])
    cfg.region_compat = compat
    rng = np.random.default_rng(3 + compat)
    n = 20000
    s = E.sample_states(cfg.model, n, 8, cfg.v_min, cfg.v_max)
    s[: n // 4] = rng.uniform(-150, 250, (n // 4, cfg.state_dim)).astype(np.float32)
    edge = np.array([0.0, 100.0, 12.5, 25.0, -0.0, 1e30, -1e30, np.inf, -np.inf, np.nan, np.pi, -np.pi,
                     np.float32(np.pi) * 0.25, 30.0, -30.0, 0.5, 2.0], np.float32)
    k = n // 4
    s[k: k + 4000] = rng.choice(edge, size=(4000, cfg.state_dim))
    d_s = dev(torch, s)
    r1 = torch.zeros(n, dtype=torch.int32, device="cuda")
    r2 = torch.zeros(n, dtype=torch.int32, device="cuda")
    kpax.region_batch(cfg, d_s.data_ptr(), n, r1.data_ptr(), r2.data_ptr())
    torch.cuda.synchronize()
    o1, o2 = O.regions(cfg, s)
    g1, g2 = r1.cpu().numpy(), r2.cpu().numpy()
    assert np.array_equal(g1, o1), np.where(g1 != o1)[0][:10]
    assert np.array_equal(g2, o2), np.where(g2 != o2)[0][:10]


def test_collision_bit_exact_and_grid(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs, _, _ = E.quad_scene()
    d_obs = dev(torch, obs)
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    cells, entries = env.stats()
    off, ent = O.OEnv(cfg, obs).grid()
    # the device maps coordinates to cells by a reciprocal multiply, the oracle by the reference's
    # division: points on a cell face may land one cell apart, the verdicts below may not
    assert cells == off.size - 1 and abs(entries - ent.size) <= ent.size // 100
    rng = np.random.default_rng(11)
    n = 50000
    lo = rng.uniform(-5, 105, (n, 3)).astype(np.float32)
    hi = (lo + rng.uniform(0, 4, (n, 3))).astype(np.float32)
    lo[:500] = obs[:500, 3:]  # touching faces are free
    hi[:500] = obs[:500, 3:] + 2.0
    lo[500:1000] = obs[:500, :3] - 1.0
    hi[500:1000] = obs[:500, :3]
    free = torch.zeros(n, dtype=torch.uint8, device="cuda")
    d_lo, d_hi = dev(torch, lo), dev(torch, hi)  # keep the tensors alive while the kernel runs
    kpax.collide_batch(env, d_lo.data_ptr(), d_hi.data_ptr(), n, free.data_ptr())
    torch.cuda.synchronize()
    want = O.OEnv(cfg, obs).collide(lo, hi)
    assert np.array_equal(free.cpu().numpy(), want)
    assert 0.05 < want.mean() < 0.95


def test_empty_environment_and_zero_batch(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_DI)
    empty = np.zeros((0, 6), np.float32)
    par = E.sample_states(1, 64, 1)
    d = E.uniform_draws(64, 2)
    rows, valid, steps, env = gpu_propagate(torch, cfg, empty, par, d)
    orow, oval, *_ = O.propagate(cfg, empty, par, d)
    assert np.array_equal(bits(rows), bits(orow)) and np.array_equal(valid, oval)
    assert env.stats()[1] == 0
    kpax.propagate_batch(cfg, env, 0, None, 0, 0, 0, 0)  # n = 0 is a no-op


def test_invalid_arguments_are_reported(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_DI)
    obs = np.zeros((1, 6), np.float32)
    d_obs = dev(torch, obs)
    env = kpax.Env(cfg, d_obs.data_ptr(), 1)
    with pytest.raises(kpax.KpaxError) as e:
        kpax.propagate_batch(cfg, env, 0, None, 0, 16, 0, 0)
    assert e.value.status == kpax.EINVAL
    other = kpax.preset(kpax.PRESET_DI)
    other.hash_cell_size = 2.0
    buf = torch.zeros(16 * 10, device="cuda")
    with pytest.raises(kpax.KpaxError):
        kpax.propagate_batch(other, env, buf.data_ptr(), None, 0, 1, buf.data_ptr(), buf.data_ptr())


def test_sincos_within_a_few_ulp_of_cuda(cuda):
    """The propagation kernels' branch-free sine/cosine against CUDA's sincosf."""
    import torch

    rng = np.random.default_rng(12)
    x = np.concatenate([rng.uniform(-4, 4, 200000), rng.uniform(-200, 200, 100000), rng.uniform(-8192, 8192, 50000),
                        np.array([0.0, -0.0, np.pi / 2, -np.pi / 2, np.pi, 1e-30, 8192.0, 8193.0, 1e6, 3e30, np.inf, np.nan])
                        ]).astype(np.float32)
    d_x = dev(torch, x)
    out = torch.zeros((x.size, 4), device="cuda")
    kpax.check(kpax.load().kpax_test_sincos(d_x.data_ptr(), x.size, out.data_ptr(), None), "kpax_test_sincos")
    torch.cuda.synchronize()
    o = out.cpu().numpy().astype(np.float64)
    fin = np.isfinite(x)
    for a, b in ((o[fin, 0], o[fin, 2]), (o[fin, 1], o[fin, 3])):
        ulp = np.spacing(np.abs(b).astype(np.float32)).astype(np.float64)
        err = np.abs(a - b)
        assert np.all(err <= np.maximum(4 * ulp, 2e-7)), float((err / np.maximum(ulp, 1e-45)).max())
    assert np.all(np.isnan(o[~fin, :2]))


@pytest.mark.parametrize("name", list(PRESETS))
def test_phased_large_batch_equals_one_pass(cuda, name):
    """Batches of 2^18 segments or more run in phases (the first steps of every segment, then the
    live ones compacted, twice); rows, verdicts and step counts equal the one-pass kernel's, which
    smaller batches use: here the same draws propagated in slices of 2^17."""
    import torch

    cfg = kpax.preset(PRESETS[name])
    obs, _, _ = SCENES[name]()
    n = (1 << 18) + 123  # ragged: the last warp of the head is partly empty
    S = cfg.sample_dim
    par = E.sample_states(cfg.model, n, 91, cfg.v_min, cfg.v_max)
    draws = np.ascontiguousarray(E.uniform_draws(n, 92)[:, :5])
    d_obs = dev(torch, obs.astype(np.float32))
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    d_par, d_draw = dev(torch, par), dev(torch, draws)

    def run(lo, hi, rows, valid, steps):
        m = hi - lo
        kpax.propagate_batch(cfg, env, d_par[lo:hi].data_ptr(), d_draw[lo:hi].data_ptr(), 0, m, rows[lo:hi].data_ptr(),
                             valid[lo:hi].data_ptr(), steps[lo:hi].data_ptr())

    out = [(torch.zeros((n, S), device="cuda"), torch.zeros(n, dtype=torch.uint8, device="cuda"),
            torch.zeros(n, dtype=torch.int32, device="cuda")) for _ in range(2)]
    run(0, n, *out[0])
    for lo in range(0, n, 1 << 17):
        run(lo, min(n, lo + (1 << 17)), *out[1])
    torch.cuda.synchronize()
    a, b = [[x.cpu().numpy() for x in o] for o in out]
    assert np.array_equal(bits(a[0]), bits(b[0])), f"{name}: rows differ"
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), f"{name}: verdicts or step counts differ"
    assert 0 < a[1].mean() < 1


@pytest.mark.parametrize("n,density", [(0, 0.3), (1, 1.0), (5000, 0.3), ((1 << 20) + 37, 0.2)])
def test_frontier_compaction_bit_exact(cuda, n, density):
    """kpax_frontier_compact (the planner's two frontier kernels on a caller's repeat bytes) against
    the oracle: R, k, E, n, the entry list and the repeat bytes after, for budgets from 0 to all
    entries (k = children per entry), through k = 2 and one child each with strided entries."""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    rng = np.random.default_rng(n)
    rep = np.where(rng.random(n) < density, rng.integers(1, 16, n), 0).astype(np.uint8)
    rep[rng.random(n) < 0.02] = 255  # pending: counts as the sparse repeat
    R = int(np.where(rep == 255, cfg.sparse_repeat, rep).sum())
    for budget in sorted({0, 1, 7, max(R - 1, 1), 2 * R + 5, R * cfg.children_per_entry, 1 << 16}):
        d_rep = torch.from_numpy(rep.copy()).cuda() if n else torch.zeros(1, dtype=torch.uint8, device="cuda")
        d_ent = torch.full((max(budget, 1),), -1, dtype=torch.int32, device="cuda")
        st = kpax.frontier_compact(cfg, d_rep.data_ptr(), n, budget, d_ent.data_ptr())
        o_rep, o_ent, o_st = O.frontier_compact(cfg, rep, budget)
        assert st == o_st, (budget, st, o_st)
        assert np.array_equal(d_ent[: st["E"]].cpu().numpy().view(np.uint32), o_ent), budget
        assert np.array_equal(d_rep.cpu().numpy()[:n], o_rep), budget
        assert st["E"] == budget or st["E"] == R or st["E"] * st["k"] <= budget


def test_frontier_compaction_of_unaligned_repeat_bytes(cuda):
    """The count pass reads four repeat bytes at a time only from 4-byte aligned arrays: repeat
    bytes that start one byte into a buffer give the oracle's result too."""
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    n = 70001
    rng = np.random.default_rng(11)
    rep = np.where(rng.random(n) < 0.3, rng.integers(1, 16, n), 0).astype(np.uint8)
    rep[rng.random(n) < 0.02] = 255
    buf = torch.zeros(n + 1, dtype=torch.uint8, device="cuda")
    buf[1:] = torch.from_numpy(rep).cuda()
    for budget in (1 << 12, 1 << 16):
        buf[1:] = torch.from_numpy(rep).cuda()
        d_ent = torch.full((budget,), -1, dtype=torch.int32, device="cuda")
        st = kpax.frontier_compact(cfg, buf.data_ptr() + 1, n, budget, d_ent.data_ptr())
        o_rep, o_ent, o_st = O.frontier_compact(cfg, rep, budget)
        assert st == o_st, (budget, st, o_st)
        assert np.array_equal(d_ent[: st["E"]].cpu().numpy().view(np.uint32), o_ent), budget
        assert np.array_equal(buf.cpu().numpy()[1:], o_rep), budget


def test_bounded_wait_gives_up_and_context_stays_usable(cuda):
    """A device-side wait that nothing ends (the expansion's look-back wait on a tile that never
    publishes) gives up after its poll limit: the kernel stores a timeout status and returns, the
    call reports ETIMEOUT, and the context keeps working (a batch then matches the oracle)."""
    import time

    import torch

    t0 = time.perf_counter()
    with pytest.raises(kpax.KpaxError) as e:
        kpax.test_wait_timeout(1 << 12)
    assert e.value.status == kpax.ETIMEOUT and "gave up" in str(e.value)
    assert time.perf_counter() - t0 < 10.0
    cfg = kpax.preset(kpax.PRESET_DI)
    obs, _, _ = E.di_scene()
    par = E.sample_states(cfg.model, 256, 7)
    draws = E.uniform_draws(256, 8)
    rows, valid, _, _ = gpu_propagate(torch, cfg, obs, par, draws)
    orow, oval, *_ = O.propagate(cfg, obs, par, draws)
    assert np.array_equal(valid, oval) and np.array_equal(bits(rows), bits(orow))


def test_fp32_peak_microkernel(cuda):
    """kpax_fp32_peak times its FMA chains: on a B200 the rate lies between a third of and just
    above the nominal 148 SM x 128 lanes x 2 FLOP x 1.965 GHz = 74.4 TFLOP/s."""
    t, ms = kpax.fp32_peak(1 << 14)
    assert ms > 0.0 and 25.0 < t < 80.0, (t, ms)

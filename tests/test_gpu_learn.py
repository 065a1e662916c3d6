"""Learned proposal on the GPU against the network oracle (oracle/mlp_oracle.py).

Bit-exact: occupancy bits, input features, the planner's mixture records against the standalone
tensor-core pass on the same states, and plans with epsilon = 1 against plain plans.  Within
stated tolerances: the FP32 training kernels (forward, loss, gradient, Adam) against float64,
and each BF16 tensor-core layer against the oracle fed the GPU's own previous layer."""
import numpy as np
import pytest

import kpax
import kpax_envs as E
import mlp_oracle as M
import oracle as O

pytestmark = pytest.mark.gpu


def rand_params(seed=0, s1=0.25, s2=0.08, s3=0.08):
    rng = np.random.default_rng(seed)
    w = np.zeros(M.NUM_PARAMS, np.float32)
    W1, b1, W2, b2, W3, b3 = M.unpack(w)
    W1[:, : M.IN] = rng.normal(0, s1, (M.H, M.IN))
    W2[:] = rng.normal(0, s2, (M.H, M.H))
    W3[: M.OUT] = rng.normal(0, s3, (M.OUT, M.H))
    b1[:] = rng.normal(0, 0.1, M.H)
    b2[:] = rng.normal(0, 0.1, M.H)
    b3[: M.OUT] = rng.normal(0, 0.3, M.OUT)
    return w


def quad_states(n, seed=1, lo=0.0, hi=100.0):
    rng = np.random.default_rng(seed)
    s = np.zeros((n, 12), np.float32)
    s[:, :3] = rng.uniform(lo, hi, (n, 3))
    s[:, 3:6] = rng.uniform(-1.0, 1.0, (n, 3))
    s[:, 6:9] = rng.uniform(-8.0, 8.0, (n, 3))
    s[:, 9:12] = rng.uniform(-2.0, 2.0, (n, 3))
    return s


@pytest.fixture(scope="module")
def scene(cuda):
    import torch

    cfg = kpax.preset(kpax.PRESET_QUAD)
    obs = E.building(300, seed=11)
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    occ = M.occupancy(obs)
    return cfg, obs, d_obs, env, occ


def bf16_bits_to_f32(h):
    return (np.asarray(h, np.uint16).astype(np.uint32) << 16).view(np.float32)


def test_occupancy_bit_exact(scene):
    import torch

    cfg, obs, _, env, occ = scene
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    kpax.env_occupancy(env, d.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), M.pack_bits(occ))
    assert 0 < occ.sum() < occ.size


def test_features_bit_exact(scene):
    import torch

    cfg, obs, _, env, occ = scene
    s = quad_states(3000, lo=-20.0, hi=120.0)  # includes cells outside the grid (clamped)
    g = np.random.default_rng(2).uniform(0, 100, (3000, 3)).astype(np.float32)
    d_s, d_g = torch.from_numpy(s).cuda(), torch.from_numpy(g).cuda()
    d_x = torch.zeros((3000, M.IN_PAD), device="cuda")
    kpax.mlp_features(env, d_s.data_ptr(), 12, d_g.data_ptr(), 3000, d_x.data_ptr())
    torch.cuda.synchronize()
    want = M.features(s, g, occ)
    assert np.array_equal(d_x.cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_fp32_forward_loss_and_gradient(cuda):
    import torch

    w = rand_params(3)
    rng = np.random.default_rng(4)
    n = 512
    x = np.zeros((n, M.IN_PAD), np.float32)
    x[:, : M.IN] = rng.normal(0, 1, (n, M.IN))
    y = rng.normal(0, 2, (n, M.DIM)).astype(np.float32)
    net = kpax.MLP(max_batch=n)
    net.set_params(w)
    net.set_loss_mask([1, 1, 1, 1, 0])
    d_x, d_y = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    d_o = torch.zeros((n, M.OUT_PAD), device="cuda")
    net.forward(d_x.data_ptr(), n, d_o.data_ptr())
    torch.cuda.synchronize()
    o_ref = M.forward(w.astype(np.float64), x)[-1]
    assert np.max(np.abs(d_o.cpu().numpy() - o_ref)) <= 1e-5 * max(1.0, np.max(np.abs(o_ref)))
    d_g = torch.zeros(M.NUM_PARAMS, device="cuda")
    loss = net.loss_grad(d_x.data_ptr(), d_y.data_ptr(), n, d_g.data_ptr())
    l_ref, g_ref = M.loss_grad(w.astype(np.float64), x, y, (1, 1, 1, 1, 0))
    assert abs(loss - l_ref) <= 1e-5 * max(1.0, abs(l_ref))
    g = d_g.cpu().numpy()
    for name, a, b in zip(("W1", "b1", "W2", "b2", "W3", "b3"), M.unpack(g), M.unpack(g_ref)):
        err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-12)
        assert err <= 1e-4, (name, err)


def test_adam_step_matches_oracle(cuda):
    import torch

    w = rand_params(5)
    rng = np.random.default_rng(6)
    n = 256
    x = np.zeros((n, M.IN_PAD), np.float32)
    x[:, : M.IN] = rng.normal(0, 1, (n, M.IN))
    y = rng.normal(0, 2, (n, M.DIM)).astype(np.float32)
    d_x, d_y = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    net = kpax.MLP(max_batch=n)
    net.set_params(w)
    d_g = torch.zeros(M.NUM_PARAMS, device="cuda")
    net.loss_grad(d_x.data_ptr(), d_y.data_ptr(), n, d_g.data_ptr())
    g = d_g.cpu().numpy()
    net.train_step(d_x.data_ptr(), d_y.data_ptr(), idx.data_ptr(), n, 1e-3)
    w1 = net.get_params()
    m, v, step = net.adam_state()
    wr, mr, vr = M.adam_step(w, g, np.zeros_like(w), np.zeros_like(w), 1, 1e-3)
    assert step == 1
    assert np.max(np.abs(m - mr)) <= 1e-6 * max(1e-12, np.max(np.abs(mr))) + 1e-12
    assert np.max(np.abs(v - vr)) <= 1e-5 * max(1e-20, np.max(np.abs(vr))) + 1e-20
    assert np.max(np.abs(w1 - wr)) <= 1e-6


def test_training_reduces_loss(cuda):
    import torch

    rng = np.random.default_rng(8)
    n = 8192
    x = np.zeros((n, M.IN_PAD), np.float32)
    x[:, : M.IN] = rng.normal(0, 1, (n, M.IN))
    y = (2.0 * np.tanh(x[:, :5] * 1.5) + 0.2 * rng.normal(0, 1, (n, 5))).astype(np.float32)
    net = kpax.MLP(max_batch=1024)
    net.set_params(rand_params(9, s3=0.02))
    d_x, d_y = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    g = torch.Generator(device="cuda").manual_seed(0)
    losses = []
    for step in range(400):
        idx = torch.randint(0, n, (1024,), device="cuda", dtype=torch.int32, generator=g)
        losses.append(net.train_step(d_x.data_ptr(), d_y.data_ptr(), idx.data_ptr(), 1024, 2e-3, want_loss=step % 50 == 0))
    first, last = losses[0], [l for l in losses if l is not None][-1]
    full = net.loss_grad(d_x.data_ptr(), d_y.data_ptr(), 1024)
    print(f"loss {first:.3f} -> {last:.3f}; first-batch loss {full:.3f}")
    assert last < first - 1.0


def tc_check(scene, n, seed):
    import torch

    cfg, obs, _, env, occ = scene
    w = rand_params(seed)
    net = kpax.MLP(max_batch=256)
    net.set_params(w)
    s = quad_states(n, seed=seed + 1)
    g = np.tile(np.array([[80.0, 95.0, 90.0]], np.float32), (n, 1))
    d_s, d_g = torch.from_numpy(s).cuda(), torch.from_numpy(g).cuda()
    d_mix = torch.zeros((n, M.MIX), device="cuda")
    d_out = torch.zeros((n, M.OUT_PAD), device="cuda")
    d_h1 = torch.zeros((n, M.H), dtype=torch.int16, device="cuda")
    d_h2 = torch.zeros((n, M.H), dtype=torch.int16, device="cuda")
    net.propose(env, d_s.data_ptr(), 12, d_g.data_ptr(), n, d_mix.data_ptr(), d_out.data_ptr(), d_h1.data_ptr(),
                d_h2.data_ptr())
    torch.cuda.synchronize()
    h1 = bf16_bits_to_f32(d_h1.cpu().numpy().view(np.uint16))
    h2 = bf16_bits_to_f32(d_h2.cpu().numpy().view(np.uint16))
    out, mix = d_out.cpu().numpy(), d_mix.cpu().numpy()
    x = M.features(s, g, occ)
    # layer by layer, each from the GPU's own input (bounds in mlp_oracle.tc_layer_violation)
    viol = M.tc_layer_violation(w, x, h1, h2, out)
    assert all(v <= 0.0 for v in viol.values()), viol
    out = out[:, : M.OUT]
    # the records are the outputs (biases included)
    assert np.array_equal(mix.view(np.uint32), np.ascontiguousarray(out).view(np.uint32))
    # end to end against the oracle's own BF16 pass (no teacher forcing): small drift only
    _, _, o_ref = M.forward_bf16(w, x)
    assert np.max(np.abs(out - o_ref[:, : M.OUT])) <= 0.02 * max(1.0, np.max(np.abs(o_ref)))
    return out


def test_tensor_core_pass_one_tile(scene):
    tc_check(scene, 100, 10)


def test_tensor_core_pass_many_tiles_per_cta(scene):
    # 148 SMs: 2.4 tiles of 128 rows per CTA, last tile ragged
    tc_check(scene, 148 * 128 * 2 + 77 + 128 * 60, 20)


def quad_cfg_small(iters=8):
    cfg = kpax.preset(kpax.PRESET_QUAD)
    cfg.max_iter = iters
    cfg.max_tree_size = 1 << 18
    cfg.expansions_per_iter = 1 << 13
    cfg.unroll_iters = 1
    return cfg


def test_epsilon_one_equals_plain_plan(cuda):
    import torch

    cfg = quad_cfg_small(10)
    obs, s, goal = E.quad_scene()
    d_obs = torch.from_numpy(obs).cuda()
    net = kpax.MLP(max_batch=64)
    net.set_params(rand_params(30))
    plain = kpax.KPAX(cfg)
    r0 = plain.plan(s, goal, d_obs.data_ptr(), obs.shape[0])
    rows0, par0, _ = plain.export_tree()
    learned = kpax.KPAX(cfg)
    learned.set_proposal(net, 1.0)
    r1 = learned.plan(s, goal, d_obs.data_ptr(), obs.shape[0])
    rows1, par1, _ = learned.export_tree()
    assert (r0.tree_size, r0.iters, r0.valid_expansions) == (r1.tree_size, r1.iters, r1.valid_expansions)
    assert np.array_equal(rows0.view(np.uint32), rows1.view(np.uint32)) and np.array_equal(par0, par1)
    # turning it off again restores the plain sampler
    learned.set_proposal(None)
    learned.plan(s, goal, d_obs.data_ptr(), obs.shape[0])


def test_planner_draws_follow_the_mixture(scene):
    import torch

    cfg = quad_cfg_small(4)
    obs, s, goal = E.quad_scene()
    d_obs = torch.from_numpy(obs).cuda()
    env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
    net = kpax.MLP(max_batch=64)
    net.set_params(rand_params(31))
    eps = 0.2
    pl = kpax.KPAX(cfg)
    pl.set_proposal(net, eps)
    pl.debug_capture(True)
    pl.begin(s, goal, d_obs.data_ptr(), obs.shape[0])
    learned_total = 0
    for it in range(1, 4):
        rows, _, _ = pl.export_tree()
        pl.iterate(1)
        c_rows, c_valid, _, _, _, c_par = pl.export_children()
        mix = pl.export_proposal()
        n, E_ = c_par.size, mix.shape[0]
        assert E_ > 0 and n % E_ == 0
        k = n // E_
        # the planner's records equal the standalone tensor-core pass on the entries' nodes
        ent_states = np.ascontiguousarray(rows[c_par[::k], :12])
        d_st = torch.from_numpy(ent_states).cuda()
        d_g = torch.from_numpy(np.tile(goal[:3].astype(np.float32), (E_, 1))).cuda()
        d_mix = torch.zeros((E_, M.MIX), device="cuda")
        net.propose(env, d_st.data_ptr(), 12, d_g.data_ptr(), E_, d_mix.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(d_mix.cpu().numpy().view(np.uint32), mix.view(np.uint32))
        # each child's controls: the oracle sampler on its entry's record
        plain = O.child_draws(cfg.seed, 0, it, n)
        u, learned, _, margin = M.mixture_draws(mix[np.arange(n) // k].astype(np.float64), plain, eps, cfg.seed, 0, it,
                                                np.arange(n))
        # children whose component uniform lies within 1e-6 of a cumulative weight may pick the
        # neighbouring component (FP32 softmax on the GPU); they are counted and skipped
        close = learned & (margin < 1e-6)
        if close.any():
            print(f"iteration {it}: {int(close.sum())} children at a component boundary")
        learned_ok = learned & ~close
        clo = np.array(cfg.ctrl_min[:4], np.float32)
        crng = (np.array(cfg.ctrl_max[:4], np.float32) - clo).astype(np.float32)
        want = clo + u[:, :4].astype(np.float32) * crng
        got = c_rows[:, 12:16]
        assert np.array_equal(got[~learned].view(np.uint32), (clo + plain[~learned, :4] * crng).astype(np.float32).view(np.uint32))
        assert np.all(np.abs(got[learned_ok] - want[learned_ok]) <= 1e-5 * crng + 1e-7)
        learned_total += int(learned.sum())
        assert abs((~learned).mean() - eps) < 0.05
    assert learned_total > 0

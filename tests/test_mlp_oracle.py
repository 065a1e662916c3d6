"""The network oracle pinned on the CPU: its Philox matches the C oracle's (itself checked against
the published known-answer vectors), its float64 gradient matches central finite differences,
its float32 gradient matches the float64 one, and the BF16 rounding and the mixture sampler
behave as specified."""
import numpy as np
import pytest

import mlp_oracle as M
import oracle as O


def small_params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    w = np.zeros(M.NUM_PARAMS, np.float64)
    W1, b1, W2, b2, W3, b3 = M.unpack(w)
    W1[:, : M.IN] = rng.normal(0, scale, (M.H, M.IN))
    W2[:] = rng.normal(0, scale / 4, (M.H, M.H))
    W3[: M.OUT] = rng.normal(0, scale / 4, (M.OUT, M.H))
    b1[:] = rng.normal(0, 0.1, M.H)
    b2[:] = rng.normal(0, 0.1, M.H)
    b3[: M.OUT] = rng.normal(0, 0.1, M.OUT)
    return w


def batch(n=6, seed=1):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, M.IN_PAD))
    x[:, : M.IN] = rng.normal(0, 1, (n, M.IN))
    y = rng.normal(0, 2, (n, M.DIM))
    return x, y


def test_philox_matches_c_oracle():
    rng = np.random.default_rng(3)
    for _ in range(20):
        c = rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)
        k = rng.integers(0, 2 ** 32, 2, dtype=np.uint64).astype(np.uint32)
        want = O.philox(c, k)
        got = M.philox_vec(c[0], c[1], c[2], c[3], int(k[0]), int(k[1]))
        assert np.array_equal(got, want)


def test_float64_gradient_matches_finite_differences():
    w = small_params()
    x, y = batch()
    mask = (1, 1, 1, 1, 0)
    _, g = M.loss_grad(w, x, y, mask)
    rng = np.random.default_rng(5)
    # probe every tensor: W1 (used columns), b1, W2, b2, W3 (used rows), b3 (used entries)
    probes = np.concatenate([
        M.OFF_W1 + rng.integers(0, M.H, 8) * M.IN_PAD + rng.integers(0, M.IN, 8),
        M.OFF_B1 + rng.integers(0, M.H, 4),
        M.OFF_W2 + rng.integers(0, M.H * M.H, 8),
        M.OFF_B2 + rng.integers(0, M.H, 4),
        M.OFF_W3 + rng.integers(0, M.OUT, 8) * M.H + rng.integers(0, M.H, 8),
        M.OFF_B3 + np.arange(0, M.OUT, 7),
    ])
    h = 1e-6
    for i in probes:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (M.loss_grad(wp, x, y, mask)[0] - M.loss_grad(wm, x, y, mask)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-8, (int(i), fd, g[i])
    # padded inputs and outputs carry no gradient
    gW1, _, _, _, gW3, gb3 = M.unpack(g)
    assert np.all(gW1[:, M.IN:] == 0) and np.all(gW3[M.OUT:] == 0) and np.all(gb3[M.OUT:] == 0)


def test_float32_gradient_matches_float64():
    w = small_params(1)
    x, y = batch(64, 2)
    l64, g64 = M.loss_grad(w, x, y)
    l32, g32 = M.loss_grad(w.astype(np.float32), x.astype(np.float32), y.astype(np.float32), dtype=np.float32)
    assert abs(l32 - l64) <= 1e-5 * max(1.0, abs(l64))
    for a, b in zip(M.unpack(g32), M.unpack(g64)):
        assert np.max(np.abs(a - b)) <= 1e-4 * max(np.max(np.abs(b)), 1e-6)


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7, -2.5, 1e-30, 65504.0], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -6) and r[3] == np.float32(1.0 + 2 ** -7)
    assert r[4] == -2.5
    assert np.all((r.view(np.uint32) & 0xFFFF) == 0)


def test_mixture_sampler():
    w = small_params(2)
    x, _ = batch(16, 4)
    o = M.forward(w, x)[-1][:, : M.OUT]
    wts, mu, sig = M.mixture_parts(o)
    assert np.allclose(wts.sum(1), 1.0)
    assert np.all(sig > np.exp(-7.0)) and np.all(sig < np.exp(3.0))
    n = 4096
    rec_n = np.repeat(o[:1], n, 0)
    plain = np.full((n, 6), 0.5)
    u, learned, _, _ = M.mixture_draws(rec_n, plain, 1.0, 7, 0, 1, np.arange(n))
    assert not learned.any() and np.array_equal(u, plain)
    u, learned, comp, _ = M.mixture_draws(rec_n, plain, 0.0, 7, 0, 1, np.arange(n))
    assert learned.all() and np.all((u[:, :5] > 0) & (u[:, :5] <= 1)) and np.all(u[:, 5] == 0.5)
    # component frequencies follow the mixture weights
    freq = np.bincount(comp, minlength=M.COMP) / n
    assert np.max(np.abs(freq - wts[0])) < 0.05
    u, learned, _, _ = M.mixture_draws(rec_n, plain, 0.2, 7, 0, 1, np.arange(n))
    assert abs((~learned).mean() - 0.2) < 0.03


def test_occupancy_and_features():
    W1 = 8
    assert not M.occupancy(np.zeros((0, 6), np.float32)).any()
    assert M.occupancy(np.array([[-1, -1, -1, 101, 101, 101]], np.float32)).all()
    # one box covering exactly cell (1, 2, 3): [12.5, 25] x [25, 37.5] x [37.5, 50]
    bits = M.occupancy(np.array([[12.5, 25.0, 37.5, 25.0, 37.5, 50.0]], np.float32))
    assert np.nonzero(bits)[0].tolist() == [(3 * W1 + 2) * W1 + 1]
    s = np.zeros((2, 12), np.float32)
    s[0, :3] = (18.0, 30.0, 40.0)      # inside cell (1, 2, 3)
    s[1, :3] = (1.0, 1.0, 1.0)         # corner cell: out-of-grid neighbours count as blocked
    s[:, 6] = 5.0
    g = np.array([[80, 95, 90], [1, 1, 1]], np.float32)
    x = M.features(s, g, bits)
    assert x[0, 24 + 13] == 1.0 and x[0, 24:51].sum() == 1.0
    assert x[1, 24:51].sum() == 27 - 8
    assert x[0, 6] == np.float32(5.0) * np.float32(0.1) and x[0, 12] == np.float32(62.0) * np.float32(0.01)
    assert np.all(x[:, 51:] == 0)

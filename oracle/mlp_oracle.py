"""CPU restatement of the learned proposal network — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, and only
as the checker.  The reference planner has no learned component (it draws controls and durations
uniformly in propagateAndCheck, src/statePropagator/statePropagatorSpatialHash.cu), so this is the
oracle of the build's own network: the same parameter layout, features, loss, optimiser step and
mixture sampler as kino-pax-fork_b200/csrc/kpax_mlp.h, kpax_mlp_tc.cuh and kpax_learn.cu, written
with numpy in float64 (the gradient reference, checked against finite differences) and float32
(the arithmetic of the CUDA kernels).  BF16 inference is emulated by rounding weights and
activations to bfloat16 where the tensor-core pass rounds them and accumulating in float64.
"""
from __future__ import annotations

import numpy as np

IN, IN_PAD, H, OUT, OUT_PAD, COMP, DIM, CSTRIDE = 51, 64, 256, 88, 96, 8, 5, 11
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN_PAD
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT_PAD * H
NUM_PARAMS = OFF_B3 + OUT_PAD
SIG_MID, SIG_HALF = -2.0, 5.0
MIX = COMP * (1 + 2 * DIM)
FLOP_PER_INFERENCE = 2 * (IN * H + H * H + H * OUT)


def unpack(w: np.ndarray):
    """(W1 [256,64], b1, W2 [256,256], b2, W3 [96,256], b3) views of the flat parameter vector."""
    return (w[OFF_W1:OFF_B1].reshape(H, IN_PAD), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(H, H), w[OFF_B2:OFF_W3],
            w[OFF_W3:OFF_B3].reshape(OUT_PAD, H), w[OFF_B3:])


# ---------------------------------------------------------------------------------------------
# Philox4x32-10 (Salmon et al., SC'11), vectorised; counters and keys are uint32 arrays.

_M0, _M1, _W0, _W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox_vec(c0, c1, c2, c3, k0, k1) -> np.ndarray:
    c = [np.asarray(x, np.uint64) & 0xFFFFFFFF for x in (c0, c1, c2, c3)]
    c = np.broadcast_arrays(*c)
    c = [x.copy() for x in c]
    k0 = np.uint64(k0) & np.uint64(0xFFFFFFFF)
    k1 = np.uint64(k1) & np.uint64(0xFFFFFFFF)
    mask = np.uint64(0xFFFFFFFF)
    for _ in range(10):
        p0 = np.uint64(_M0) * c[0]
        p1 = np.uint64(_M1) * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & mask
        hi1, lo1 = p1 >> np.uint64(32), p1 & mask
        c = [(hi1 ^ c[1] ^ k0) & mask, lo1, (hi0 ^ c[3] ^ k1) & mask, lo0]
        k0 = (k0 + np.uint64(_W0)) & mask
        k1 = (k1 + np.uint64(_W1)) & mask
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def u01(x) -> np.ndarray:
    return (((np.asarray(x, np.uint32) >> np.uint32(8)).astype(np.float32) + np.float32(1.0)) * np.float32(2.0 ** -24))


# ---------------------------------------------------------------------------------------------
# Environment occupancy and input features (float32, the device's operation order)

def occupancy(obs: np.ndarray, W1: int = 8, wmin: float = 0.0, wmax: float = 100.0) -> np.ndarray:
    """Occupancy bits of the W1^3 R1 workspace cells, index (z*W1 + y)*W1 + x: a cell is blocked
    when >= 32 of the 4x4x4 lattice points wmin + (c + (2i+1)/8) * w1size lie in a closed box."""
    f = np.float32
    w1size = f(f(f(wmax) - f(wmin)) / f(W1))
    off = f(0.125) * np.arange(1, 8, 2, dtype=np.float32)                 # (2i+1)/8
    cells = np.arange(W1, dtype=np.float32)
    axis = (f(wmin) + ((cells[:, None] + off[None, :]).astype(np.float32) * w1size).astype(np.float32)).astype(np.float32)
    # points: [cx, ix] per axis -> full lattice per cell
    obs = np.asarray(obs, np.float32).reshape(-1, 6)
    bits = np.zeros(W1 ** 3, bool)
    for cz in range(W1):
        for cy in range(W1):
            for cx in range(W1):
                px, py, pz = np.meshgrid(axis[cx], axis[cy], axis[cz], indexing="ij")
                p = np.stack([px.ravel(), py.ravel(), pz.ravel()], 1)
                if obs.shape[0]:
                    inside = ((obs[None, :, 0:3] <= p[:, None, :]) & (p[:, None, :] <= obs[None, :, 3:6])).all(-1).any(-1)
                    cnt = int(inside.sum())
                else:
                    cnt = 0
                bits[(cz * W1 + cy) * W1 + cx] = cnt >= 32
    return bits


def pack_bits(bits: np.ndarray) -> np.ndarray:
    words = np.zeros((bits.size + 31) // 32, np.uint32)
    for i in np.nonzero(bits)[0]:
        words[i >> 5] |= np.uint32(1 << (i & 31))
    return words


def input_scale() -> np.ndarray:
    s = np.ones(IN_PAD, np.float32)
    for i in range(24):
        d = i % 12
        s[i] = np.float32(0.01) if d < 3 else (np.float32(0.1) if 6 <= d < 9 else np.float32(1.0))
    return s


def features(states: np.ndarray, goals: np.ndarray, occ_bits: np.ndarray, W1: int = 8, wmin: float = 0.0,
             wmax: float = 100.0) -> np.ndarray:
    """Features of n 12D states with goals (n x 3): scaled state, scaled goal - state (goal
    non-position components 0), 27 neighbour occupancy bits (dx fastest), zero padding."""
    f = np.float32
    s = np.asarray(states, np.float32)[:, :12]
    g = np.zeros_like(s)
    g[:, :3] = np.asarray(goals, np.float32)[:, :3]
    sc = input_scale()
    n = s.shape[0]
    x = np.zeros((n, IN_PAD), np.float32)
    x[:, :12] = (s * sc[:12]).astype(np.float32)
    x[:, 12:24] = ((g - s).astype(np.float32) * sc[12:24]).astype(np.float32)
    wspan = f(f(wmax) - f(wmin))
    t = (f(W1) * (s[:, :3] - f(wmin)).astype(np.float32)).astype(np.float32)
    q = (t / wspan).astype(np.float32)
    cell = np.clip(np.trunc(np.nan_to_num(q, nan=0.0, posinf=2 ** 30, neginf=-2 ** 30)).astype(np.int64), 0, W1 - 1)
    for j in range(27):
        d = np.array([j % 3 - 1, (j // 3) % 3 - 1, j // 9 - 1])
        c = cell + d
        out = ((c < 0) | (c >= W1)).any(1)
        idx = (np.clip(c[:, 2], 0, W1 - 1) * W1 + np.clip(c[:, 1], 0, W1 - 1)) * W1 + np.clip(c[:, 0], 0, W1 - 1)
        x[:, 24 + j] = np.where(out, 1.0, occ_bits[idx].astype(np.float32))
    return x


# ---------------------------------------------------------------------------------------------
# Forward, loss and gradient

def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(w: np.ndarray, x: np.ndarray, dtype=np.float64):
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(w))
    x = x.astype(dtype)
    z1 = x @ W1.T + b1
    a1 = silu(z1)
    z2 = a1 @ W2.T + b2
    a2 = silu(z2)
    o = a2 @ W3.T + b3
    return z1, a1, z2, a2, o


def mdn_loss_grad(o: np.ndarray, y: np.ndarray, mask) -> tuple[np.ndarray, np.ndarray]:
    """Per-sample negative log-likelihood and d(mean loss)/d(outputs) (same dtype as o)."""
    dt = o.dtype
    n = o.shape[0]
    m = np.asarray(mask, dt)
    a = o[:, 0:OUT:CSTRIDE]                                    # n x 8 logits
    mu = np.stack([o[:, k * CSTRIDE + 1:k * CSTRIDE + 1 + DIM] for k in range(COMP)], 1)        # n x 8 x 5
    raw = np.stack([o[:, k * CSTRIDE + 1 + DIM:k * CSTRIDE + 1 + 2 * DIM] for k in range(COMP)], 1)
    th = np.tanh(raw * dt.type(1.0 / SIG_HALF))
    s = dt.type(SIG_MID) + dt.type(SIG_HALF) * th
    inv = np.exp(-s)
    e = (y[:, None, :].astype(dt) - mu) * inv
    amax = a.max(1, keepdims=True)
    alse = amax + np.log(np.exp(a - amax).sum(1, keepdims=True))
    lp = (a - alse) + (m * (-0.5 * e * e - s - dt.type(0.5 * np.log(2 * np.pi)))).sum(-1)
    lmax = lp.max(1, keepdims=True)
    lse = lmax + np.log(np.exp(lp - lmax).sum(1, keepdims=True))
    loss = -lse[:, 0]
    r = np.exp(lp - lse)
    pi = np.exp(a - alse)
    g = np.zeros((n, OUT_PAD), dt)
    g[:, 0:OUT:CSTRIDE] = (pi - r) / n
    gmu = -r[:, :, None] * m * e * inv / n
    graw = -r[:, :, None] * m * (e * e - 1.0) * (1.0 - th * th) / n
    for k in range(COMP):
        g[:, k * CSTRIDE + 1:k * CSTRIDE + 1 + DIM] = gmu[:, k]
        g[:, k * CSTRIDE + 1 + DIM:k * CSTRIDE + 1 + 2 * DIM] = graw[:, k]
    return loss, g


def loss_grad(w: np.ndarray, x: np.ndarray, y: np.ndarray, mask=(1, 1, 1, 1, 1), dtype=np.float64):
    """Mean loss and its gradient with respect to the flat parameter vector."""
    z1, a1, z2, a2, o = forward(w, x, dtype)
    loss, go = mdn_loss_grad(o, y, mask)
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(w))
    g = np.zeros(NUM_PARAMS, dtype)
    gW1, gb1, gW2, gb2, gW3, gb3 = unpack(g)
    gW3[:] = go.T @ a2
    gb3[:] = go.sum(0)
    da2 = go @ W3

    def dsilu(z):
        sg = 1.0 / (1.0 + np.exp(-z))
        return sg * (1.0 + z * (1.0 - sg))

    dz2 = da2 * dsilu(z2)
    gW2[:] = dz2.T @ a1
    gb2[:] = dz2.sum(0)
    dz1 = (dz2 @ W2) * dsilu(z1)
    gW1[:] = dz1.T @ x.astype(dtype)
    gb1[:] = dz1.sum(0)
    return loss.mean(), g


def adam_step(w, g, m, v, step: int, lr: float, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step in float32 with the bias corrections folded as the kernel does."""
    f = np.float32
    c1 = f(lr / (1.0 - b1 ** step))
    c2 = f(1.0 / (1.0 - b2 ** step))
    m = (f(b1) * m + (f(1.0) - f(b1)) * g).astype(np.float32)
    v = (f(b2) * v + (f(1.0) - f(b2)) * g * g).astype(np.float32)
    w = (w - c1 * m / (np.sqrt(v * c2) + f(eps))).astype(np.float32)
    return w, m, v


# ---------------------------------------------------------------------------------------------
# BF16 inference emulation and the mixture

def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> np.uint64(16)) & np.uint64(1)) + np.uint64(0x7FFF)
    return ((u + r) & np.uint64(0xFFFF0000)).astype(np.uint32).view(np.float32)


def forward_bf16(w: np.ndarray, x: np.ndarray):
    """Tensor-core pass: BF16 inputs/weights/activations, exact products, float64 sums, FP32
    bias; returns (h1, h2, outputs) with h1/h2 the BF16-rounded activations."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(w, np.float32))
    h0 = bf16(x).astype(np.float64)
    z1 = (h0 @ bf16(W1).astype(np.float64).T).astype(np.float32) + b1
    h1 = bf16(silu(z1.astype(np.float32)).astype(np.float32))
    z2 = (h1.astype(np.float64) @ bf16(W2).astype(np.float64).T).astype(np.float32) + b2
    h2 = bf16(silu(z2.astype(np.float32)).astype(np.float32))
    o = (h2.astype(np.float64) @ bf16(W3).astype(np.float64).T).astype(np.float32) + b3
    return h1, h2, o.astype(np.float32)


def layer_bf16(h_in: np.ndarray, W: np.ndarray, b: np.ndarray, act: bool):
    """One tensor-core layer from a given BF16 input: float32 pre-activation (float64 sums)."""
    z = (bf16(h_in).astype(np.float64) @ bf16(W).astype(np.float64).T).astype(np.float32) + b
    return (silu(z.astype(np.float64)).astype(np.float32) if act else z), z


def ulp_bf16(v: np.ndarray) -> np.ndarray:
    """One BF16 unit in the last place at |v| (8 significant bits)."""
    e = np.floor(np.log2(np.maximum(np.abs(v), 1e-30)))
    return 2.0 ** (e - 7)


def tc_layer_violation(w: np.ndarray, x: np.ndarray, h1: np.ndarray, h2: np.ndarray, out: np.ndarray) -> dict:
    """Teacher-forced bounds of the tensor-core pass, each layer fed the pass's own previous layer.

    Hidden layers: BF16 activations within one BF16 ulp of the emulation, plus the error of the
    kernel's SiLU (h + h tanh(h), h = z / 2, tanh in BF16: |error| < 2^-8 |z|), plus the FP32
    accumulation error 1e-6 * sum |terms|; their mean difference at most half an ulp.  Outputs:
    FP32 sums of exact BF16 products within 1e-5 of the terms' magnitude.  Returns the largest
    excess over each bound (<= 0 everywhere when the pass is within them)."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(w, np.float32))
    res = {}
    for name, h_in, W, b, h_gpu in (("h1", x, W1, b1, h1), ("h2", h1, W2, b2, h2)):
        act, z = layer_bf16(h_in, W, b, act=True)
        want = bf16(act)
        bound = np.abs(bf16(h_in).astype(np.float64)) @ np.abs(bf16(W).astype(np.float64)).T
        diff = np.abs(np.asarray(h_gpu, np.float64) - want)
        tol = ulp_bf16(want) * 1.01 + 2.0 ** -8 * np.abs(z) + 1e-6 * bound
        res[name] = float((diff - tol).max())
        res[name + "_mean"] = float(np.mean(diff) - 0.5 * np.mean(ulp_bf16(want)))
    z = bf16(h2).astype(np.float64) @ bf16(W3).astype(np.float64).T
    bound = np.abs(bf16(h2).astype(np.float64)) @ np.abs(bf16(W3).astype(np.float64)).T
    want = (z + b3)[:, :OUT]
    tol = 1e-5 * bound[:, :OUT] + 1e-5 * np.abs(b3[:OUT]) + 1e-6
    res["out"] = float((np.abs(np.asarray(out, np.float64)[:, :OUT] - want) - tol).max())
    return res


def mixture_parts(o: np.ndarray):
    """Softmax weights (n x 8), means and sigmas (n x 8 x 5) of rows of outputs (float64)."""
    o = np.asarray(o, np.float64)
    a = o[:, 0:OUT:CSTRIDE]
    e = np.exp(a - a.max(1, keepdims=True))
    w = e / e.sum(1, keepdims=True)
    mu = np.stack([o[:, k * CSTRIDE + 1:k * CSTRIDE + 1 + DIM] for k in range(COMP)], 1)
    raw = np.stack([o[:, k * CSTRIDE + 1 + DIM:k * CSTRIDE + 1 + 2 * DIM] for k in range(COMP)], 1)
    return w, mu, np.exp(SIG_MID + SIG_HALF * np.tanh(raw / SIG_HALF))


def mixture_draws(rec: np.ndarray, u_plain: np.ndarray, eps: float, seed: int, stream: int, it: int, index: np.ndarray):
    """Draws of children `index` from the records (network outputs, one row per child) in float64:
    Philox stream 3 keeps the plain draws when its uniform is <= eps; otherwise the component is
    the first whose cumulative softmax weight reaches a stream-3 uniform (the last if none) and
    u = sigmoid(mu + sigma n) with Box-Muller normals from streams 3 and 4.  Returns (u (n x 6),
    learned mask, component, distance of the component uniform from the nearest cumulative
    weight)."""
    index = np.asarray(index, np.uint32)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    a = philox_vec(index, it, 3, stream, k0, k1)
    b = philox_vec(index, it, 4, stream, k0, k1)
    ua = u01(a).astype(np.float64)
    ub = u01(b).astype(np.float64)
    keep = ua[:, 0] <= np.float32(eps)
    w, mu_all, sg_all = mixture_parts(rec)
    cdf = np.cumsum(w, 1)
    comp = np.minimum((cdf[:, : COMP - 1] < ua[:, 1:2]).sum(1), COMP - 1)
    margin = np.abs(cdf[:, : COMP - 1] - ua[:, 1:2]).min(1)
    bm = np.concatenate([ua[:, 2:4], ub], 1)            # 6 uniforms: pairs (0,1), (2,3), (4,5)
    r = np.sqrt(-2.0 * np.log(bm[:, 0::2]))
    th = 2.0 * np.pi * bm[:, 1::2]
    nrm = np.stack([r[:, 0] * np.cos(th[:, 0]), r[:, 0] * np.sin(th[:, 0]), r[:, 1] * np.cos(th[:, 1]),
                    r[:, 1] * np.sin(th[:, 1]), r[:, 2] * np.cos(th[:, 2])], 1)
    rows = np.arange(rec.shape[0])
    z = mu_all[rows, comp] + sg_all[rows, comp] * nrm
    u_l = np.clip(1.0 / (1.0 + np.exp(-z)), 5.9604645e-8, 1.0)
    u = np.asarray(u_plain, np.float64).copy()
    u[~keep, :DIM] = u_l[~keep]
    return u, ~keep, comp, margin

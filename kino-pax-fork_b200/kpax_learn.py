"""Learned proposal for the 12D quadrotor: data harvest, GPU training and evaluation.

Harvest.  The plain planner (uniform draws, as the reference's propagateAndCheck) plans each
training scene of the family (kpax_envs.learned_family).  Every tree edge parent -> child gives a
pair (parent state, child controls).  Its goal is relabelled in hindsight (Andrychowicz et al.,
"Hindsight Experience Replay", 2017) as the position of a node further down the same branch,
drawn with probability growing with that node's distance from the root; edges of solution paths
also appear with the true goal.  Targets are the logits of the draw uniforms that produce the
edge's controls, u = (c - c_min) / (c_max - c_min), clamped to [1e-4, 1 - 1e-4].

Training.  Adam with a cosine learning-rate schedule on the mixture-density loss, through the
library's FP32 training kernels (kpax.MLP); the trained network is packed to BF16 for the
tensor-core proposal pass.

Evaluation.  The learned (epsilon-mixed) and the plain planner plan the same held-out scenes
with the same random streams: success rate and time-to-solution percentiles.

Command line:
  python kpax_learn.py train --envs 512 --pairs 1000000 --out weights/quad_proposal.npz
  python kpax_learn.py eval --weights weights/quad_proposal.npz --seeds 256 --eps 0.2
"""
from __future__ import annotations

import argparse
import json
import math
import time
from pathlib import Path

import numpy as np

import kpax
import kpax_envs as E

HERE = Path(__file__).resolve().parent
DEFAULT_WEIGHTS = HERE / "weights" / "quad_proposal.npz"
TRAIN_SEED0, EVAL_SEED0 = 100_000, 200_000
IN, IN_PAD, H, OUT, OUT_PAD = 51, 64, 256, 88, 96
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN_PAD
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + OUT_PAD * H
NUM_PARAMS = OFF_B3 + OUT_PAD
U_CLAMP = 1e-4


def quad_config(max_iter: int | None = None) -> kpax.Config:
    cfg = kpax.preset(kpax.PRESET_QUAD)
    if max_iter:
        cfg.max_iter = max_iter
    return cfg


def loss_mask(cfg: kpax.Config) -> list[float]:
    """The duration dimension is learned only when the configuration draws durations."""
    return [1.0, 1.0, 1.0, 1.0, 0.0 if cfg.fixed_steps else 1.0]


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal hidden layers, a near-zero output layer whose biases give equal mixture weights,
    zero means and sigma ~1.8 in logit space (close to the logistic spread of a uniform draw)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NUM_PARAMS, np.float32)
    w[OFF_W1:OFF_B1].reshape(H, IN_PAD)[:, :IN] = rng.normal(0.0, math.sqrt(2.0 / IN), (H, IN))
    w[OFF_W2:OFF_B2] = rng.normal(0.0, math.sqrt(2.0 / H), H * H)
    w[OFF_W3:OFF_B3].reshape(OUT_PAD, H)[:OUT] = rng.normal(0.0, 0.01 / math.sqrt(H), (OUT, H))
    b3 = w[OFF_B3:]
    raw = 5.0 * math.atanh((math.log(1.8) + 2.0) / 5.0)
    for k in range(8):
        b3[k * 11 + 1: k * 11 + 6] = rng.normal(0.0, 0.5, 5)  # spread the components' means
        b3[k * 11 + 6: k * 11 + 11] = raw
    return w


def save_params(path: Path, w: np.ndarray, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=np.asarray(w, np.float32), meta=np.array(json.dumps(meta)))


def load_params(path: Path = DEFAULT_WEIGHTS) -> tuple[np.ndarray, dict]:
    z = np.load(Path(path), allow_pickle=False)
    return z["params"].astype(np.float32), json.loads(str(z["meta"]))


def load_network(path: Path = DEFAULT_WEIGHTS, stream: int = 0) -> kpax.MLP:
    w, _ = load_params(path)
    net = kpax.MLP(max_batch=256, stream=stream)
    net.set_params(w)
    return net


# ---------------------------------------------------------------------------------------------
# harvest

def depths(parents: np.ndarray) -> np.ndarray:
    """Depth of every node (parents precede children; the root's parent is -1)."""
    d = np.zeros(parents.size, np.int32)
    if parents.size < 2:
        return d
    p = parents[1:].astype(np.int64)
    while True:
        nd = d[p] + 1
        if np.array_equal(nd, d[1:]):
            return d
        d[1:] = nd


def hindsight_pairs(rows: np.ndarray, parents: np.ndarray, n_pairs: int, rng: np.random.Generator, ray: bool = False,
                    select: str = "weighted", goal=None, elite: float = 0.02):
    """n_pairs (parent state, goal position, child controls) from one tree: a target node m is
    drawn, then an edge on its branch uniformly.  Target selection: "weighted" draws m with
    weight 1 + |pos(m) - pos(root)|; "far" uniformly among the `elite` fraction of nodes farthest
    from the root; "goal" among the `elite` fraction closest to `goal`.  The goal is m's position
    ("goal" selection: the true goal), or with `ray` a point 10-150 m from the edge's parent along
    the direction to m (the distances of goals met in planning)."""
    if rows.shape[0] < 2:
        return np.zeros((0, 12), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 4), np.float32)
    d = depths(parents)
    cand = np.nonzero(d >= 1)[0]
    if select == "weighted":
        wt = np.linalg.norm(rows[cand, :3] - rows[0, :3], axis=1) + 1.0
        m = rng.choice(cand, size=n_pairs, p=wt / wt.sum())
    else:
        key = (-np.linalg.norm(rows[cand, :3] - rows[0, :3], axis=1) if select == "far" else
               np.linalg.norm(rows[cand, :3] - np.asarray(goal, np.float32)[:3], axis=1))
        top = cand[np.argsort(key, kind="stable")[: max(1, int(cand.size * elite))]]
        m = rng.choice(top, size=n_pairs)
    lvl = np.floor(rng.random(n_pairs) * d[m]).astype(np.int64)  # edges above m: level 0 = m's own
    child = m.astype(np.int64).copy()
    for step in range(int(lvl.max(initial=0))):
        up = lvl > step
        child[up] = parents[child[up]]
    par = parents[child].astype(np.int64)
    if select == "goal":
        return rows[par, :12].copy(), np.tile(np.asarray(goal, np.float32)[:3], (n_pairs, 1)), rows[child, 12:16].copy()
    goal = rows[m, :3].copy()
    if ray:
        d = goal.astype(np.float64) - rows[par, :3]
        nrm = np.linalg.norm(d, axis=1, keepdims=True)
        far = rng.uniform(10.0, 150.0, (n_pairs, 1))
        goal = np.where(nrm > 1e-3, rows[par, :3] + d / np.maximum(nrm, 1e-3) * far, goal).astype(np.float32)
    return rows[par, :12].copy(), goal, rows[child, 12:16].copy()


def solution_pairs(tree_rows: np.ndarray, parents: np.ndarray, goal_idx: int, goal: np.ndarray):
    """Edges of the solution path from node goal_idx to the root with the true goal (none for
    goal_idx 0)."""
    nodes = []
    i = goal_idx
    while i > 0:
        nodes.append(i)
        i = int(parents[i])
    nodes = np.asarray(nodes, np.int64)
    if nodes.size == 0:
        return np.zeros((0, 12), np.float32), np.zeros((0, 3), np.float32), np.zeros((0, 4), np.float32)
    return (tree_rows[parents[nodes], :12].copy(), np.tile(goal[:3].astype(np.float32), (nodes.size, 1)),
            tree_rows[nodes, 12:16].copy())


def logit_targets(ctrl: np.ndarray, cfg: kpax.Config) -> np.ndarray:
    clo = np.array(cfg.ctrl_min[:4], np.float64)
    rng = np.array(cfg.ctrl_max[:4], np.float64) - clo
    u = np.clip((ctrl.astype(np.float64) - clo) / rng, U_CLAMP, 1.0 - U_CLAMP)
    y = np.zeros((ctrl.shape[0], 5), np.float32)
    y[:, :4] = np.log(u / (1.0 - u))
    return y


# Start-goal separation bands (m) of a mixed harvest: scene j of the training seeds draws from band
# j mod 4, so the network sees near goals (whose plans mostly succeed and contribute solution
# edges) as well as the 25-45 m family it is evaluated on.
SEP_BANDS = ((6.0, 12.0), (12.0, 20.0), (20.0, 30.0), (25.0, 45.0))


def harvest(seeds, pairs_per_env: int, cfg: kpax.Config, net: kpax.MLP | None = None, eps: float = 0.2, seed: int = 0,
            log=print, ray: bool = False, select: str = "weighted", elite: float = 0.02, sep_mix: bool = False):
    """Plans every scene of `seeds` (plain sampler, or `net` with epsilon `eps`) and returns the
    device feature / target tensors and per-scene plan statistics.  sep_mix: scene j's start and
    goal are SEP_BANDS[j % 4] apart instead of the family's 25-45 m."""
    import torch

    rng = np.random.default_rng(seed)
    planner = kpax.KPAX(cfg)
    if net is not None:
        planner.set_proposal(net, eps)
    n_total = pairs_per_env * len(seeds)
    X = torch.zeros((n_total, IN_PAD), device="cuda")
    Y = torch.zeros((n_total, 5), device="cuda")
    stats = []
    filled = 0
    t0 = time.time()
    for j, sd in enumerate(seeds):
        if sep_mix:
            lo, hi = SEP_BANDS[j % len(SEP_BANDS)]
            obs, start, goal = E.learned_family(int(sd), min_sep=lo, max_sep=hi)
        else:
            obs, start, goal = E.learned_family(int(sd))
        d_obs = torch.from_numpy(obs).cuda()
        r = planner.plan(start, goal, d_obs.data_ptr(), obs.shape[0])
        rows, parents, _ = planner.export_tree()
        stats.append({"seed": int(sd), "found": int(r.found), "ms": float(r.ms), "tree": int(r.tree_size), "iters": int(r.iters),
                      "closest": float(np.linalg.norm(rows[:, :3] - goal[:3], axis=1).min())})
        s_sol, g_sol, c_sol = solution_pairs(rows, parents, int(r.goal_idx) if r.found else 0, goal)
        k = max(0, pairs_per_env - s_sol.shape[0])
        s_h, g_h, c_h = hindsight_pairs(rows, parents, k, rng, ray=ray, select=select, goal=goal, elite=elite)
        s = np.ascontiguousarray(np.concatenate([s_sol, s_h])[:pairs_per_env], np.float32)
        g = np.ascontiguousarray(np.concatenate([g_sol, g_h])[:pairs_per_env], np.float32)
        c = np.concatenate([c_sol, c_h])[:pairs_per_env]
        n = s.shape[0]
        if n:
            env = kpax.Env(cfg, d_obs.data_ptr(), obs.shape[0])
            d_s, d_g = torch.from_numpy(s).cuda(), torch.from_numpy(g).cuda()
            kpax.mlp_features(env, d_s.data_ptr(), 12, d_g.data_ptr(), n, X[filled:filled + n].data_ptr())
            Y[filled:filled + n] = torch.from_numpy(logit_targets(c, cfg)).cuda()
            torch.cuda.synchronize()
            env.close()
            filled += n
        if log and (j + 1) % 64 == 0:
            ok = sum(x["found"] for x in stats)
            log(f"harvest {j + 1}/{len(seeds)} scenes, {filled} pairs, {ok} solved, {time.time() - t0:.1f}s")
    planner.close()
    return X[:filled], Y[:filled], stats


# ---------------------------------------------------------------------------------------------
# training

def train(X, Y, steps: int, cfg: kpax.Config, batch: int = 4096, lr: float = 1e-3, seed: int = 0, w0=None, log=print,
          val_frac: float = 0.02):
    """Adam with cosine decay on (X, Y); returns the network (packed) and a history dict."""
    import torch

    n = X.shape[0]
    g = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(n, device="cuda", generator=g)
    n_val = max(batch, int(n * val_frac)) if n > 4 * batch else 0
    val_idx, tr_idx = perm[:n_val].to(torch.int32), perm[n_val:].to(torch.int32)
    net = kpax.MLP(max_batch=batch)
    net.set_params(init_params(seed) if w0 is None else w0)
    net.set_loss_mask(loss_mask(cfg))
    hist = {"step": [], "train_loss": [], "val_loss": []}

    def val_loss():
        if not n_val:
            return float("nan")
        tot, cnt = 0.0, 0
        for a in range(0, n_val - batch + 1, batch):
            idx = val_idx[a:a + batch].long()
            xb, yb = X[idx].contiguous(), Y[idx].contiguous()
            tot += net.loss_grad(xb.data_ptr(), yb.data_ptr(), batch) * batch
            cnt += batch
        return tot / cnt

    torch.cuda.synchronize()
    t0 = time.time()
    for step in range(steps):
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
        idx = tr_idx[torch.randint(0, tr_idx.numel(), (batch,), device="cuda", generator=g)]
        want = step % 500 == 0 or step == steps - 1
        loss = net.train_step(X.data_ptr(), Y.data_ptr(), idx.data_ptr(), batch, lr_t, want_loss=want)
        if want:
            v = val_loss()
            hist["step"].append(step), hist["train_loss"].append(loss), hist["val_loss"].append(v)
            if log:
                log(f"step {step}: lr {lr_t:.2e} train {loss:.4f} val {v:.4f} ({time.time() - t0:.1f}s)")
    torch.cuda.synchronize()
    hist["seconds"] = time.time() - t0
    hist["samples_per_s"] = steps * batch / max(hist["seconds"], 1e-9)
    net.pack()
    return net, hist


# ---------------------------------------------------------------------------------------------
# evaluation

def evaluate(seeds, cfg: kpax.Config, net: kpax.MLP | None = None, eps: float = 0.2, progress: bool = False,
             family: dict | None = None):
    """Plans every held-out scene (kpax_envs.learned_family with the `family` keywords: obstacle
    range, start-goal separation); returns per-scene found / ms / iters / tree size."""
    import torch

    planner = kpax.KPAX(cfg)
    if net is not None:
        planner.set_proposal(net, eps)
    out = []
    for sd in seeds:
        obs, start, goal = E.learned_family(int(sd), **(family or {}))
        d_obs = torch.from_numpy(obs).cuda()
        r = planner.plan(start, goal, d_obs.data_ptr(), obs.shape[0])
        rec = {"seed": int(sd), "found": int(r.found), "ms": float(r.ms), "iters": int(r.iters), "tree": int(r.tree_size),
               "valid": int(r.valid_expansions), "cost": float(r.path_cost)}
        if progress:  # closest approach of the tree to the goal and its farthest reach from the start
            rows, _, _ = planner.export_tree()
            rec["closest"] = float(np.linalg.norm(rows[:, :3] - goal[:3], axis=1).min())
            rec["reach"] = float(np.linalg.norm(rows[:, :3] - start[:3], axis=1).max())
        out.append(rec)
    planner.close()
    return out


def summarize(res) -> dict:
    found = np.array([r["found"] for r in res], bool)
    ms = np.array([r["ms"] for r in res])
    tts = np.where(found, ms, np.inf)
    # time-to-solution percentiles with unsolved plans counted as infinite
    s = {"n": len(res), "success": float(found.mean()) if len(res) else 0.0,
         "p50_ms": float(np.quantile(tts, 0.50, method="inverted_cdf")) if len(res) else float("inf"),
         "p95_ms": float(np.quantile(tts, 0.95, method="inverted_cdf")) if len(res) else float("inf"),
         "p50_ms_solved": float(np.median(ms[found])) if found.any() else float("inf"),
         "mean_ms": float(ms.mean()) if len(res) else 0.0,
         "valid_per_s": float(sum(r["valid"] for r in res) / max(ms.sum() * 1e-3, 1e-12)) if res and "valid" in res[0] else 0.0}
    if res and "closest" in res[0]:
        s["closest_median"] = float(np.median([r["closest"] for r in res]))
        s["reach_median"] = float(np.median([r["reach"] for r in res]))
    return s


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--envs", type=int, default=512)
    t.add_argument("--pairs", type=int, default=1_000_000)
    t.add_argument("--steps", type=int, default=6000)
    t.add_argument("--batch", type=int, default=4096)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--rounds", type=int, default=1, help="later rounds harvest with the network of the previous round")
    t.add_argument("--eps", type=float, default=0.2)
    t.add_argument("--max-iter", type=int, default=0)
    t.add_argument("--select", choices=("weighted", "far", "goal"), default="goal")
    t.add_argument("--ray", action="store_true")
    t.add_argument("--sep-mix", action="store_true", help="harvest scenes from the four separation bands of SEP_BANDS")
    t.add_argument("--eval-seeds", type=int, default=256)
    t.add_argument("--out", type=Path, default=DEFAULT_WEIGHTS)
    e = sub.add_parser("eval")
    e.add_argument("--weights", type=Path, default=DEFAULT_WEIGHTS)
    e.add_argument("--seeds", type=int, default=256)
    e.add_argument("--eps", type=float, default=0.2)
    e.add_argument("--max-iter", type=int, default=0)
    e.add_argument("--expansions-log2", type=int, default=0, help="expansions per iteration (log2; 0 = preset)")
    e.add_argument("--tree-log2", type=int, default=0, help="tree capacity (log2; 0 = preset)")
    e.add_argument("--obs", type=int, nargs=2, default=(200, 2000), metavar=("MIN", "MAX"),
                   help="obstacle count range of the held-out scenes")
    e.add_argument("--sep", type=float, nargs=2, default=(25.0, 45.0), metavar=("MIN", "MAX"),
                   help="start-goal separation range (m) of the held-out scenes")
    pp = sub.add_parser("propose", help="time the tensor-core proposal pass on random states")
    pp.add_argument("--weights", type=Path, default=DEFAULT_WEIGHTS)
    pp.add_argument("--rows", type=int, default=1 << 16)
    pp.add_argument("--reps", type=int, default=10)
    a = ap.parse_args(argv)
    if a.cmd == "propose":
        import torch

        net = load_network(a.weights)
        obs, _, _ = E.learned_family(EVAL_SEED0)
        d_obs = torch.from_numpy(obs).cuda()
        env = kpax.Env(quad_config(), d_obs.data_ptr(), obs.shape[0])
        g = torch.Generator(device="cuda").manual_seed(0)
        st = (torch.rand((a.rows, 12), device="cuda", generator=g) * 100).contiguous()
        go = (torch.rand((a.rows, 3), device="cuda", generator=g) * 100).contiguous()
        mix = torch.zeros((a.rows, kpax.MLP_MIX), device="cuda")
        ms = []
        for _ in range(a.reps):
            net.propose(env, st.data_ptr(), 12, go.data_ptr(), a.rows, mix.data_ptr())
            ms.append(net.last_propose_ms())
        t = float(np.median(ms))
        print(json.dumps({"rows": a.rows, "ms_median": t, "tflops": a.rows * 202240 / (t * 1e-3) / 1e12}))
        return
    cfg = quad_config(a.max_iter or None)
    if a.cmd == "train":
        seeds = [TRAIN_SEED0 + i for i in range(a.envs)]
        net, w = None, None
        meta = {"envs": a.envs, "pairs": a.pairs, "steps": a.steps, "batch": a.batch, "lr": a.lr, "select": a.select,
                "ray": a.ray, "eps": a.eps, "sep_mix": bool(a.sep_mix), "rounds": []}
        eval_seeds = [EVAL_SEED0 + i for i in range(a.eval_seeds)]
        if a.eval_seeds:
            meta["plain"] = summarize(evaluate(eval_seeds, cfg, progress=True))
            print(json.dumps({"plain": meta["plain"]}))
        for rnd in range(a.rounds):
            t0 = time.time()
            X, Y, st = harvest(seeds, a.pairs // a.envs, cfg, net=net, eps=a.eps, seed=rnd, select=a.select, ray=a.ray,
                               sep_mix=a.sep_mix)
            t_h = time.time() - t0
            net, hist = train(X, Y, a.steps, cfg, a.batch, a.lr, seed=rnd, w0=w)
            w = net.get_params()
            solved = sum(x["found"] for x in st)
            rec = {"pairs": int(X.shape[0]), "harvest_s": t_h, "harvest_solved": solved, "train_s": hist["seconds"],
                   "samples_per_s": hist["samples_per_s"], "val_loss": hist["val_loss"][-1]}
            if a.eval_seeds:
                rec["learned"] = summarize(evaluate(eval_seeds, cfg, net, a.eps, progress=True))
            meta["rounds"].append(rec)
            print(json.dumps(rec))
            del X, Y
        save_params(a.out, w, meta)
        print(f"saved {a.out}")
    else:
        net = load_network(a.weights)
        seeds = [EVAL_SEED0 + i for i in range(a.seeds)]
        if a.expansions_log2:
            cfg.expansions_per_iter = 1 << a.expansions_log2
        if a.tree_log2:
            cfg.max_tree_size = 1 << a.tree_log2
        fam = {"obs_range": tuple(a.obs), "min_sep": a.sep[0], "max_sep": a.sep[1]}
        plain = summarize(evaluate(seeds, cfg, family=fam))
        learned = summarize(evaluate(seeds, cfg, net, a.eps, family=fam))
        print(json.dumps({"family": fam, "plain": plain, "learned": learned}))


if __name__ == "__main__":
    main()

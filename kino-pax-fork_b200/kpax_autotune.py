"""Autotuner of the planner's launch parameters: expansion block size, samples (children) per
thread, spatial-hash cell size, and planner iterations per captured CUDA graph.

None of these changes a plan: children are appended in child order whatever the block shape,
and the hash grid keeps every obstacle of a cell (no per-cell cap), so collision verdicts do not
depend on the cell size.  Every candidate therefore expands the identical tree, and the tuner
compares device time per iteration directly (CUDA events on the planner stream, L2 flushed
before each timed iteration) and checks that the valid-expansion totals agree.

Results are cached as JSON (tuning/autotune.json next to this file), keyed by the GPU and the
workload (model, expansions per iteration, obstacle-count bucket).

  python kpax_autotune.py --workload quad      # tune one benchmark workload and store it
  python kpax_autotune.py --workload all
"""
from __future__ import annotations

import argparse
import itertools
import json
import math
import time
from pathlib import Path

import numpy as np

import kpax
import kpax_envs as E

HERE = Path(__file__).resolve().parent
CACHE = HERE / "tuning" / "autotune.json"
SPACE = {
    "block_size": [128, 256, 448, 512],
    "samples_per_thread": [1, 2],
    "hash_cell_size": [2.5, 5.0, 10.0],
}
FLUSH_BYTES = 256 << 20
WORKLOADS = {
    "quad": (kpax.PRESET_QUAD, E.quad_scene),
    "dubins": (kpax.PRESET_DUBINS, E.dubins_scene),
    "di": (kpax.PRESET_DI, E.di_scene),
}


def gpu_key() -> str:
    import torch

    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}SM"


def obs_bucket(n_obs: int) -> int:
    """Obstacle counts in powers-of-two buckets (a tuning result covers a bucket)."""
    return 0 if n_obs <= 0 else int(math.floor(math.log2(n_obs)))


def workload_key(cfg: kpax.Config, n_obs: int) -> str:
    return f"model{cfg.model}|exp{cfg.expansions_per_iter}|obs2^{obs_bucket(n_obs)}"


def apply(cfg: kpax.Config, params: dict) -> kpax.Config:
    c = cfg.copy()
    for k, v in params.items():
        setattr(c, k, type(getattr(c, k))(v))
    return c


def measure(cfg: kpax.Config, d_obs: int, n_obs: int, start, goal, warm: int = 8, iters: int = 10):
    """Mean device ms per iteration after `warm` iterations, and the valid expansions timed."""
    pl = kpax.KPAX(cfg)
    try:
        pl.begin(start, goal, d_obs, n_obs)
        pl.iterate_timed(warm, 0)
        t, tot = pl.iterate_timed(iters, FLUSH_BYTES, split=False)
        return float(t[:, 0].mean()), tot["valid"]
    finally:
        pl.close()


def tune(cfg: kpax.Config, obstacles: np.ndarray, start, goal, space: dict = SPACE, log=print) -> tuple[dict, list]:
    """Grid search over `space`; returns the fastest parameters and the table of timings."""
    import torch

    d_obs = torch.from_numpy(np.ascontiguousarray(obstacles, np.float32)).cuda()
    keys = list(space)
    table, ref_valid = [], None
    for combo in itertools.product(*(space[k] for k in keys)):
        params = dict(zip(keys, combo))
        try:
            c = apply(cfg, params)
            if kpax.load().kpax_config_validate(c) != kpax.OK:
                continue
            ms, valid = measure(c, d_obs.data_ptr(), obstacles.shape[0], start, goal)
        except kpax.KpaxError as e:
            if log:
                log(f"  {params}: rejected ({e})")
            continue
        if ref_valid is None:
            ref_valid = valid
        if valid != ref_valid:  # every candidate must expand the identical tree
            raise RuntimeError(f"parameters {params} changed the plan: {valid} vs {ref_valid} valid expansions")
        table.append({**params, "ms_per_iter": ms})
        if log:
            log(f"  {params}: {ms * 1e3:.1f} us/iteration")
    best = min(table, key=lambda r: r["ms_per_iter"])
    return {k: best[k] for k in keys}, table


def load_cache(path: Path = CACHE) -> dict:
    p = Path(path)
    return json.loads(p.read_text()) if p.exists() else {}


def store(key_gpu: str, key_work: str, best: dict, table: list, path: Path = CACHE) -> None:
    data = load_cache(path)
    data.setdefault(key_gpu, {})[key_work] = {"best": best, "table": table, "time": time.strftime("%Y-%m-%d")}
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    Path(path).write_text(json.dumps(data, indent=1, sort_keys=True))


def tuned(cfg: kpax.Config, n_obs: int, path: Path = CACHE) -> tuple[kpax.Config, dict | None]:
    """cfg with the cached best parameters of its workload on this GPU (unchanged if none)."""
    try:
        entry = load_cache(path).get(gpu_key(), {}).get(workload_key(cfg, n_obs))
    except Exception:
        entry = None
    if not entry:
        return cfg.copy(), None
    return apply(cfg, entry["best"]), entry["best"]


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["all"], default="quad")
    ap.add_argument("--out", type=Path, default=CACHE)
    a = ap.parse_args(argv)
    names = sorted(WORKLOADS) if a.workload == "all" else [a.workload]
    for name in names:
        pre, scene = WORKLOADS[name]
        cfg = kpax.preset(pre)
        obs, start, goal = scene()
        print(f"{name}: {len(list(itertools.product(*SPACE.values())))} candidates", flush=True)
        best, table = tune(cfg, obs, start, goal)
        store(gpu_key(), workload_key(cfg, obs.shape[0]), best, table, a.out)
        default = next((r["ms_per_iter"] for r in table if r["block_size"] == 448 and r["samples_per_thread"] == 1
                        and r["hash_cell_size"] == 5.0), None)
        fastest = min(r["ms_per_iter"] for r in table)
        print(json.dumps({"workload": name, "best": best, "us_per_iter": fastest * 1e3,
                          "default_us_per_iter": default * 1e3 if default else None}), flush=True)


if __name__ == "__main__":
    main()

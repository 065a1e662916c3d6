"""Driver of the reference's own CUDA planner build (TEST INFRASTRUCTURE, never the measured product).

`oracle/_ref/kref_cuda_<cfg>` is the reference's KPAX planner compiled unmodified for sm_100a with the
configuration header `refcuda/cfg/<cfg>/config/config.h` and the harness `refcuda/ref_plan.cu`, which
times whole plans through KPAX::plan (src/planners/KPAX.cu:51-115) and reads the reference's own
valid-expansion counter (the sum of d_validCounterArray_, KPAX.cu:393).  This module writes a scene
and a query list, runs the binary under a time limit and summarises its JSON.

Configurations:
  quad_c2   the 12D quadrotor benchmark configuration (h 0.02 s, steps 1 + (int)(u * 25), Zc in [0, 2g],
            torques in [-0.1, 0.1], tree capacity 2^20)
  quad_ref  the reference's own active quadrotor block (include/config/config.h:209-307: h 0.1 s,
            steps 1 + (int)(u * 10), Zc in [0, 30], torques in [-pi, pi], capacity 400000)
"""
from __future__ import annotations

import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE.parent / "_ref"


def binary(cfg: str) -> Path:
    return REF_DIR / f"kref_cuda_{cfg}"


def run(cfg: str, obstacles: np.ndarray, queries, iteration_cap: int, repeats: int = 1,
        timeout_s: float = 300.0) -> dict:
    """Plans every query `repeats` times (queries: rows of start xyz, goal xyz).  Returns the harness's
    JSON (config, plans) or {"unavailable": reason}."""
    exe = binary(cfg)
    if not exe.exists():
        return {"unavailable": f"{exe.name} not built (the reference tree was absent at build time)"}
    with tempfile.TemporaryDirectory(prefix="kref_cuda_") as td:
        td = Path(td)
        np.savetxt(td / "obstacles.csv", np.asarray(obstacles, np.float32), fmt="%.9g", delimiter=",")
        with open(td / "queries.txt", "w") as f:
            for q in np.asarray(queries, np.float32).reshape(-1, 6):
                f.write(" ".join(f"{v:.9g}" for v in q) + "\n")
        out = td / "out.json"
        cmd = [str(exe), str(td / "obstacles.csv"), str(td / "queries.txt"), str(out), str(td / "work"),
               str(int(iteration_cap)), str(int(repeats))]
        try:
            p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"{exe.name} did not finish within {timeout_s:.0f} s"}
        if not out.exists():
            return {"unavailable": f"{exe.name} exited {p.returncode} without output: {p.stderr.strip()[-200:]}"}
        res = json.loads(out.read_text())
        if p.returncode != 0 and "unavailable" not in res:
            res = {"unavailable": f"{exe.name} exited {p.returncode}"}
        return res


def plan_seconds(plan: dict) -> float:
    """Host seconds of one KPAX::plan call without the harness's own per-iteration check."""
    return plan["wall_s"] - plan["guard_s"]


def summarise(res: dict, steady_min_children: int = 1 << 15) -> dict:
    """Whole-plan valid expansions/s, the rate of the large iterations, and plan outcomes."""
    if "unavailable" in res:
        return res
    plans = res["plans"]
    t = sum(plan_seconds(p) for p in plans)
    valid = sum(p["valid"] for p in plans)
    children = sum(p["children"] for p in plans)
    its = np.array([it for p in plans for it in p["iterations"]], np.float64).reshape(-1, 3)
    big = its[its[:, 0] >= steady_min_children] if its.size else its
    found = [p for p in plans if p["found"]]
    tts = sorted(1000.0 * plan_seconds(p) for p in found)
    return {
        "value": valid / t if t > 0 else None,
        "plans": len(plans),
        "valid": valid,
        "children": children,
        "seconds": t,
        "iterations": int(sum(p["iters"] for p in plans)),
        "capacity_stops": int(sum(p["capacity_stop"] for p in plans)),
        "steady": {
            "min_children": steady_min_children,
            "iterations": int(big.shape[0]),
            "children_per_iter": float(big[:, 0].mean()) if big.size else None,
            "ms_per_iter": float(1000 * big[:, 2].mean()) if big.size else None,
            "value": float(big[:, 1].sum() / big[:, 2].sum()) if big.size and big[:, 2].sum() > 0 else None,
        },
        "success_rate": len(found) / max(len(plans), 1),
        "tts_ms": tts,
        "path_costs": sorted(p["path_cost"] for p in found),
        "config": res["config"],
    }

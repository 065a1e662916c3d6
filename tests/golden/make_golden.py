"""Generate the golden vectors in tests/golden/ from the reference's own code.

The reference has no tests or known-answer vectors.  These fixtures are produced by running
its propagation, collision and region routines compiled for the host (oracle/_ref, built from
the reference sources by oracle/Makefile) on seeded inputs, so the GPU tests can compare the
CUDA path with the reference's outputs on a machine where the reference tree is absent.

    python tests/golden/make_golden.py

Each <config>.npz holds: obstacles, parents, draws (n x 6 uniforms: controls in draw order,
duration, frontier draw), rows and valid from propagateAndCheck*SpatialHash, valid_brute from
the brute-force propagateAndCheck*, and r1/r2 from getRegion/getSubRegion of the rows.
quad_<scene>.npz do the same for the quadrotor in the reference's own obstacle files
(include/config/obstacles/<scene>/obstacles.csv, read with the reference's CSV format).
"""
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT / "kino-pax-fork_b200"), str(ROOT / "oracle")]

import kpax  # noqa: E402
import kpax_envs as E  # noqa: E402
import oracle as O  # noqa: E402

N = 512
# the reference tree: $KPAX_REFERENCE_ROOT, else a `reference` directory beside the repository
REF_ROOT = Path(os.environ.get("KPAX_REFERENCE_ROOT", ROOT.parent / "reference"))
REF_SCENES = REF_ROOT / "include" / "config" / "obstacles"
QUAD_SCENES = ("quadTrees", "quadHouse", "quadPillars")


def edge_draws(cfg, n: int, seed: int) -> np.ndarray:
    d = E.uniform_draws(n, seed)
    d[0, :] = 1.0  # u == 1: steps = N + 1 and controls at their maxima
    d[1, :] = 2.0 ** -24  # smallest draw
    if cfg.fixed_steps:
        N_ = cfg.max_propagation_duration
        d[:, 4] = np.float32((N_ - 0.5) / N_)  # the reference draws steps; this draw gives N
    return d


def main() -> None:
    out_dir = Path(__file__).resolve().parent
    for name, pre, scene in [("di", kpax.PRESET_DI, E.di_scene), ("dubins", kpax.PRESET_DUBINS, E.dubins_scene),
                             ("quad", kpax.PRESET_QUAD, E.quad_scene)]:
        cfg = kpax.preset(pre)
        obs, start, goal = scene()
        ref = O.RefLib(cfg.model)
        overflow = ref.set_obstacles(obs)
        parents = E.sample_states(cfg.model, N, 100 + pre, cfg.v_min, cfg.v_max)
        parents[2, :3] = [-1.0, 50.0, 50.0]  # outside the workspace
        parents[3, :3] = [100.0, 0.0, 50.0]  # on the workspace boundary
        draws = edge_draws(cfg, N, 200 + pre)
        rows, valid = ref.propagate(parents, draws, use_hash=True)
        _, valid_b = ref.propagate(parents, draws, use_hash=False)
        r1, r2 = ref.regions(rows)
        np.savez_compressed(out_dir / f"{name}.npz", obstacles=obs, parents=parents, draws=draws, rows=rows, valid=valid,
                            valid_brute=valid_b, r1=r1, r2=r2, overflow_cells=np.int32(overflow),
                            start=start, goal=goal)
        print(name, "valid", valid.mean(), "overflow cells", overflow)
    cfg = kpax.preset(kpax.PRESET_QUAD)
    for k, scene in enumerate(QUAD_SCENES):
        obs = E.read_obstacles_csv(REF_SCENES / scene / "obstacles.csv")
        ref = O.RefLib(cfg.model)
        overflow = ref.set_obstacles(obs)
        parents = E.sample_states(cfg.model, N, 300 + k, cfg.v_min, cfg.v_max)
        draws = edge_draws(cfg, N, 400 + k)
        rows, valid = ref.propagate(parents, draws, use_hash=True)
        _, valid_b = ref.propagate(parents, draws, use_hash=False)
        r1, r2 = ref.regions(rows)
        np.savez_compressed(out_dir / f"quad_{scene}.npz", obstacles=obs, parents=parents, draws=draws, rows=rows,
                            valid=valid, valid_brute=valid_b, r1=r1, r2=r2, overflow_cells=np.int32(overflow))
        print(f"quad_{scene}", obs.shape[0], "obstacles, valid", valid.mean(), "overflow cells", overflow)


if __name__ == "__main__":
    main()

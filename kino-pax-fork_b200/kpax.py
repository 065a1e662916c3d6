"""ctypes binding of libkpax.so (the C ABI declared in include/kpax.h).

The Python mirror of the reference planner: ``KPAX(config).plan(h_initial, h_goal,
d_obstacles_ptr, h_obstaclesCount, saveTree)`` (src/planners/KPAX.cu:51) with the reference's
public result fields (``h_pathToGoal_``, ``h_itr_``, ``h_treeSize_``,
``h_controlPathToGoal_``; include/planners/Planner.cuh:31-43).  Device buffers are passed as
integer pointers (e.g. ``torch.Tensor.data_ptr()``).  There is no CPU fallback: loading fails
loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libkpax.so"
ABI_VERSION = 3  # KPAX_ABI_VERSION of include/kpax.h this binding was written for

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ECAPACITY, ENOTFOUND = range(7)
MODEL_DOUBLE_INTEGRATOR, MODEL_DUBINS_AIRPLANE, MODEL_QUADROTOR = 1, 2, 3
PRESET_DI, PRESET_DUBINS, PRESET_QUAD, PRESET_QUAD_REF = 0, 1, 2, 3


class KpaxError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32),
        ("state_dim", ctypes.c_int32),
        ("control_dim", ctypes.c_int32),
        ("max_tree_size", ctypes.c_uint32),
        ("max_iter", ctypes.c_uint32),
        ("step_size", ctypes.c_float),
        ("max_propagation_duration", ctypes.c_int32),
        ("fixed_steps", ctypes.c_int32),
        ("goal_thresh", ctypes.c_float),
        ("w_min", ctypes.c_float),
        ("w_max", ctypes.c_float),
        ("w_size", ctypes.c_float),
        ("c_min", ctypes.c_double),
        ("c_max", ctypes.c_double),
        ("v_min", ctypes.c_float),
        ("v_max", ctypes.c_float),
        ("ctrl_min", ctypes.c_float * 4),
        ("ctrl_max", ctypes.c_float * 4),
        ("pitch_min", ctypes.c_double),
        ("pitch_max", ctypes.c_double),
        ("c_dim", ctypes.c_int32),
        ("v_dim", ctypes.c_int32),
        ("w_r1_length", ctypes.c_int32),
        ("c_r1_length", ctypes.c_int32),
        ("v_r1_length", ctypes.c_int32),
        ("w_r2_length", ctypes.c_int32),
        ("c_r2_length", ctypes.c_int32),
        ("v_r2_length", ctypes.c_int32),
        ("region_compat", ctypes.c_int32),
        ("epsilon", ctypes.c_float),
        ("hash_cell_size", ctypes.c_float),
        ("expansions_per_iter", ctypes.c_uint32),
        ("children_per_entry", ctypes.c_uint32),
        ("root_repeat", ctypes.c_uint32),
        ("sparse_repeat", ctypes.c_uint32),
        ("sparse_valid_threshold", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("block_size", ctypes.c_int32),
        ("unroll_iters", ctypes.c_int32),
        ("samples_per_thread", ctypes.c_int32),
        ("prune", ctypes.c_int32),
        ("prune_goal_bias", ctypes.c_float),
        ("prune_exploration_bias", ctypes.c_float),
        ("prune_progress_scale", ctypes.c_float),
        ("iteration_kernels", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 2),
    ]

    @property
    def sample_dim(self) -> int:
        return self.state_dim + self.control_dim + 1

    def copy(self) -> "Config":
        c = Config()
        ctypes.pointer(c)[0] = self
        return c


class Result(ctypes.Structure):
    _fields_ = [
        ("found", ctypes.c_int32),
        ("goal_idx", ctypes.c_uint32),
        ("path_len", ctypes.c_uint32),
        ("tree_size", ctypes.c_uint32),
        ("iters", ctypes.c_uint32),
        ("tree_full", ctypes.c_int32),
        ("h_path", ctypes.POINTER(ctypes.c_float)),
        ("ms", ctypes.c_double),
        ("expansions", ctypes.c_uint64),
        ("valid_expansions", ctypes.c_uint64),
        ("path_cost", ctypes.c_double),
    ]


class FrontierStats(ctypes.Structure):
    _fields_ = [("R", ctypes.c_uint32), ("k", ctypes.c_uint32), ("E", ctypes.c_uint32), ("n", ctypes.c_uint32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("ms", ctypes.c_double), ("iters", ctypes.c_uint32), ("found", ctypes.c_uint32),
                ("expansions", ctypes.c_uint64), ("valid_expansions", ctypes.c_uint64), ("steps", ctypes.c_uint64)]


class IterTiming(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_float), ("ms_frontier", ctypes.c_float), ("ms_expand", ctypes.c_float),
                ("ms_scores", ctypes.c_float)]


_VP, _U32, _I32, _F = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(ctypes.c_float)
_SIGNATURES = {
    "kpax_config_preset": (_I32, [_I32, ctypes.POINTER(Config)]),
    "kpax_config_validate": (_I32, [ctypes.POINTER(Config)]),
    "kpax_config_sizes": (_I32, [ctypes.POINTER(Config), _VP, _VP, _VP]),
    "kpax_last_error": (ctypes.c_char_p, []),
    "kpax_abi_version": (_I32, []),
    "kpax_create": (_I32, [ctypes.POINTER(Config), ctypes.POINTER(_VP)]),
    "kpax_destroy": (_I32, [_VP]),
    "kpax_plan": (_I32, [_VP, _VP, _VP, _VP, _U32, _I32, ctypes.POINTER(Result)]),
    "kpax_plan_bench": (_I32, [_VP, _VP, _VP, _VP, _U32, _I32, ctypes.c_char_p, ctypes.POINTER(Result)]),
    "kpax_plan_host": (_I32, [_VP, _VP, _VP, _VP, _U32, ctypes.POINTER(Result)]),
    "kpax_plan_begin": (_I32, [_VP, _VP, _VP, _VP, _U32]),
    "kpax_plan_iterate": (_I32, [_VP, _U32, _I32]),
    "kpax_plan_result": (_I32, [_VP, ctypes.POINTER(Result)]),
    "kpax_plan_iterate_timed": (_I32, [_VP, _U32, ctypes.c_uint64, _I32, _VP, _VP]),
    "kpax_planner_stream": (_VP, [_VP]),
    "kpax_export_tree": (_I32, [_VP, _VP, _VP, _VP, _U32, _VP]),
    "kpax_export_regions": (_I32, [_VP, _VP, _VP, _VP, _VP]),
    "kpax_export_frontier": (_I32, [_VP, _VP, _VP, _U32]),
    "kpax_debug_capture": (_I32, [_VP, _I32]),
    "kpax_export_children": (_I32, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _U32, _VP]),
    "kpax_env_create": (_I32, [ctypes.POINTER(Config), _VP, _U32, _VP, ctypes.POINTER(_VP)]),
    "kpax_env_destroy": (_I32, [_VP]),
    "kpax_env_stats": (_I32, [_VP, _VP, _VP]),
    "kpax_propagate_batch": (_I32, [ctypes.POINTER(Config), _VP, _VP, _VP, _U32, _U32, _VP, _VP, _VP, _VP]),
    "kpax_fp32_peak": (_I32, [ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _VP]),
    "kpax_propagate_batch_noalloc": (_I32, [ctypes.POINTER(Config), _VP, _U32, _VP, _VP, _U32, _U32, _VP, _VP, _VP,
                                             _VP]),
    "kpax_collide_batch": (_I32, [_VP, _VP, _VP, _U32, _VP, _VP]),
    "kpax_region_batch": (_I32, [ctypes.POINTER(Config), _VP, _U32, _VP, _VP, _VP]),
    "kpax_frontier_compact": (_I32, [ctypes.POINTER(Config), _VP, _U32, _U32, _VP, ctypes.POINTER(FrontierStats), _VP]),
    "kpax_test_wait_timeout": (_I32, [_U32, ctypes.POINTER(_U32), _VP]),
    "kpax_kernel_launches": (ctypes.c_uint64, []),
    "kpax_batch_create": (_I32, [_VP, _U32, ctypes.POINTER(_VP)]),
    "kpax_batch_destroy": (_I32, [_VP]),
    "kpax_batch_plan": (_I32, [_VP, _VP, _VP, _U32, _VP, _VP, _VP, ctypes.POINTER(BatchStats)]),
    "kpax_test_sincos": (_I32, [_VP, _U32, _VP, _VP]),
    "kpax_mlp_create": (_I32, [_U32, ctypes.POINTER(_VP)]),
    "kpax_mlp_destroy": (_I32, [_VP]),
    "kpax_mlp_num_params": (_U32, []),
    "kpax_mlp_set_params": (_I32, [_VP, _VP, _VP]),
    "kpax_mlp_get_params": (_I32, [_VP, _VP, _VP]),
    "kpax_mlp_set_loss_mask": (_I32, [_VP, _VP, _VP]),
    "kpax_mlp_pack": (_I32, [_VP, _VP]),
    "kpax_mlp_forward": (_I32, [_VP, _VP, _U32, _VP, _VP]),
    "kpax_mlp_loss_grad": (_I32, [_VP, _VP, _VP, _U32, _VP, _VP, _VP]),
    "kpax_mlp_train_step": (_I32, [_VP, _VP, _VP, _VP, _U32, ctypes.c_float, _VP, _VP]),
    "kpax_mlp_adam_state": (_I32, [_VP, _VP, _VP, _VP, _VP]),
    "kpax_env_occupancy": (_I32, [_VP, _VP, _VP]),
    "kpax_mlp_features": (_I32, [_VP, _VP, _U32, _VP, _U32, _VP, _VP]),
    "kpax_mlp_propose": (_I32, [_VP, _VP, _VP, _U32, _VP, _U32, _VP, _VP, _VP, _VP, _VP]),
    "kpax_mlp_last_propose_ms": (ctypes.c_float, [_VP]),
    "kpax_set_proposal": (_I32, [_VP, _VP, ctypes.c_float]),
    "kpax_write_rows_csv": (_I32, [_VP, _U32, _U32, ctypes.c_char_p, _I32]),
    "kpax_read_obstacles_csv": (_I32, [ctypes.c_char_p, _VP, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "kpax_rekino_defaults": (_I32, [_VP]),
    "kpax_rekino_create": (_I32, [ctypes.POINTER(Config), _VP, ctypes.POINTER(_VP)]),
    "kpax_rekino_destroy": (_I32, [_VP]),
    "kpax_rekino_plan": (_I32, [_VP, _VP, _VP, _VP, _U32, ctypes.POINTER(Result)]),
    "kpax_write_solution_csv": (_I32, [_VP, ctypes.c_char_p, _I32]),
    "kpax_export_proposal": (_I32, [_VP, _VP, _U32, _VP]),
    "kpax_batch_set_proposal": (_I32, [_VP, _VP, ctypes.c_float, _VP]),
}

MLP_FEATURES, MLP_OUTPUTS, MLP_MIX, MLP_HIDDEN = 64, 96, 88, 256


class RekinoParams(ctypes.Structure):
    _fields_ = [("num_warps", ctypes.c_uint32), ("samples_per_thread", ctypes.c_uint32), ("epsilon_greedy", ctypes.c_float),
                ("max_iterations", ctypes.c_uint32), ("timeout_ms", ctypes.c_double), ("reserved", ctypes.c_uint32 * 4)]

_lib = None


def load(path: os.PathLike | None = None) -> ctypes.CDLL:
    """Load libkpax.so (built by `make -C kino-pax-fork_b200`); raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `make -C {HERE}` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(p))
    # the version first: a library of another version may lack some of the entries bound below
    ver = getattr(lib, "kpax_abi_version", None)
    if ver is None:
        raise ImportError(f"{p} exports no kpax_abi_version: rebuild it")
    ver.restype, ver.argtypes = ctypes.c_int32, []
    if ver() != ABI_VERSION:
        raise ImportError(f"{p} has ABI version {ver()}, this binding expects {ABI_VERSION}: rebuild it")
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    if path is None:
        _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def check(status: int, where: str) -> None:
    if status != OK:
        raise KpaxError(status, where, load().kpax_last_error().decode(errors="replace"))


def preset(which: int) -> Config:
    c = Config()
    check(load().kpax_config_preset(which, ctypes.byref(c)), "kpax_config_preset")
    return c


def sizes(cfg: Config) -> tuple[int, int, int]:
    a, b, s = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    check(load().kpax_config_sizes(ctypes.byref(cfg), ctypes.byref(a), ctypes.byref(b), ctypes.byref(s)), "kpax_config_sizes")
    return a.value, b.value, s.value


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Env:
    """Spatial-hash grid over a device obstacle buffer (n x 6 floats)."""

    def __init__(self, cfg: Config, d_obstacles: int, n_obs: int, stream: int = 0):
        self._h = _VP()
        check(load().kpax_env_create(ctypes.byref(cfg), d_obstacles, n_obs, stream, ctypes.byref(self._h)), "kpax_env_create")

    @property
    def handle(self) -> int:
        return self._h.value

    def stats(self) -> tuple[int, int]:
        a, b = ctypes.c_uint32(), ctypes.c_uint32()
        check(load().kpax_env_stats(self._h, ctypes.byref(a), ctypes.byref(b)), "kpax_env_stats")
        return a.value, b.value

    def close(self) -> None:
        if self._h:
            load().kpax_env_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def propagate_batch(cfg: Config, env: Env, d_parents: int, d_draws: int | None, draw_stream: int, n: int, d_rows: int,
                    d_valid: int, d_steps: int | None = None, stream: int = 0) -> None:
    check(load().kpax_propagate_batch(ctypes.byref(cfg), env.handle, d_parents, d_draws or None, draw_stream, n, d_rows,
                                      d_valid, d_steps or None, stream), "kpax_propagate_batch")


def propagate_batch_noalloc(cfg: Config, d_obstacles: int, n_obs: int, d_parents: int, d_draws: int | None,
                            draw_stream: int, n: int, d_rows: int, d_valid: int, d_steps: int | None = None,
                            stream: int = 0) -> None:
    """kpax_propagate_batch without any device allocation (grid in the library's fixed array)."""
    check(load().kpax_propagate_batch_noalloc(ctypes.byref(cfg), d_obstacles or None, n_obs, d_parents, d_draws or None,
                                              draw_stream, n, d_rows, d_valid, d_steps or None, stream),
          "kpax_propagate_batch_noalloc")


def collide_batch(env: Env, d_bbmin: int, d_bbmax: int, n: int, d_free: int, stream: int = 0) -> None:
    check(load().kpax_collide_batch(env.handle, d_bbmin, d_bbmax, n, d_free, stream), "kpax_collide_batch")


def region_batch(cfg: Config, d_states: int, n: int, d_r1: int, d_r2: int | None, stream: int = 0) -> None:
    check(load().kpax_region_batch(ctypes.byref(cfg), d_states, n, d_r1, d_r2 or None, stream), "kpax_region_batch")


def frontier_compact(cfg: Config, d_repeat: int, n_nodes: int, budget: int, d_entries: int, stream: int = 0) -> dict:
    """The planner's frontier compaction on repeat bytes at d_repeat (kpax_frontier_compact):
    entry node ids to d_entries, repeats of the nodes taken set to 0; returns R, k, E, n."""
    st = FrontierStats()
    check(load().kpax_frontier_compact(ctypes.byref(cfg), d_repeat, n_nodes, budget, d_entries or None, ctypes.byref(st),
                                       stream), "kpax_frontier_compact")
    return {"R": st.R, "k": st.k, "E": st.E, "n": st.n}


def test_wait_timeout(spin_limit: int, stream: int = 0) -> None:
    """Runs the expansion's look-back wait against a tile that never publishes (kpax_test_wait_timeout):
    raises KpaxError with status ETIMEOUT once the wait gives up."""
    st = ctypes.c_uint32(0)
    check(load().kpax_test_wait_timeout(spin_limit, ctypes.byref(st), stream), "kpax_test_wait_timeout")


def fp32_peak(iters: int = 1 << 16, stream: int = 0) -> tuple[float, float]:
    """Measured FP32 rate of the GPU (TFLOP/s) and the timed launch's ms (kpax_fp32_peak)."""
    t, ms = ctypes.c_double(), ctypes.c_double()
    check(load().kpax_fp32_peak(iters, ctypes.byref(t), ctypes.byref(ms), stream), "kpax_fp32_peak")
    return t.value, ms.value


def kernel_launches() -> int:
    return int(load().kpax_kernel_launches())


class KPAX:
    """Planner handle with the reference's plan() entry and public result fields."""

    def __init__(self, cfg: Config):
        self.cfg = cfg.copy()
        self.num_r1, self.r2_per_r1, self.sample_dim = sizes(self.cfg)
        self._h = _VP()
        check(load().kpax_create(ctypes.byref(self.cfg), ctypes.byref(self._h)), "kpax_create")
        self.result = Result()
        self.h_pathToGoal_ = 0
        self.h_itr_ = 0
        self.h_treeSize_ = 0
        self.h_controlPathToGoal_ = np.zeros((0, self.sample_dim), np.float32)

    @property
    def stream(self) -> int:
        return load().kpax_planner_stream(self._h) or 0

    def _publish(self) -> Result:
        r = self.result
        self.h_pathToGoal_ = int(r.goal_idx)
        self.h_itr_ = int(r.iters)
        self.h_treeSize_ = int(r.tree_size)
        if r.path_len:
            flat = np.ctypeslib.as_array(r.h_path, shape=(r.path_len * self.sample_dim,))
            self.h_controlPathToGoal_ = flat.reshape(r.path_len, self.sample_dim).copy()
        else:
            self.h_controlPathToGoal_ = np.zeros((0, self.sample_dim), np.float32)
        return r

    @staticmethod
    def _row(x, S: int) -> np.ndarray:
        a = np.zeros(S, np.float32)
        x = np.asarray(x, np.float32).ravel()
        a[: min(S, x.size)] = x[:S]
        return a

    def plan(self, h_initial, h_goal, d_obstacles_ptr: int, h_obstaclesCount: int, saveTree: bool = False) -> Result:
        S = self.sample_dim
        init, goal = self._row(h_initial, S), self._row(h_goal, S)
        check(load().kpax_plan(self._h, _ptr(init), _ptr(goal), d_obstacles_ptr, h_obstaclesCount, int(saveTree),
                               ctypes.byref(self.result)), "kpax_plan")
        return self._publish()

    def planBench(self, h_initial, h_goal, d_obstacles_ptr: int, h_obstaclesCount: int, benchItr: int,
                  out_dir: str | os.PathLike = ".") -> Result:
        """KPAX::planBench: the plan with the reference's per-iteration CSV dumps under out_dir/Data."""
        S = self.sample_dim
        init, goal = self._row(h_initial, S), self._row(h_goal, S)
        check(load().kpax_plan_bench(self._h, _ptr(init), _ptr(goal), d_obstacles_ptr, h_obstaclesCount, int(benchItr),
                                     os.fsencode(os.fspath(out_dir)), ctypes.byref(self.result)), "kpax_plan_bench")
        return self._publish()

    def plan_host(self, h_initial, h_goal, obstacles: np.ndarray) -> Result:
        S = self.sample_dim
        init, goal = self._row(h_initial, S), self._row(h_goal, S)
        obs = np.ascontiguousarray(obstacles, np.float32).reshape(-1, 6)
        check(load().kpax_plan_host(self._h, _ptr(init), _ptr(goal), _ptr(obs), obs.shape[0], ctypes.byref(self.result)),
              "kpax_plan_host")
        return self._publish()

    def begin(self, h_initial, h_goal, d_obstacles_ptr: int, n_obs: int) -> None:
        S = self.sample_dim
        init, goal = self._row(h_initial, S), self._row(h_goal, S)
        check(load().kpax_plan_begin(self._h, _ptr(init), _ptr(goal), d_obstacles_ptr, n_obs), "kpax_plan_begin")

    def iterate(self, n_iters: int, stop_at_goal: bool = False) -> None:
        check(load().kpax_plan_iterate(self._h, n_iters, int(stop_at_goal)), "kpax_plan_iterate")

    def iterate_timed(self, n_iters: int, flush_bytes: int = 0, split: bool = True):
        """Per-iteration kernel times (ms: total, frontier, expand, scores) and the totals
        (children, valid children, RK4 steps, appended nodes) over the n_iters.  split=False
        times whole iterations only (no events between their kernels; the parts read 0)."""
        times = (IterTiming * max(n_iters, 1))()
        totals = np.zeros(4, np.uint64)
        check(load().kpax_plan_iterate_timed(self._h, n_iters, flush_bytes, int(split), ctypes.addressof(times),
                                             _ptr(totals)), "kpax_plan_iterate_timed")
        t = np.array([[x.ms_total, x.ms_frontier, x.ms_expand, x.ms_scores] for x in times[:n_iters]], np.float64)
        return t, {"children": int(totals[0]), "valid": int(totals[1]), "steps": int(totals[2]), "appended": int(totals[3])}

    def finish(self) -> Result:
        check(load().kpax_plan_result(self._h, ctypes.byref(self.result)), "kpax_plan_result")
        return self._publish()

    def export_tree(self, max_rows: int | None = None):
        n_max = max_rows or self.cfg.max_tree_size
        rows = np.zeros((n_max, self.sample_dim), np.float32)
        parents = np.zeros(n_max, np.int32)
        costs = np.zeros(n_max, np.float32)
        n = ctypes.c_uint32()
        check(load().kpax_export_tree(self._h, _ptr(rows), _ptr(parents), _ptr(costs), n_max, ctypes.byref(n)),
              "kpax_export_tree")
        k = n.value
        return rows[:k], parents[:k], costs[:k]

    def export_regions(self):
        words = (self.num_r1 * self.r2_per_r1 + 31) // 32
        counter = np.zeros(self.num_r1, np.int32)
        valid = np.zeros(self.num_r1, np.int32)
        scores = np.zeros(self.num_r1, np.float32)
        bits = np.zeros(words, np.uint32)
        check(load().kpax_export_regions(self._h, _ptr(counter), _ptr(valid), _ptr(scores), _ptr(bits)), "kpax_export_regions")
        return counter, valid, scores, bits

    def export_frontier(self, n: int):
        rep = np.zeros(n, np.uint8)
        r1 = np.zeros(n, np.int32)
        check(load().kpax_export_frontier(self._h, _ptr(rep), _ptr(r1), n), "kpax_export_frontier")
        return rep, r1

    def set_proposal(self, net: "MLP | None", epsilon: float = 0.2) -> None:
        """Learned proposal on (net) or off (None) for this quadrotor planner."""
        check(load().kpax_set_proposal(self._h, net.handle if net else None, float(epsilon)), "kpax_set_proposal")

    def write_solution_csv(self, filename, append: bool = False) -> None:
        """The last plan's path (goal first, root last) in the reference's controlPathToGoal.csv format."""
        check(load().kpax_write_solution_csv(self._h, os.fsencode(filename), int(append)), "kpax_write_solution_csv")

    def export_proposal(self) -> np.ndarray:
        """Mixture records of the last iteration's frontier entries (E x 88)."""
        mix = np.zeros((self.cfg.expansions_per_iter, MLP_MIX), np.float32)
        n = ctypes.c_uint32()
        check(load().kpax_export_proposal(self._h, _ptr(mix), mix.shape[0], ctypes.byref(n)), "kpax_export_proposal")
        return mix[: n.value]

    def debug_capture(self, on: bool = True) -> None:
        check(load().kpax_debug_capture(self._h, int(on)), "kpax_debug_capture")

    def export_children(self):
        n_max = self.cfg.expansions_per_iter
        rows = np.zeros((n_max, self.sample_dim), np.float32)
        valid = np.zeros(n_max, np.uint8)
        r1 = np.zeros(n_max, np.int32)
        r2 = np.zeros(n_max, np.int32)
        nxt = np.zeros(n_max, np.uint8)
        par = np.zeros(n_max, np.int32)
        n = ctypes.c_uint32()
        check(load().kpax_export_children(self._h, _ptr(rows), _ptr(valid), _ptr(r1), _ptr(r2), _ptr(nxt), _ptr(par), n_max,
                                          ctypes.byref(n)), "kpax_export_children")
        k = n.value
        return rows[:k], valid[:k], r1[:k], r2[:k], nxt[:k], par[:k]

    def close(self) -> None:
        if self._h:
            load().kpax_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent queries planned together: every iteration stage is one launch per kernel
    over all queries (models may differ between queries)."""

    def __init__(self, cfgs):
        self.cfgs = [c.copy() for c in cfgs]
        arr = (Config * len(self.cfgs))(*self.cfgs)
        self._h = _VP()
        check(load().kpax_batch_create(ctypes.addressof(arr), len(self.cfgs), ctypes.byref(self._h)), "kpax_batch_create")
        self.n = len(self.cfgs)
        self.stride = max(c.sample_dim for c in self.cfgs)

    def set_proposal(self, net: "MLP | None", epsilon: float = 0.2, enable=None) -> None:
        """Learned proposal for the quadrotor queries (enable: per-query flags, None = all)."""
        en = None if enable is None else np.ascontiguousarray(enable, np.uint8)
        check(load().kpax_batch_set_proposal(self._h, net.handle if net else None, float(epsilon),
                                             None if en is None else _ptr(en)), "kpax_batch_set_proposal")
        self._enable = en

    def plan(self, starts, goals, d_obstacles, n_obs):
        """starts/goals: per-query state vectors; d_obstacles: device pointers; n_obs: counts."""
        S = self.stride
        init = np.zeros((self.n, S), np.float32)
        goal = np.zeros((self.n, S), np.float32)
        for q in range(self.n):
            a, b = np.asarray(starts[q], np.float32).ravel(), np.asarray(goals[q], np.float32).ravel()
            init[q, : min(S, a.size)] = a[:S]
            goal[q, : min(S, b.size)] = b[:S]
        ptrs = (ctypes.c_void_p * self.n)(*[int(p) for p in d_obstacles])
        counts = np.ascontiguousarray(n_obs, np.uint32)
        res = (Result * self.n)()
        stats = BatchStats()
        check(load().kpax_batch_plan(self._h, _ptr(init), _ptr(goal), S, ctypes.addressof(ptrs), _ptr(counts),
                                     ctypes.addressof(res), ctypes.byref(stats)), "kpax_batch_plan")
        out = []
        for q in range(self.n):
            r = res[q]
            sd = self.cfgs[q].sample_dim
            path = (np.ctypeslib.as_array(r.h_path, shape=(r.path_len * sd,)).reshape(r.path_len, sd).copy()
                    if r.path_len else np.zeros((0, sd), np.float32))
            out.append({f: getattr(r, f) for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full", "ms",
                                                     "expansions", "valid_expansions", "path_cost")} | {"path": path})
        return out, {f: getattr(stats, f) for f in ("ms", "iters", "found", "expansions", "valid_expansions", "steps")}

    def close(self) -> None:
        if self._h:
            load().kpax_batch_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """The learned proposal network: FP32 parameters trained by the library's SIMT kernels and a
    packed BF16 image for the tensor-core inference pass.  Device buffers are integer pointers."""

    def __init__(self, max_batch: int = 4096, stream: int = 0):
        self._h = _VP()
        self.stream = stream
        self.max_batch = max_batch
        check(load().kpax_mlp_create(max_batch, ctypes.byref(self._h)), "kpax_mlp_create")
        self.num_params = int(load().kpax_mlp_num_params())

    @property
    def handle(self) -> int:
        return self._h.value

    def set_params(self, params: np.ndarray) -> None:
        w = np.ascontiguousarray(params, np.float32).ravel()
        if w.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {w.size}")
        check(load().kpax_mlp_set_params(self._h, _ptr(w), self.stream), "kpax_mlp_set_params")

    def get_params(self) -> np.ndarray:
        w = np.zeros(self.num_params, np.float32)
        check(load().kpax_mlp_get_params(self._h, _ptr(w), self.stream), "kpax_mlp_get_params")
        return w

    def set_loss_mask(self, mask) -> None:
        m = np.ascontiguousarray(mask, np.float32).ravel()
        check(load().kpax_mlp_set_loss_mask(self._h, _ptr(m), self.stream), "kpax_mlp_set_loss_mask")

    def pack(self) -> None:
        check(load().kpax_mlp_pack(self._h, self.stream), "kpax_mlp_pack")

    def forward(self, d_x: int, n: int, d_out: int) -> None:
        check(load().kpax_mlp_forward(self._h, d_x, n, d_out, self.stream), "kpax_mlp_forward")

    def loss_grad(self, d_x: int, d_y: int, n: int, d_grad: int | None = None) -> float:
        loss = ctypes.c_float()
        check(load().kpax_mlp_loss_grad(self._h, d_x, d_y, n, ctypes.byref(loss), d_grad or None, self.stream),
              "kpax_mlp_loss_grad")
        return float(loss.value)

    def train_step(self, d_x: int, d_y: int, d_idx: int, batch: int, lr: float, want_loss: bool = False) -> float | None:
        loss = ctypes.c_float()
        check(load().kpax_mlp_train_step(self._h, d_x, d_y, d_idx, batch, float(lr),
                                         ctypes.byref(loss) if want_loss else None, self.stream), "kpax_mlp_train_step")
        return float(loss.value) if want_loss else None

    def adam_state(self):
        m = np.zeros(self.num_params, np.float32)
        v = np.zeros(self.num_params, np.float32)
        step = ctypes.c_uint64()
        check(load().kpax_mlp_adam_state(self._h, _ptr(m), _ptr(v), ctypes.byref(step), self.stream), "kpax_mlp_adam_state")
        return m, v, int(step.value)

    def propose(self, env: Env, d_states: int, stride: int, d_goals: int, n: int, d_mix: int, d_out: int | None = None,
                d_h1: int | None = None, d_h2: int | None = None) -> None:
        check(load().kpax_mlp_propose(self._h, env.handle, d_states, stride, d_goals, n, d_mix, d_out or None, d_h1 or None,
                                      d_h2 or None, self.stream), "kpax_mlp_propose")

    def last_propose_ms(self) -> float:
        return float(load().kpax_mlp_last_propose_ms(self._h))

    def close(self) -> None:
        if self._h:
            load().kpax_mlp_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_csv_floats(filename) -> np.ndarray:
    """Every float of an obstacle CSV file through the C ABI (readObstaclesFromCSV's token rule)."""
    L, name = load(), os.fsencode(filename)
    n, m = ctypes.c_uint64(0), ctypes.c_uint64(0)
    check(L.kpax_read_obstacles_csv(name, None, 0, ctypes.byref(n)), "kpax_read_obstacles_csv")
    out = np.zeros(n.value, np.float32)
    check(L.kpax_read_obstacles_csv(name, _ptr(out) if n.value else None, n.value, ctypes.byref(m)),
          "kpax_read_obstacles_csv")
    return out[: min(n.value, m.value)]


def read_obstacles_csv(filename) -> np.ndarray:
    """Obstacles of a CSV file (n x 6 float32) through the C ABI: the first n // 6 rows of its floats."""
    v = read_csv_floats(filename)
    k = v.size // 6
    return v[: 6 * k].reshape(k, 6)


def write_rows_csv(rows: np.ndarray, filename, append: bool = False) -> None:
    """Rows as CSV in the reference's format (6 decimals, comma-separated)."""
    a = np.ascontiguousarray(rows, np.float32)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    check(load().kpax_write_rows_csv(_ptr(a), a.shape[0], a.shape[1], os.fsencode(filename), int(append)),
          "kpax_write_rows_csv")


def env_occupancy(env: Env, d_words: int, stream: int = 0) -> None:
    check(load().kpax_env_occupancy(env.handle, d_words, stream), "kpax_env_occupancy")


def mlp_features(env: Env, d_states: int, stride: int, d_goals: int, n: int, d_x: int, stream: int = 0) -> None:
    check(load().kpax_mlp_features(env.handle, d_states, stride, d_goals, n, d_x, stream), "kpax_mlp_features")


class ReKinoLite:
    """The fork's warp-greedy planner (src/ReKino/ReKinoLite.cu) on the library's kernels; plan()
    returns the Result with the winning warp in goal_idx and its path (goal first)."""

    def __init__(self, cfg: Config, **params):
        self.cfg = cfg.copy()
        self.params = RekinoParams()
        check(load().kpax_rekino_defaults(ctypes.byref(self.params)), "kpax_rekino_defaults")
        for k, v in params.items():
            setattr(self.params, k, v)
        self.sample_dim = sizes(self.cfg)[2]
        self._h = _VP()
        check(load().kpax_rekino_create(ctypes.byref(self.cfg), ctypes.byref(self.params), ctypes.byref(self._h)),
              "kpax_rekino_create")
        self.result = Result()

    def plan(self, h_initial, h_goal, d_obstacles_ptr: int, n_obs: int):
        S = self.sample_dim
        init, goal = KPAX._row(h_initial, S), KPAX._row(h_goal, S)
        check(load().kpax_rekino_plan(self._h, _ptr(init), _ptr(goal), d_obstacles_ptr, n_obs, ctypes.byref(self.result)),
              "kpax_rekino_plan")
        r = self.result
        path = (np.ctypeslib.as_array(r.h_path, shape=(r.path_len * S,)).reshape(r.path_len, S).copy() if r.path_len
                else np.zeros((0, S), np.float32))
        return r, path

    def close(self) -> None:
        if self._h:
            load().kpax_rekino_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""ctypes loaders for the oracle libraries — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, and only
as the checker or the timed CPU baseline.

  liboracle.so            CPU restatement (kpax_oracle.c / kpax_oracle.h)
  _ref/libkref_<cfg>.so   the reference's own propagation, collision and region routines compiled
                          for the host from the reference sources (see Makefile); cfg in
                          {di, dubins, quad} with the macro values of the benchmark configurations
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_NAMES = {1: "di", 2: "dubins", 3: "quad"}
_VP, _U32, _I32, _F32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_float


class SegDiag(ctypes.Structure):
    _fields_ = [("margin", ctypes.c_float), ("nonfinite", ctypes.c_int32), ("fail_kind", ctypes.c_int32)]


def build() -> None:
    """Build liboracle.so and, where the reference tree exists, the _ref libraries."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = ORACLE_DIR / "liboracle.so"
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        sig = {
            "ko_philox4x32_10": (None, [_VP, _VP, _VP]),
            "ko_child_draws": (None, [ctypes.c_uint64, _U32, _U32, _U32, _VP]),
            "ko_reactivate_draw": (_F32, [ctypes.c_uint64, _U32, _U32, _U32]),
            "ko_env_create": (_VP, [_VP, _VP, _U32]),
            "ko_env_destroy": (None, [_VP]),
            "ko_env_grid": (None, [_VP, _VP, _VP, _VP, _VP]),
            "ko_collide_hash": (_I32, [_VP, _VP, _VP]),
            "ko_collide_brute": (_I32, [_VP, _U32, _VP, _VP]),
            "ko_separation": (_F32, [_VP, _U32, _VP, _VP]),
            "ko_propagate_batch": (None, [_VP, _VP, _VP, _VP, _U32, _U32, _VP, _VP, _VP, _VP, ctypes.c_int]),
            "ko_integrate_f64": (None, [_VP, _VP, _VP, ctypes.c_int, ctypes.c_int, _VP]),
            "ko_table_cols": (ctypes.c_int, [_VP]),
            "ko_region_table": (None, [_VP, _VP]),
            "ko_region_r1": (ctypes.c_int, [_VP, _VP]),
            "ko_region_r2": (ctypes.c_int, [_VP, _VP, _VP, ctypes.c_int]),
            "ko_scores": (None, [_VP, _VP, _VP, _VP, _VP]),
            "ko_faccept": (_F32, [_VP, _U32, _U32]),
            "ko_frontier_compact": (None, [_VP, _VP, _U32, _U32, _VP, _VP]),
            "ko_plan": (ctypes.c_int, [_VP, _VP, _VP, _VP, _U32, _U32, _U32, ctypes.c_int, _VP]),
            "ko_sizes": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def _c(cfg) -> int:
    return ctypes.addressof(cfg)


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().ko_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def child_draws(seed: int, stream: int, it: int, n: int) -> np.ndarray:
    out = np.zeros((n, 6), np.float32)
    L = lib()
    for i in range(n):
        L.ko_child_draws(seed, stream, it, i, out[i].ctypes.data)
    return out


def sizes(cfg) -> tuple[int, int, int]:
    a, b, s = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    lib().ko_sizes(_c(cfg), ctypes.byref(a), ctypes.byref(b), ctypes.byref(s))
    return a.value, b.value, s.value


class OEnv:
    def __init__(self, cfg, obs: np.ndarray):
        self.obs = np.ascontiguousarray(obs, np.float32).reshape(-1, 6)
        self.h = lib().ko_env_create(_c(cfg), _p(self.obs), self.obs.shape[0])

    def grid(self):
        nc, ne = ctypes.c_uint32(), ctypes.c_uint32()
        lib().ko_env_grid(self.h, ctypes.byref(nc), ctypes.byref(ne), None, None)
        off = np.zeros(nc.value + 1, np.uint32)
        ent = np.zeros(max(ne.value, 1), np.uint32)
        lib().ko_env_grid(self.h, None, None, _p(off), _p(ent))
        return off, ent[: ne.value]

    def collide(self, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
        lo = np.ascontiguousarray(lo, np.float32).reshape(-1, 3)
        hi = np.ascontiguousarray(hi, np.float32).reshape(-1, 3)
        return np.array([lib().ko_collide_hash(self.h, _p(lo[i]), _p(hi[i])) for i in range(lo.shape[0])], np.uint8)

    def __del__(self):
        try:
            lib().ko_env_destroy(self.h)
        except Exception:
            pass


def collide_brute(obs: np.ndarray, lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    obs = np.ascontiguousarray(obs, np.float32).reshape(-1, 6)
    lo = np.ascontiguousarray(lo, np.float32).reshape(-1, 3)
    hi = np.ascontiguousarray(hi, np.float32).reshape(-1, 3)
    L = lib()
    return np.array([L.ko_collide_brute(_p(obs), obs.shape[0], _p(lo[i]), _p(hi[i])) for i in range(lo.shape[0])], np.uint8)


def propagate(cfg, obs: np.ndarray | None, parents: np.ndarray, draws: np.ndarray | None = None, stream: int = 0,
              nthreads: int = 1):
    """FP32 restatement over a batch; returns rows, valid, steps, margin, nonfinite, fail_kind."""
    parents = np.ascontiguousarray(parents, np.float32)
    n = parents.shape[0]
    S = cfg.state_dim + cfg.control_dim + 1
    rows = np.zeros((n, S), np.float32)
    valid = np.zeros(n, np.uint8)
    steps = np.zeros(n, np.int32)
    diag = (SegDiag * max(n, 1))()
    env = OEnv(cfg, obs if obs is not None else np.zeros((0, 6), np.float32))
    d = None if draws is None else np.ascontiguousarray(draws, np.float32).reshape(n, 6)
    lib().ko_propagate_batch(_c(cfg), env.h, _p(parents), _p(d), stream, n, _p(rows), _p(valid), _p(steps),
                             ctypes.addressof(diag), nthreads)
    margin = np.array([diag[i].margin for i in range(n)], np.float32)
    nonfinite = np.array([diag[i].nonfinite for i in range(n)], np.int32)
    kind = np.array([diag[i].fail_kind for i in range(n)], np.int32)
    return rows, valid, steps, margin, nonfinite, kind


def integrate_f64(cfg, x0: np.ndarray, ctrl_row: np.ndarray, steps: int, mode: int = 0) -> np.ndarray:
    x = np.ascontiguousarray(x0, np.float64)
    c = np.ascontiguousarray(ctrl_row, np.float32)
    out = np.zeros(cfg.state_dim, np.float64)
    lib().ko_integrate_f64(_c(cfg), _p(x), _p(c), int(steps), mode, _p(out))
    return out


def region_table(cfg) -> np.ndarray:
    n1, _, _ = sizes(cfg)
    cols = lib().ko_table_cols(_c(cfg))
    t = np.zeros((n1, cols), np.float32)
    lib().ko_region_table(_c(cfg), _p(t))
    return t


def frontier_compact(cfg, repeat: np.ndarray, budget: int):
    """Frontier compaction on its own: (repeat bytes after, entry node ids, {R, k, E, n})."""
    rep = np.ascontiguousarray(repeat, np.uint8).copy()
    entries = np.zeros(max(int(budget), 1), np.uint32)
    stats = np.zeros(4, np.uint32)
    lib().ko_frontier_compact(_c(cfg), _p(rep), rep.size, int(budget), _p(entries), _p(stats))
    R, k, E, n = (int(x) for x in stats)
    return rep, entries[:E].copy(), {"R": R, "k": k, "E": E, "n": n}


def regions(cfg, states: np.ndarray):
    states = np.ascontiguousarray(states, np.float32)
    t = region_table(cfg)
    L = lib()
    r1 = np.zeros(states.shape[0], np.int32)
    r2 = np.zeros(states.shape[0], np.int32)
    for i in range(states.shape[0]):
        a = L.ko_region_r1(_c(cfg), _p(states[i]))
        r1[i] = a
        r2[i] = L.ko_region_r2(_c(cfg), _p(t), _p(states[i]), a)
    return r1, r2


def scores(cfg, counter: np.ndarray, valid: np.ndarray, bits: np.ndarray) -> np.ndarray:
    n1, _, _ = sizes(cfg)
    out = np.zeros(n1, np.float32)
    lib().ko_scores(_c(cfg), _p(np.ascontiguousarray(counter, np.int32)), _p(np.ascontiguousarray(valid, np.int32)),
                    _p(np.ascontiguousarray(bits, np.uint32)), _p(out))
    return out


class PlanOut(ctypes.Structure):
    _fields_ = [("rows", _VP), ("parents", _VP), ("costs", _VP), ("r1", _VP), ("repeat", _VP), ("counter", _VP),
                ("valid", _VP), ("scores", _VP), ("r2_bits", _VP), ("path", _VP), ("iter_children", _VP),
                ("iter_appended", _VP)]


def plan(cfg, init, goal, obs, plan_idx: int = 0, max_iters: int | None = None, stop_at_goal: bool = True) -> dict:
    """Whole-plan restatement; returns the tree, region buffers and the result fields."""
    import kpax  # the Result struct layout is the ABI's

    class Out(ctypes.Structure):
        _fields_ = PlanOut._fields_ + [("result", kpax.Result)]

    n1, P, S = sizes(cfg)
    cap = cfg.max_tree_size
    iters = max_iters or cfg.max_iter
    words = (n1 * P + 31) // 32
    a = {
        "rows": np.zeros((cap, S), np.float32), "parents": np.zeros(cap, np.int32), "costs": np.zeros(cap, np.float32),
        "r1": np.zeros(cap, np.int32), "repeat": np.zeros(cap, np.uint8), "counter": np.zeros(n1, np.int32),
        "valid": np.zeros(n1, np.int32), "scores": np.zeros(n1, np.float32), "r2_bits": np.zeros(words, np.uint32),
        "path": np.zeros((cfg.max_iter + 2, S), np.float32), "iter_children": np.zeros(iters, np.uint32),
        "iter_appended": np.zeros(iters, np.uint32),
    }
    out = Out(**{k: v.ctypes.data for k, v in a.items()})
    i0 = np.zeros(S, np.float32)
    i0[: min(S, np.asarray(init).size)] = np.asarray(init, np.float32).ravel()[:S]
    g0 = np.zeros(S, np.float32)
    g0[: min(S, np.asarray(goal).size)] = np.asarray(goal, np.float32).ravel()[:S]
    obs = np.ascontiguousarray(obs, np.float32).reshape(-1, 6)
    lib().ko_plan(_c(cfg), _p(i0), _p(g0), _p(obs), obs.shape[0], plan_idx, iters, int(stop_at_goal), ctypes.byref(out))
    r = out.result
    t = r.tree_size
    res = {k: v[:t] for k, v in a.items() if k in ("rows", "parents", "costs", "r1", "repeat")}
    res.update({k: a[k] for k in ("counter", "valid", "scores", "r2_bits")})
    res["path"] = a["path"][: r.path_len]
    res["iter_children"] = a["iter_children"][: r.iters]
    res["iter_appended"] = a["iter_appended"][: r.iters]
    res.update({f: getattr(r, f) for f in ("found", "goal_idx", "path_len", "tree_size", "iters", "tree_full", "expansions",
                                            "valid_expansions", "path_cost")})
    return res


class RefLib:
    """The reference's own routines built for the host (one library per configuration)."""

    def __init__(self, model: int, name: str | None = None):
        """name: the configuration's library (default the model's benchmark configuration; "quad_ref"
        for the reference's own quadrotor block)."""
        self.name = name or REF_NAMES[model]
        path = ORACLE_DIR / "_ref" / f"libkref_{self.name}.so"
        if not path.exists():
            build()
        if not path.exists():
            raise FileNotFoundError(f"{path} (the reference tree is needed to build it)")
        L = ctypes.CDLL(str(path))
        for name, res, args in [
            ("kref_info", ctypes.c_int, [ctypes.c_int]),
            ("kref_set_obstacles", ctypes.c_int, [_VP, ctypes.c_int]),
            ("kref_cell_count", ctypes.c_int, [ctypes.c_int]),
            ("kref_propagate", None, [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, _VP, ctypes.c_int]),
            ("kref_region", None, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP]),
            ("kref_min_table", None, [_VP]),
            ("kref_collide", ctypes.c_int, [_VP, _VP, ctypes.c_int]),
            ("kref_expand", ctypes.c_longlong, [_VP, ctypes.c_int, _VP, ctypes.c_int, _VP, _VP, _VP, _VP, _VP, _VP,
                                                ctypes.c_int]),
            ("kref_max_threads", ctypes.c_int, []),
            ("kref_read_obstacles_csv", ctypes.c_int, [ctypes.c_char_p, _VP, ctypes.c_int, _VP]),
            ("kref_collide_batch", None, [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_int]),
        ]:
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        self.L = L
        info = [L.kref_info(i) for i in range(10)]
        (self.model, self.state_dim, self.control_dim, self.sample_dim, self.grid_size, self.slots, self.num_r1,
         self.r2_per_r1, self.max_duration, self.grid_dim) = info
        self.obs = np.zeros((0, 6), np.float32)

    def read_obstacles_csv(self, path, cap: int = 1 << 16):
        """readObstaclesFromCSV (helper.cu:13-39): every float read and numObstacles."""
        out = np.zeros(cap, np.float32)
        n_obs = ctypes.c_int(0)
        n = self.L.kref_read_obstacles_csv(str(path).encode(), _p(out), cap, ctypes.byref(n_obs))
        if n < 0:
            raise FileNotFoundError(path)
        return out[: min(n, cap)].copy(), n_obs.value

    def set_obstacles(self, obs: np.ndarray) -> int:
        self.obs = np.ascontiguousarray(obs, np.float32).reshape(-1, 6)
        return self.L.kref_set_obstacles(_p(self.obs), self.obs.shape[0])

    def propagate(self, parents: np.ndarray, draws: np.ndarray, use_hash: bool = True, nthreads: int = 1):
        parents = np.ascontiguousarray(parents, np.float32)
        draws = np.ascontiguousarray(draws, np.float32).reshape(-1, 6)
        n = parents.shape[0]
        rows = np.zeros((n, self.sample_dim), np.float32)
        valid = np.zeros(n, np.uint8)
        self.L.kref_propagate(_p(parents), _p(draws), n, int(use_hash), _p(rows), _p(valid), nthreads)
        return rows, valid

    def regions(self, states: np.ndarray):
        states = np.ascontiguousarray(states, np.float32)
        n = states.shape[0]
        r1 = np.zeros(n, np.int32)
        r2 = np.zeros(n, np.int32)
        self.L.kref_region(_p(states), states.shape[1], n, _p(r1), _p(r2))
        return r1, r2

    def min_table(self) -> np.ndarray:
        t = np.zeros((self.num_r1, self.state_dim), np.float32)
        self.L.kref_min_table(_p(t))
        return t

    def collide(self, lo, hi, use_hash: bool = False) -> np.ndarray:
        lo = np.ascontiguousarray(lo, np.float32).reshape(-1, 3)
        hi = np.ascontiguousarray(hi, np.float32).reshape(-1, 3)
        return np.array([self.L.kref_collide(_p(lo[i]), _p(hi[i]), int(use_hash)) for i in range(lo.shape[0])], np.uint8)

    def collide_batch(self, lo, hi, use_hash: bool = True, nthreads: int = 1) -> np.ndarray:
        """kref_collide over n boxes with OpenMP: 1 = free."""
        lo = np.ascontiguousarray(lo, np.float32).reshape(-1, 3)
        hi = np.ascontiguousarray(hi, np.float32).reshape(-1, 3)
        out = np.zeros(lo.shape[0], np.uint8)
        self.L.kref_collide_batch(_p(lo), _p(hi), lo.shape[0], int(use_hash), _p(out), nthreads)
        return out

    def expand(self, parents, per_parent, draws, scores, r2flags, counter, valid_counter, nthreads):
        parents = np.ascontiguousarray(parents, np.float32)
        draws = np.ascontiguousarray(draws, np.float32)
        n = draws.shape[0]
        fnext = np.zeros(n, np.uint8)
        rows = np.zeros((n, self.sample_dim), np.float32)
        nv = self.L.kref_expand(_p(parents), per_parent, _p(draws), n, _p(scores), _p(r2flags), _p(counter),
                                _p(valid_counter), _p(fnext), _p(rows), nthreads)
        return nv, fnext, rows


def rekino(cfg, init, goal, obs, num_warps: int, spt: int = 1, eps: float = 0.0, max_iter: int = 2000,
           plan_idx: int = 0) -> dict:
    """ReKinoLite restatement: the winner (warp, iteration) and its path (start first)."""
    n1, P, S = sizes(cfg)
    path = np.zeros((200, S), np.float32)
    ln, w, it = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    o = np.ascontiguousarray(obs, np.float32).reshape(-1, 6)
    i0 = np.zeros(S, np.float32)
    g0 = np.zeros(S, np.float32)
    a, b = np.asarray(init, np.float32).ravel(), np.asarray(goal, np.float32).ravel()
    i0[: min(S, a.size)] = a[:S]
    g0[: min(S, b.size)] = b[:S]
    L = lib()
    L.ko_rekino.restype = _I32
    L.ko_rekino.argtypes = [_VP, _VP, _VP, _VP, _U32, _U32, _U32, _F32, _U32, _U32, _VP, _VP, _VP, _VP]
    found = L.ko_rekino(_c(cfg), _p(i0), _p(g0), _p(o) if o.shape[0] else None, o.shape[0], num_warps, spt, eps, max_iter,
                        plan_idx, _p(path), ctypes.byref(ln), ctypes.byref(w), ctypes.byref(it))
    return {"found": int(found), "warp": w.value, "iter": it.value, "path": path[: ln.value + 1].copy() if found else
            np.zeros((0, S), np.float32)}

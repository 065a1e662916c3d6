"""Seeded synthetic environments, start states and the obstacle CSV format.

Obstacles are rows [min x, min y, min z, max x, max y, max z] (float32), the layout the
reference reads from include/config/obstacles/*/obstacles.csv (src/helper/helper.cu:13-39).
All generators use numpy's PCG64 with an explicit seed, so every run sees the same scene.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

W_MIN, W_MAX = 0.0, 100.0


_WS = " \t\n\v\f\r"
_DIGITS = "0123456789"
_strtof = None


def _to_float32(token: str):
    """The float a C++ stream extracts from a complete numeric token (strtof in the "C" locale),
    or None where the extraction fails (|value| beyond the float range)."""
    global _strtof
    if _strtof is None:
        import ctypes

        libc = ctypes.CDLL(None)
        _strtof = libc.strtof
        _strtof.restype, _strtof.argtypes = ctypes.c_float, [ctypes.c_char_p, ctypes.c_void_p]
    v = np.float32(_strtof(token.encode(), None))
    return None if np.isinf(v) else v


def _line_floats(line: str) -> list:
    """Floats of one line as readObstaclesFromCSV takes them (helper.cu:13-39): `ss >> value` after
    skipping white space accepts [sign] digits [. digits] [e|E [sign] digits] (at least one mantissa
    digit; an exponent only after one, and then with at least one digit), and one comma right
    after a value is skipped.  The first token that does not extract ends the line."""
    out, i, n = [], 0, len(line)
    while True:
        while i < n and line[i] in _WS:
            i += 1
        j = i
        if j < n and line[j] in "+-":
            j += 1
        d0 = j
        while j < n and line[j] in _DIGITS:
            j += 1
        digits = j > d0
        if j < n and line[j] == ".":
            j += 1
            f0 = j
            while j < n and line[j] in _DIGITS:
                j += 1
            digits = digits or j > f0
        if not digits:
            return out
        if j < n and line[j] in "eE":
            k = j + 1
            if k < n and line[k] in "+-":
                k += 1
            e0 = k
            while k < n and line[k] in _DIGITS:
                k += 1
            if k == e0:  # "1e" or "1e+": the collected token does not convert
                return out
            j = k
        v = _to_float32(line[i:j])
        if v is None:
            return out
        out.append(v)
        i = j + 1 if j < n and line[j] == "," else j


def read_csv_floats(path: str | Path) -> np.ndarray:
    """Every float of an obstacle file, read line by line as readObstaclesFromCSV (helper.cu:13-39)
    reads it (the same rule as kpax_read_obstacles_csv in the C ABI)."""
    vals: list = []
    text = Path(path).read_bytes().decode("latin-1")  # bytes as they are; lines end at "\n" only, as std::getline's
    for line in text.split("\n"):
        vals.extend(_line_floats(line))
    return np.asarray(vals, np.float32)


def read_obstacles_csv(path: str | Path) -> np.ndarray:
    """Obstacles of a CSV file, 6 floats each (readObstaclesFromCSV, helper.cu:13-39): the first
    n // 6 rows of its floats; a trailing partial row is not an obstacle."""
    vals = read_csv_floats(path)
    n = vals.size // 6
    return vals[: 6 * n].reshape(n, 6)


def write_obstacles_csv(path: str | Path, obs: np.ndarray) -> None:
    with open(path, "w") as f:
        for row in np.asarray(obs, np.float32).reshape(-1, 6):
            f.write(",".join(f"{v:.6f}" for v in row) + "\n")


def _covers(box: np.ndarray, p: np.ndarray) -> bool:
    p = np.asarray(p, np.float32)[:3]
    return bool(np.all(box[:3] <= p) and np.all(p <= box[3:]))


def random_boxes(n: int, seed: int, side=(5.0, 15.0), avoid=(), rng: np.random.Generator | None = None) -> np.ndarray:
    """n axis-aligned boxes: centres U[0,100]^3, sides U[side]; boxes covering a point of
    `avoid` are redrawn."""
    rng = rng or np.random.default_rng(seed)
    avoid = [np.asarray(a, np.float32)[:3] for a in avoid]
    out = []
    while len(out) < n:
        c = rng.uniform(W_MIN, W_MAX, 3)
        s = rng.uniform(side[0], side[1], 3)
        b = np.concatenate([c - s / 2, c + s / 2]).astype(np.float32)
        if any(_covers(b, a) for a in avoid):
            continue
        out.append(b)
    return np.asarray(out, np.float32).reshape(-1, 6)


def di_scene(seed: int = 0):
    """Double-integrator benchmark: 20 boxes (sides U[5,15]) avoiding start (5,5,5) and the goal
    centre (95,95,95); goal ball radius 5."""
    start = np.array([5, 5, 5, 0, 0, 0], np.float32)
    goal = np.array([95, 95, 95, 0, 0, 0], np.float32)
    return random_boxes(20, seed, avoid=(start, goal)), start, goal


def forest(n: int = 200, seed: int = 1) -> np.ndarray:
    """Vertical columns from z = 0: xy footprint sides U[2,6], height U[20,100], centres U[0,100]^2."""
    rng = np.random.default_rng(seed)
    xy = rng.uniform(W_MIN, W_MAX, (n, 2))
    fp = rng.uniform(2.0, 6.0, (n, 2))
    h = rng.uniform(20.0, 100.0, n)
    lo = np.column_stack([xy - fp / 2, np.zeros(n)])
    hi = np.column_stack([xy + fp / 2, h])
    return np.concatenate([lo, hi], axis=1).astype(np.float32)


def dubins_scene(seed: int = 1):
    start = np.array([5, 5, 50, 0.7853982, 0, 1.0], np.float32)
    goal = np.array([95, 95, 50, 0, 0, 0], np.float32)
    obs = forest(200, seed)
    keep = [b for b in obs if not (_covers(b, start) or _covers(b, goal))]
    return np.asarray(keep, np.float32).reshape(-1, 6), start, goal


WALL_X, WALL_T, WINDOW = 50.0, 1.0, 6.0
WINDOW_CENTRES = ((25.0, 25.0), (75.0, 25.0), (25.0, 75.0), (75.0, 75.0))


def wall_with_windows() -> np.ndarray:
    """A 1 m thick wall at x = 50 spanning y, z in [0,100] with four 6x6 windows, as boxes."""
    x0, x1 = WALL_X - WALL_T / 2, WALL_X + WALL_T / 2
    zs = sorted({0.0, 100.0, *(c[1] - WINDOW / 2 for c in WINDOW_CENTRES), *(c[1] + WINDOW / 2 for c in WINDOW_CENTRES)})
    ys = sorted({0.0, 100.0, *(c[0] - WINDOW / 2 for c in WINDOW_CENTRES), *(c[0] + WINDOW / 2 for c in WINDOW_CENTRES)})
    boxes = []
    for za, zb in zip(zs[:-1], zs[1:]):
        zm = (za + zb) / 2
        in_band = any(abs(zm - c[1]) < WINDOW / 2 for c in WINDOW_CENTRES)
        if not in_band:
            boxes.append([x0, 0.0, za, x1, 100.0, zb])
            continue
        for ya, yb in zip(ys[:-1], ys[1:]):
            ym = (ya + yb) / 2
            if any(abs(ym - c[0]) < WINDOW / 2 and abs(zm - c[1]) < WINDOW / 2 for c in WINDOW_CENTRES):
                continue
            boxes.append([x0, ya, za, x1, yb, zb])
    return np.asarray(boxes, np.float32)


def building(n_total: int = 1000, seed: int = 2, start=(10.0, 8.0, 5.0), goal=(80.0, 95.0, 90.0)) -> np.ndarray:
    """`n_total` boxes: the windowed wall plus random boxes (sides U[5,15]) that leave the start,
    the goal and the window openings (extended 4 m either side of the wall) free."""
    wall = wall_with_windows()
    rng = np.random.default_rng(seed)
    tunnels = [np.array([WALL_X - 4, cy - WINDOW / 2, cz - WINDOW / 2, WALL_X + 4, cy + WINDOW / 2, cz + WINDOW / 2])
               for cy, cz in WINDOW_CENTRES]
    out = []
    p_s, p_g = np.asarray(start, np.float32), np.asarray(goal, np.float32)
    while len(out) < n_total - len(wall):
        b = random_boxes(1, 0, rng=rng)[0]
        if _covers(b, p_s) or _covers(b, p_g):
            continue
        if any(np.all(b[:3] < t[3:]) and np.all(t[:3] < b[3:]) for t in tunnels):
            continue
        out.append(b)
    return np.concatenate([wall, np.asarray(out, np.float32)]).astype(np.float32)


def quad_scene(seed: int = 2, n_total: int = 1000):
    start = np.array([10, 8, 5] + [0] * 9, np.float32)
    goal = np.array([80, 95, 90] + [0] * 9, np.float32)
    return building(n_total, seed, start[:3], goal[:3]), start, goal


def sample_states(model: int, n: int, seed: int, vmin: float = -1.0, vmax: float = 1.0) -> np.ndarray:
    """Parent states uniform within the model's bounds (positions in [0,100]^3)."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(W_MIN, W_MAX, (n, 3))
    if model == 1:
        vel = rng.uniform(vmin, vmax, (n, 3))
        return np.column_stack([pos, vel]).astype(np.float32)
    if model == 2:
        yaw = rng.uniform(-math.pi, math.pi, n)
        pitch = rng.uniform(-math.pi / 3, math.pi / 3, n)
        v = rng.uniform(max(vmin, 0.5), vmax, n)
        return np.column_stack([pos, yaw, pitch, v]).astype(np.float32)
    ang = rng.uniform(-0.5, 0.5, (n, 3))
    vel = rng.uniform(-5.0, 5.0, (n, 3))
    rates = rng.uniform(-0.5, 0.5, (n, 3))
    return np.column_stack([pos, ang, vel, rates]).astype(np.float32)


def uniform_draws(n: int, seed: int) -> np.ndarray:
    """n x 6 uniforms in (0, 1] on the 2^-24 grid the device generator uses."""
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 1 << 24, (n, 6), endpoint=True)
    return (k.astype(np.float64) * 2.0 ** -24).astype(np.float32)


def boxes_avoiding(rng: np.random.Generator, n: int, points, side=(5.0, 15.0)) -> np.ndarray:
    """n boxes (centres U[0,100]^3, sides U[side]) none of which covers one of `points`."""
    pts = np.asarray([np.asarray(p, np.float32)[:3] for p in points], np.float32).reshape(-1, 3)
    out = np.zeros((0, 6), np.float32)
    while out.shape[0] < n:
        m = int((n - out.shape[0]) * 1.5) + 8
        c = rng.uniform(W_MIN, W_MAX, (m, 3))
        s = rng.uniform(side[0], side[1], (m, 3))
        b = np.concatenate([c - s / 2, c + s / 2], axis=1).astype(np.float32)
        cover = np.zeros(m, bool)
        for p in pts:
            cover |= np.all(b[:, :3] <= p, axis=1) & np.all(p <= b[:, 3:], axis=1)
        out = np.concatenate([out, b[~cover]])
    return out[:n]


def batch_queries(n: int = 1024, seed: int = 4, mix=(0.4, 0.3, 0.3), obs_range=(10, 5000), tree_range=(1 << 14, 1 << 20),
                  min_sep: float = 50.0):
    """The batched benchmark: n queries, mixing double integrator / Dubins / quadrotor in `mix`
    proportions; obstacle counts and tree budgets log-uniform in their ranges; start and goal
    uniform in the workspace at least `min_sep` apart, with no box covering either.
    Returns a list of dicts: model, n_obs, tree, obstacles, start, goal."""
    rng = np.random.default_rng(seed)
    counts = [int(round(n * f)) for f in mix]
    counts[0] += n - sum(counts)
    models = np.concatenate([np.full(c, m + 1) for m, c in enumerate(counts)])
    rng.shuffle(models)
    out = []
    for q in range(n):
        model = int(models[q])
        n_obs = int(round(math.exp(rng.uniform(math.log(obs_range[0]), math.log(obs_range[1])))))
        tree = int(round(2.0 ** rng.uniform(math.log2(tree_range[0]), math.log2(tree_range[1]))))
        while True:
            a, b = rng.uniform(W_MIN, W_MAX, 3), rng.uniform(W_MIN, W_MAX, 3)
            if np.linalg.norm(a - b) >= min_sep:
                break
        sd = 12 if model == 3 else 6
        start, goal = np.zeros(sd, np.float32), np.zeros(sd, np.float32)
        start[:3], goal[:3] = a, b
        if model == 2:
            start[3] = rng.uniform(-math.pi, math.pi)
            start[5] = 1.0
        out.append({"model": model, "n_obs": n_obs, "tree": tree, "start": start, "goal": goal,
                    "obstacles": boxes_avoiding(rng, n_obs, (a, b))})
    return out


def free_queries(obs: np.ndarray, n: int, seed: int, min_sep: float = 6.0, max_sep: float = 15.0, margin: float = 1.0,
                 lo: float = 5.0, hi: float = 95.0) -> np.ndarray:
    """n start/goal pairs (rows: start xyz, goal xyz) in the free space of a fixed scene: points
    uniform in [lo, hi]^3 at least `margin` from every box, start and goal min_sep..max_sep apart."""
    rng = np.random.default_rng(seed)
    b = np.asarray(obs, np.float32).reshape(-1, 6)
    lo_b, hi_b = b[:, :3] - margin, b[:, 3:] + margin

    def free(p):
        return not np.any(np.all(lo_b <= p, axis=1) & np.all(p <= hi_b, axis=1))

    out = []
    while len(out) < n:
        a = rng.uniform(lo, hi, 3)
        if not free(a):
            continue
        d = rng.normal(0.0, 1.0, 3)
        g = a + d / np.linalg.norm(d) * rng.uniform(min_sep, max_sep)
        if np.any(g < lo) or np.any(g > hi) or not free(g):
            continue
        out.append(np.concatenate([a, g]))
    return np.asarray(out, np.float32)


def learned_family(seed: int, obs_range=(200, 2000), min_sep: float = 25.0, max_sep: float = 45.0, fixed: bool = False):
    """The learned-proposal family of the 12D quadrotor: a 'building' scene (windowed wall at
    x = 50 plus random boxes) with a seeded obstacle count uniform in obs_range.  Start and goal
    are uniform in [5, 95]^3, min_sep..max_sep apart (within the reach of a 2^20-node plain tree
    under the +-0.1 torque limits) and off the wall, or with `fixed` the benchmark pair
    (10, 8, 5) -> (80, 95, 90).  Returns (obstacles, start, goal)."""
    rng = np.random.default_rng(seed)
    n_total = int(rng.integers(obs_range[0], obs_range[1], endpoint=True))
    if fixed:
        return quad_scene(seed=seed, n_total=n_total)
    while True:
        a, b = rng.uniform(5.0, 95.0, 3), rng.uniform(5.0, 95.0, 3)
        off_wall = abs(a[0] - WALL_X) > 2.0 and abs(b[0] - WALL_X) > 2.0
        if off_wall and min_sep <= np.linalg.norm(a - b) <= max_sep:
            break
    start, goal = np.zeros(12, np.float32), np.zeros(12, np.float32)
    start[:3], goal[:3] = a, b
    return building(n_total, seed, start[:3], goal[:3]), start, goal

"""The oracle's frontier compaction (ko_frontier_compact, shared with its whole-plan loop) against a
direct restatement of the entry rule: R entries from the repeat counts, k children per entry
(CHILDREN_PER_ENTRY, or max(1, B // R) when R k > B), E = min(R, B // k) entries taken, entry j
being virtual entry floor(j R / E) in node order, taken nodes leaving the frontier."""
import numpy as np
import pytest

import kpax
import oracle as O


def restated(cfg, rep, budget):
    rep = rep.astype(np.int64)
    pending = rep == 255
    rep[pending] = cfg.sparse_repeat if cfg.sparse_valid_threshold > 0 else 1
    R = int(rep.sum())
    k, E = cfg.children_per_entry, 0
    if budget and R:
        if R * k > budget:
            k = max(1, budget // R)
        E = min(R, budget // k)
    owner = np.repeat(np.arange(rep.size), rep)  # virtual entry -> node
    entries = owner[(np.arange(E) * R) // E] if E else np.zeros(0, np.int64)
    out = rep.copy()
    out[np.unique(entries)] = 0
    return out.astype(np.uint8), entries.astype(np.uint32), {"R": R, "k": k, "E": E, "n": E * k}


@pytest.mark.parametrize("seed", range(6))
def test_oracle_compaction_matches_the_entry_rule(seed):
    rng = np.random.default_rng(seed)
    cfg = kpax.preset(kpax.PRESET_QUAD)
    n = int(rng.integers(0, 3000))
    rep = np.where(rng.random(n) < 0.3, rng.integers(1, 16, n), 0).astype(np.uint8)
    rep[rng.random(n) < 0.05] = 255
    R = int(np.where(rep == 255, cfg.sparse_repeat, rep).sum())
    for budget in (0, 1, 7, max(R - 1, 1), R, R * cfg.children_per_entry, 1 << 16, int(rng.integers(1, 5000))):
        got = O.frontier_compact(cfg, rep, budget)
        want = restated(cfg, rep, budget)
        assert got[2] == want[2], (budget, got[2], want[2])
        assert np.array_equal(got[1], want[1]) and np.array_equal(got[0], want[0]), budget

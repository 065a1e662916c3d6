"""Host side of the harness of the reference's own CUDA build (oracle/refcuda/ref_plan.cu), which
needs no GPU: its hash-grid guard refuses a scene in which the reference's cell query would read
past the end of its 16-slot-per-cell array (spatialHash.cu:166-173) before any device work, and
the Python driver turns every failure into an `unavailable` record instead of raising."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle" / "refcuda"))
import refcuda  # noqa: E402

pytestmark = pytest.mark.skipif(not refcuda.binary("quad_c2").exists(), reason="reference CUDA build not compiled")


def test_scene_that_overruns_the_slot_array_is_refused():
    # 20 boxes in the corner cell (the last of the 21^3 cells): its count runs 4 slots past the
    # end of the array, which the reference's query would read
    corner = np.tile(np.array([[99.0, 99.0, 99.0, 100.0, 100.0, 100.0]], np.float32), (20, 1))
    res = refcuda.run("quad_c2", corner, [[10, 8, 5, 80, 95, 90]], iteration_cap=5, timeout_s=60)
    assert "unavailable" in res and "slot array" in res["unavailable"]


def test_overflow_inside_the_array_is_accepted_by_the_guard():
    # 20 boxes in the first cell overrun its 16 slots into the next cell's, inside the array: the
    # guard passes it on (without a GPU the run then stops at the first CUDA call)
    first = np.tile(np.array([[0.0, 0.0, 0.0, 1.0, 1.0, 1.0]], np.float32), (20, 1))
    res = refcuda.run("quad_c2", first, [[10, 8, 5, 80, 95, 90]], iteration_cap=5, timeout_s=60)
    if "unavailable" in res:  # no device here
        assert "slot array" not in res["unavailable"]
    else:
        assert res["config"]["grid_cells_over_16"] == 1 and res["config"]["grid_max_count"] == 20


def test_summary_of_an_unavailable_run_passes_it_through():
    assert refcuda.summarise({"unavailable": "why"}) == {"unavailable": "why"}
    res = refcuda.run("no_such_cfg", np.zeros((0, 6), np.float32), [[0, 0, 0, 1, 1, 1]], 1)
    assert "unavailable" in res and "not built" in res["unavailable"]

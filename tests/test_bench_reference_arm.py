"""bench.py's reference arm on the host: the reference's own propagation + collision routines
(oracle/_ref) timed on a bounded sample, printed as one JSON line of the benchmark contract; the
workloads with no reference counterpart print an `unavailable` line."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def run(*args):
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args], cwd=ROOT,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libkref_dubins.so").exists(), reason="reference routines not built")
def test_segments_reference_line():
    d = run("--workload", "segments", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference" and d["metric"] == "valid expansions/s" and d["unit"] == "expansions/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    cpu = d["cpu_baseline"]
    assert cpu["kind"] == "reference" and cpu["cores"] >= 1 and cpu["value"] == d["value"] and cpu["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libkref_quad.so").exists(), reason="reference routines not built")
def test_collide_reference_line():
    d = run("--workload", "collide", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference" and d["metric"] == "swept-box queries/s" and d["unit"] == "queries/s"
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("workload", ["learned", "batch"])
def test_no_counterpart_lines(workload):
    d = run("--workload", workload)
    assert d["impl"] == "reference" and d["unavailable"]


@pytest.mark.skipif(not (ROOT / "oracle" / "_ref" / "libkref_quad_ref.so").exists(), reason="reference routines not built")
def test_quad_ref_reference_line():
    """The reference's own quadrotor block (h 0.1 s, up to 10 steps, torques in [-pi, pi]) on its
    quadTrees scene: the host-compiled reference body of that block."""
    d = run("--workload", "quad-ref", "--steps", "1", "--warmup", "1")
    assert d["impl"] == "reference" and d["metric"] == "valid expansions/s" and d["value"] > 0
    assert "quadTrees" in d["config"]["workload"] and d["config"]["expansions_per_iter"] > 0

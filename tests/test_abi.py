"""The C ABI library loads without a GPU, exports every symbol include/kpax.h declares, and its
pure-host calls (presets, validation, sizes) behave as documented.  No device calls here."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import kpax
import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    text = (ROOT / "include" / "kpax.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(kpax_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol():
    lib = kpax.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding types every declared entry point
    assert names <= set(kpax.exported_symbols())


def test_abi_version():
    assert kpax.load().kpax_abi_version() == kpax.ABI_VERSION == 3


@pytest.mark.parametrize("which", [kpax.PRESET_DI, kpax.PRESET_DUBINS, kpax.PRESET_QUAD, kpax.PRESET_QUAD_REF])
def test_presets_validate_and_size(which):
    cfg = kpax.preset(which)
    assert kpax.load().kpax_config_validate(ctypes.byref(cfg)) == kpax.OK
    n1, P, S = kpax.sizes(cfg)
    assert (n1, P, S) == O.sizes(cfg)
    assert S == cfg.state_dim + cfg.control_dim + 1


def test_preset_values_follow_benchmark_configs():
    di = kpax.preset(kpax.PRESET_DI)
    assert (di.step_size, di.max_propagation_duration, di.fixed_steps) == (np.float32(0.1), 10, 0)
    assert kpax.sizes(di)[:2] == (512, 8)
    assert di.expansions_per_iter == 1 << 14 and di.max_tree_size == 1 << 20
    q = kpax.preset(kpax.PRESET_QUAD)
    assert (q.step_size, q.max_propagation_duration, q.fixed_steps) == (np.float32(0.02), 25, 1)
    assert q.ctrl_max[0] == np.float32(19.62) and q.ctrl_min[1] == np.float32(-0.1)
    assert kpax.sizes(q)[:2] == (32768, 64)
    assert q.expansions_per_iter == 1 << 16
    d = kpax.preset(kpax.PRESET_DUBINS)
    assert (d.v_min, d.v_max) == (0.5, 2.0) and d.max_propagation_duration == 20


@pytest.mark.parametrize(
    "field,value",
    [("model", 7), ("state_dim", 5), ("max_tree_size", 1), ("step_size", 0.0), ("w_max", -1.0), ("c_r1_length", 40),
     ("hash_cell_size", 0.0), ("children_per_entry", 0), ("expansions_per_iter", 0), ("c_dim", 9), ("block_size", 33),
     ("block_size", 384), ("samples_per_thread", 9), ("samples_per_thread", -1), ("iteration_kernels", 2),
     ("iteration_kernels", -1)],
)
def test_invalid_configs_are_rejected_with_a_message(field, value):
    cfg = kpax.preset(kpax.PRESET_QUAD)
    setattr(cfg, field, value)
    lib = kpax.load()
    assert lib.kpax_config_validate(ctypes.byref(cfg)) == kpax.EINVAL
    assert lib.kpax_last_error()
    with pytest.raises(kpax.KpaxError):
        kpax.sizes(cfg)


def test_unknown_preset():
    with pytest.raises(kpax.KpaxError):
        kpax.preset(99)


def test_cpp_wrapper_header_compiles():
    """include/kpax.hpp (the C++ mirror of the reference KPAX class) compiles against the ABI."""
    import shutil
    import subprocess
    import tempfile

    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    src = '#include "kpax.hpp"\nint main(){ kpax_config c; return kpax_config_preset(KPAX_PRESET_QUAD, &c) == KPAX_OK ? 0 : 1; }\n'
    with tempfile.TemporaryDirectory() as d:
        p = Path(d) / "t.cpp"
        p.write_text(src)
        r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", f"-I{ROOT / 'include'}", str(p)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def test_cpp_driver_reads_obstacle_files(tmp_path):
    """A reference-style driver built against kpax.hpp and libkpax.so reads an obstacle file with
    readObstaclesFromCSV(filename, numObstacles, workspaceDim), as examples/gpu/main.cu does."""
    import shutil
    import subprocess

    gxx = next((g for g in ("/usr/bin/g++", shutil.which("g++")) if g and Path(g).exists()), None)
    lib = ROOT / "kino-pax-fork_b200" / "libkpax.so"
    if not gxx or not lib.exists():
        pytest.skip("no g++ or libkpax.so")
    (tmp_path / "obstacles.csv").write_text("x0,y0,z0,x1,y1,z1\n1,2,3,4,5,6\n7.5, 8, 9,10,11,12\n13,14\n")
    src = """#include "kpax.hpp"
#include <cstdio>
int main(int argc, char** argv)
{
    int numObstacles = 0;
    std::vector<float> obstacles = readObstaclesFromCSV(argv[1], numObstacles, 3);
    std::printf("%d %zu", numObstacles, obstacles.size());
    for(float v : obstacles) std::printf(" %g", v);
    try {
        readObstaclesFromCSV(std::string(argv[1]) + ".absent", numObstacles, 3);
    } catch(const std::runtime_error&) {
        std::printf(" missing-file-throws");
    }
    return 0;
}
"""
    (tmp_path / "driver.cpp").write_text(src)
    exe = tmp_path / "driver"
    r = subprocess.run([gxx, "-std=c++17", f"-I{ROOT / 'include'}", str(tmp_path / "driver.cpp"), "-o", str(exe),
                        f"-L{lib.parent}", "-lkpax", f"-Wl,-rpath,{lib.parent}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe), str(tmp_path / "obstacles.csv")], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    # the header line reads nothing; white space before a value is skipped ("7.5, 8, 9"); the
    # partial row's floats are read but are not an obstacle
    assert out.stdout == "2 14 1 2 3 4 5 6 7.5 8 9 10 11 12 13 14 missing-file-throws", out.stdout


def test_pruning_parameters_are_validated():
    """PruneKPAX's goal-progress pruning needs a positive progress scale and finite biases."""
    cfg = kpax.preset(kpax.PRESET_DI)
    assert (cfg.prune, cfg.prune_goal_bias, cfg.prune_exploration_bias, cfg.prune_progress_scale) == (
        0, np.float32(0.7), np.float32(0.3), 10.0)
    lib = kpax.load()
    cfg.prune = 1
    assert lib.kpax_config_validate(ctypes.byref(cfg)) == kpax.OK
    cfg.prune_progress_scale = 0.0
    assert lib.kpax_config_validate(ctypes.byref(cfg)) == kpax.EINVAL
    cfg.prune = 0
    assert lib.kpax_config_validate(ctypes.byref(cfg)) == kpax.OK


def test_null_arguments_are_rejected_without_a_gpu():
    """Every creation and plan call checks its pointers before touching the device."""
    lib = kpax.load()
    out = ctypes.c_void_p()
    cfg = kpax.preset(kpax.PRESET_DI)
    assert lib.kpax_create(None, ctypes.byref(out)) == kpax.EINVAL
    assert lib.kpax_create(ctypes.byref(cfg), None) == kpax.EINVAL
    assert lib.kpax_env_create(None, None, 0, None, ctypes.byref(out)) == kpax.EINVAL
    assert lib.kpax_batch_create(ctypes.byref(cfg), 0, ctypes.byref(out)) == kpax.EINVAL
    assert lib.kpax_plan(None, None, None, None, 0, 0, None) == kpax.EINVAL
    assert lib.kpax_plan_bench(None, None, None, None, 0, 0, None, None) == kpax.EINVAL
    assert lib.kpax_export_tree(None, None, None, None, 0, None) == kpax.EINVAL
    st = kpax.FrontierStats()
    assert lib.kpax_frontier_compact(None, None, 0, 0, None, ctypes.byref(st), None) == kpax.EINVAL
    assert lib.kpax_frontier_compact(ctypes.byref(cfg), None, 10, 0, None, ctypes.byref(st), None) == kpax.EINVAL
    assert lib.kpax_frontier_compact(ctypes.byref(cfg), 16, 10, 5, None, ctypes.byref(st), None) == kpax.EINVAL
    assert lib.kpax_frontier_compact(ctypes.byref(cfg), 16, (1 << 24) + 1, 0, None, ctypes.byref(st), None) == kpax.EINVAL
    assert b"2^24" in lib.kpax_last_error()
    status = ctypes.c_uint32(0)
    assert lib.kpax_test_wait_timeout(0, ctypes.byref(status), None) == kpax.EINVAL
    assert lib.kpax_test_wait_timeout(16, None, None) == kpax.EINVAL
    assert lib.kpax_test_wait_timeout((1 << 22) + 1, ctypes.byref(status), None) == kpax.EINVAL
    assert lib.kpax_last_error()


def test_fp32_peak_checks_its_arguments_without_a_gpu():
    lib = kpax.load()
    t, ms = ctypes.c_double(), ctypes.c_double()
    assert lib.kpax_fp32_peak(8, ctypes.byref(t), ctypes.byref(ms), None) == kpax.EINVAL  # fewer than 16 FMAs
    assert lib.kpax_fp32_peak(1 << 16, None, None, None) == kpax.EINVAL
    assert b"iters" in lib.kpax_last_error()


def test_config_default_runs_the_fused_iteration():
    """iteration_kernels = 0 (a single persistent launch per iteration) is every preset's default."""
    for which in (kpax.PRESET_DI, kpax.PRESET_DUBINS, kpax.PRESET_QUAD, kpax.PRESET_QUAD_REF):
        assert kpax.preset(which).iteration_kernels == 0

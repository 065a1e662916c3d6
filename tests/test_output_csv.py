"""Solution output in the reference's CSV format (writeVectorToCSV, helper.cuh:56-80): each value
printed with std::fixed and 6 digits, comma-separated, one row per line, append mode appends."""
import numpy as np

import kpax


def reference_format(rows):
    return "".join(",".join(f"{float(v):.6f}" for v in r) + "\n" for r in np.asarray(rows, np.float32))


def test_rows_csv_format_and_append(tmp_path):
    rng = np.random.default_rng(0)
    rows = (rng.normal(0, 50, (7, 17)) * rng.choice([1e-6, 1.0, 1e3], (7, 17))).astype(np.float32)
    rows[0, 0], rows[0, 1], rows[1, 0] = -0.0, 1e-7, 3.0000004
    f = tmp_path / "controlPathToGoal.csv"
    kpax.write_rows_csv(rows, f)
    assert f.read_text() == reference_format(rows)
    kpax.write_rows_csv(rows[:2], f, append=True)
    assert f.read_text() == reference_format(rows) + reference_format(rows[:2])
    back = np.loadtxt(f, delimiter=",", dtype=np.float64)
    assert back.shape == (9, 17) and np.allclose(back[:7], rows, atol=5.1e-7, rtol=0)


def test_rows_csv_rejects_bad_arguments(tmp_path):
    import pytest

    with pytest.raises(kpax.KpaxError):
        kpax.write_rows_csv(np.zeros((2, 3), np.float32), tmp_path / "no_such_dir" / "x.csv")

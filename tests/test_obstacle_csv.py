"""The obstacle CSV reader (readObstaclesFromCSV, helper.cu:13-39) on well-formed and malformed files:
the C ABI (kpax_read_obstacles_csv), the Python restatement (kpax_envs) and the reference's own
function compiled for the host read the same floats, bit for bit, and the same obstacle count."""
import numpy as np
import pytest

import kpax
import kpax_envs as E
import oracle as O

CASES = {
    "plain": "1,2,3,4,5,6\n7,8,9,10,11,12\n",
    "no final newline": "1,2,3,4,5,6",
    "crlf": "1,2,3,4,5,6\r\n7,8,9,10,11,12\r\n",
    "header line": "minx,miny,minz,maxx,maxy,maxz\n1,2,3,4,5,6\n",
    "empty field": "1,,2,3,4,5,6,7\n8,9,10,11,12,13\n",
    "spaces": "1 2 3 4 5 6\n1, 2, 3, 4, 5, 6\n",
    "space before comma": "1 ,2,3,4,5,6\n7,8,9,10,11,12\n",
    "trailing comma and partial row": "1,2,3,4,5,6,\n7,8,9\n",
    "tabs and blank lines": "\n\t1\t2,3,4,5,6\n\n\n7,8,9,10,11,12",
    "exponents and signs": "+1e1,-2.5E-1,.5,5.,-0,1e-50\n00012,-.25,3.e2,1E+05,0.1,6\n",
    "bad exponent and junk": "1e,2,3\n4,5x,6\n7,8,9,10,11,12\n",
    "inf and nan tokens": "inf,1,2\nnan\n3,4,5,6,7,8\n",
    "overflow": "1e40,1,2\n-1e39\n3.4028235e38,1,2,3,4,5\n",
    "two points": "1.2.3,4,5,6,7\n",
    "hex and semicolons": "0x10,1\n1;2;3\n9,8,7,6,5,4\n",
    "benchmark values": "50.7722,37.8436,0.0,53.37019999999999,39.3436,20.0\n0.1,0.2,0.3,99.99999,1e-7,7.0000001\n",
    "empty file": "",
}


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def ref():
    try:
        return O.RefLib(kpax.MODEL_QUADROTOR)
    except (FileNotFoundError, OSError) as exc:
        pytest.skip(f"the host build of the reference is not available: {exc}")


@pytest.mark.parametrize("case", list(CASES))
def test_reader_matches_reference(tmp_path, ref, case):
    path = tmp_path / "obstacles.csv"
    path.write_bytes(CASES[case].encode())
    want, n_obs = ref.read_obstacles_csv(path)
    got_abi = kpax.read_csv_floats(path)
    got_py = E.read_csv_floats(path)
    assert np.array_equal(bits(got_abi), bits(want)), (got_abi, want)
    assert np.array_equal(bits(got_py), bits(want)), (got_py, want)
    for obs in (kpax.read_obstacles_csv(path), E.read_obstacles_csv(path)):
        assert obs.shape == (n_obs, 6) and np.array_equal(bits(obs.ravel()), bits(want[: 6 * n_obs]))


def test_reader_round_trips_written_files(tmp_path):
    """Obstacles written in the reference's six-decimal format read back within the format's rounding."""
    obs = E.quad_scene()[0]
    E.write_obstacles_csv(tmp_path / "w.csv", obs)
    back = kpax.read_obstacles_csv(tmp_path / "w.csv")
    assert back.shape == obs.shape and np.allclose(back, obs, atol=5e-7 * 100, rtol=0)
    assert np.array_equal(bits(back), bits(E.read_obstacles_csv(tmp_path / "w.csv")))


def test_missing_file_is_an_error(tmp_path):
    """The reference exits the process; the C ABI returns KPAX_EINVAL and Python raises."""
    with pytest.raises(kpax.KpaxError) as e:
        kpax.read_csv_floats(tmp_path / "absent.csv")
    assert e.value.status == kpax.EINVAL and "absent.csv" in str(e.value)
    with pytest.raises(FileNotFoundError):
        E.read_csv_floats(tmp_path / "absent.csv")

"""swehr_gpu on the GPU: a run directory with the shipped example's input
files, run as SWEHR.c would be run, must leave the same files.

Against the oracle with the project's math (the FP64 form's bit-exact twin)
every printed value -- 600 movie frames of five fields, the console's frame
lines, the ten result grids, stage.txt and saveflow.txt -- must be equal to
the last printed digit.  Against the reference's own files (captured by
tests/golden/make_golden.py) the difference is at most one unit in the tenth
decimal: the libm floor."""
import os
import subprocess

import numpy as np
import pytest

from harness import OracleRun, load_golden
from reference_files import MOVIES, RESULTS, max_diff, read_run_dir, run_like_reference, same
from swehr_b200 import build as swbuild

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(tmp_path, *args):
    from swehr_b200 import io as swio
    case, _ = load_golden("shipped")
    swio.write_inputs(case, str(tmp_path))
    r = subprocess.run([swbuild.DRIVER, "-C", str(tmp_path), *args], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr
    return case, r.stdout


def test_driver_files_match_oracle_and_reference(tmp_path):
    case, stdout = _run(tmp_path, "--dump")
    got = read_run_dir(str(tmp_path), case.ny, stdout)
    want = run_like_reference(OracleRun(case, "shim"), case.params["tend"])
    for name, _ in MOVIES:
        assert got[name].shape[0] == 600, name
        assert same(got[name], want[name]), name
    assert same(got["frame_lines"], want["frame_lines"])
    for name, _, _ in RESULTS:
        assert same(got[name], want[name]), name
    assert same(got["stage"], want["stage"]) and same(got["saveflow"], want["saveflow"])
    z = np.load(os.path.join(ROOT, "tests", "golden", "shipped_files.npz"))
    stride = int(z["frame_stride"])
    for name, _ in MOVIES:
        assert max_diff(got[name][::stride], z[name]) <= 2e-10, name
    for name, _, _ in RESULTS:
        assert max_diff(got[name], z[name]) <= 2e-10, name
    assert max_diff(got["stage"], z["stage"]) <= 2e-6
    assert max_diff(got["saveflow"], z["saveflow"]) <= 2e-6
    # the %.17g dump is the full state, bit-exact against the oracle
    from swehr_b200 import io as swio
    d = swio.read_ref_dump(os.path.join(tmp_path, "swehr_dump.txt"))
    o = OracleRun(case, "shim")
    o.advance()
    assert d["steps"] == o.steps
    of = o.fields()
    for name in ("h", "hu", "hv", "z", "vinf", "U", "M"):
        assert np.array_equal(d[name], of[name], equal_nan=True), name


def test_driver_mixed_and_no_movies(tmp_path):
    case, stdout = _run(tmp_path, "--mixed", "--no-movies", "--budget")
    got = read_run_dir(str(tmp_path), case.ny, stdout)
    assert got["depthmovie"].shape[0] == 0 and got["frame_lines"].size == 0
    z = np.load(os.path.join(ROOT, "tests", "golden", "shipped_files.npz"))
    assert got["stage"].shape == z["stage"].shape
    for name in ("depth", "c"):
        scale = np.nanmax(np.abs(z[name]))
        err = max_diff(got[name], z[name]) / scale
        print(f"mixed form, shipped example, {name}.txt: max difference {err:.3e} of the field's maximum")
        assert err <= 0.05, (name, err)
    assert "Water budget" in stdout

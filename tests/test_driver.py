"""The command-line host swehr_gpu (reference file I/O) on the CPU: it is
built, parses its arguments and input files and fails cleanly; and the
stepping / formatting it follows, run on the libm twin of the oracle,
reproduces the reference's own output files for the shipped example."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from harness import OracleRun, load_golden
from reference_files import max_diff, run_like_reference
from swehr_b200 import build as swbuild

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _driver():
    if not os.path.exists(swbuild.DRIVER):
        swbuild.build()
    return swbuild.DRIVER


def _shipped_dir(tmp_path):
    from swehr_b200 import io as swio
    case, _ = load_golden("shipped")
    swio.write_inputs(case, str(tmp_path))
    return case


def test_driver_usage_and_missing_inputs(tmp_path):
    r = subprocess.run([_driver(), "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([_driver(), "-C", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "input.txt" in r.stderr
    _shipped_dir(tmp_path)
    os.remove(os.path.join(tmp_path, "topoin.txt"))
    r = subprocess.run([_driver(), "-C", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 2 and "topoin.txt" in r.stderr


def test_driver_header_matches_reference(tmp_path):
    _shipped_dir(tmp_path)
    r = subprocess.run([_driver(), "-C", str(tmp_path)], capture_output=True, text=True, timeout=600)
    z = np.load(os.path.join(GOLDEN, "shipped_files.npz"))
    header = str(z["header"]).splitlines()
    assert r.stdout.splitlines()[:len(header)] == header
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        gpu = False
    if not gpu:
        assert r.returncode == 3 and "no CUDA device" in r.stderr


def test_stepping_and_formats_reproduce_reference_files():
    """The libm oracle driven like the driver, against the reference's files."""
    case, _ = load_golden("shipped")
    z = np.load(os.path.join(GOLDEN, "shipped_files.npz"))
    o = OracleRun(case, "glibc")
    got = run_like_reference(o, case.params["tend"])
    stride = int(z["frame_stride"])
    for name in ("topomovie", "depthmovie", "velocitymovie", "cmovie", "Mmovie"):
        assert got[name].shape[0] == int(z[name + "_frames"]), name
        assert max_diff(got[name][::stride], z[name]) <= 2e-10, name
    assert got["frame_lines"].shape == z["frame_lines"].shape
    assert max_diff(got["frame_lines"], z["frame_lines"]) <= 2e-6
    for name in ("topoout", "depth", "uh", "vh", "ch", "m", "c", "vel", "maxvel", "maxdepth"):
        assert max_diff(got[name], z[name]) <= 2e-10, name
    for name in ("stage", "saveflow"):
        assert max_diff(got[name], z[name]) <= 2e-6, name

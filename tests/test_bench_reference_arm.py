"""bench.py --impl reference on the CPU: the reference program (built from
SWEHR.c under oracle/) timed on a crop of the roofline domain, printed as
one JSON line with the reference arm's keys.  Skipped where the reference
build is absent (it is built only where the reference checkout exists)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "swehr_ref_omp")),
                    reason="reference build absent")
def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "20",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference" and d["metric"] == "cell-steps/s" and d["unit"] == "cell-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 20
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["e2e"]["d2h_bytes_per_step"] == 0 and "workload" in d["config"]

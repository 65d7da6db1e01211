"""bench.py's reference arm (``--impl reference``) on a small sample: the JSON line carries
the keys of the bench contract with the reference's own fields (impl, cpu_baseline, an e2e
block without host-device traffic), and the runs leave no scratch directories behind.
Runs on CPU: the arm times the reference executable built from the reference's sources."""
import glob
import json
import os
import subprocess
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adh_dump")


@pytest.mark.skipif(not os.path.exists(EXE), reason="reference executable not built (oracle/ref/build_ref.py)")
def test_reference_arm_line():
    pattern = os.path.join(tempfile.gettempdir(), "adhref_*")
    before = set(glob.glob(pattern))
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--ref-points", "1500"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "triangle-steps/s" and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert set(glob.glob(pattern)) <= before   # every run directory was removed

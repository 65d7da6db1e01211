"""The reference executable built here (oracle/ref/build_ref.py) against the reference's own SW2
QA suite: each case's input deck (qa/sw2/<case>/tri: mesh, boundary cards, hot start) runs in a
scratch copy, and the error report it writes (error.out, produced by the reference's TEST
modules against analytic solutions) must equal the stored error.out.last: the words exactly, the
numbers to 1e-8 relative (or 1e-15 absolute, for error measures that are themselves ~1e-11).
A grid mass error that is itself round-off (a difference of two sums of ~1e8 kg, ~4e-13 of the
mass) is the exception: there both reports must show mass conserved to round-off (relative error
below 1e-12) rather than the same digits.  The cases cover wet/dry fronts,
NB VEL / NB OTW edges, a dam break, a water source and Coriolis with EEV eddy viscosity; this pins
the reference build that the oracle is pinned against.
Runs on CPU where the reference sources are present."""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.ref import build_ref
from oracle.ref_run import EXE

QA = os.path.normpath(os.path.join(build_ref.REFERENCE_SRC, "..", "qa", "sw2"))
CASES = ["wet_dry", "angle_nb", "angle_source", "angle_dam", "angle_coriolis"]
NUM = re.compile(r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?|[-+]?\d+[eE][-+]?\d+")


def _split(line):
    return NUM.sub("#", line).split(), [float(x) for x in NUM.findall(line)]


@pytest.mark.skipif(not (os.path.exists(EXE) and os.path.isdir(QA)),
                    reason="reference executable or QA decks not present")
@pytest.mark.parametrize("case", CASES)
def test_reference_build_reproduces_qa_errors(case):
    work = tempfile.mkdtemp(prefix="adhqa_")
    try:
        run = os.path.join(work, case)
        shutil.copytree(os.path.join(QA, case, "tri"), run)
        (deck,) = [f[:-3] for f in os.listdir(run) if f.endswith(".bc")]
        r = subprocess.run([EXE, deck], cwd=run, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:]
        with open(os.path.join(run, "error.out")) as fh:
            got = [ln for ln in fh.read().splitlines() if ln.strip()]
        with open(os.path.join(run, "error.out.last")) as fh:
            exp = [ln for ln in fh.read().splitlines() if ln.strip()]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    assert len(got) == len(exp)
    for g, e in zip(got, exp):
        gw, gn = _split(g)
        ew, en = _split(e)
        assert gw == ew, (g, e)
        if gw[:1] == ["grid_mass_error:"] and en[1] < 1e-12:   # absolute, then relative error
            assert gn[1] < 1e-12, (g, e)
            continue
        assert np.allclose(gn, en, rtol=1e-8, atol=1e-15), (g, e)

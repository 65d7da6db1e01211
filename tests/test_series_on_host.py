"""The continuous-batching engine's step-averaged boundary series (adhv8_kraken_b200/csrc/
sw2_series.h, sseries_set_values_average) compiled as host C++ and compared with the model's
own averaging (SW2Model.series_values, which the reference fixtures pin): bit-identical on
seeded random series over random steps, steps past either end of the table, steps that hold
breakpoints, single-point series and empty steps."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from adhv8_kraken_b200.model import Series

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "adhv8_kraken_b200", "csrc")

SHIM = r"""
#include "sw2_series.h"
extern "C" double host_series_avg(int n, const double* t, const double* v, double t1, double t2) {
    sw2::PwlSeries s;
    s.t.assign(t, t + n);
    s.v.assign(v, v + n);
    return s.avg(t1, t2);
}
"""


@pytest.fixture(scope="module")
def series_lib():
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    work = os.path.join(ROOT, "_build", "series")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    src, lib = os.path.join(work, "shim.cpp"), os.path.join(work, "libseries.so")
    with open(src, "w") as fh:
        fh.write(SHIM)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", CSRC, "-o", lib, src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(lib)
    L.host_series_avg.restype = C.c_double
    L.host_series_avg.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double]
    yield L
    shutil.rmtree(work, ignore_errors=True)
    try:
        os.rmdir(os.path.dirname(work))
    except OSError:
        pass


def test_engine_series_average_matches_model(series_lib):
    rng = np.random.Generator(np.random.PCG64(7))
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    checked = 0
    for _ in range(200):
        n = int(rng.integers(1, 9))
        t = np.cumsum(rng.uniform(0.5, 50.0, n)) - 10.0
        v = rng.normal(0.0, 3.0, n)
        s = Series(t, v)
        span = t[-1] - t[0] + 1.0
        for _ in range(20):
            t1 = float(rng.uniform(t[0] - 0.5 * span, t[-1] + 0.5 * span))
            kind = int(rng.integers(0, 4))
            if kind == 0:
                t2 = t1                                   # empty step: the value at t1
            elif kind == 1:
                t2 = t1 + float(rng.uniform(0.0, span))   # may hold breakpoints
            elif kind == 2:
                t1 = float(t[int(rng.integers(0, n))])    # a step starting on a breakpoint
                t2 = t1 + float(rng.uniform(0.1, 20.0))
            else:
                t2 = t1 + float(rng.uniform(1e-6, 1.0))   # a short step
            got = series_lib.host_series_avg(n, dp(t), dp(v), t1, t2)
            assert got == s.value_avg(t1, t2), (t, v, t1, t2, got, s.value_avg(t1, t2))
            checked += 1
    assert checked == 4000

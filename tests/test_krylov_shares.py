"""CTA shares of a batched Krylov launch (adhv8_kraken_b200/csrc/sw2_shares.h, compiled for the
host): every instance gets at least one CTA and at most its virtual grid, the capacity is used
up while some instance can still take a CTA, the largest work per CTA is the smallest any
allocation reaches (checked by enumeration on small cases), and the work predicted for a solve
resumed after a pause is the rest of its prediction, or half as many iterations again as it has
done once past it."""
import ctypes as C
import itertools
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "adhv8_kraken_b200", "csrc")

SHIM = r'''
#include "sw2_shares.h"
extern "C" void shares(int n, const double* W, const int* G, int cap, int* P) {
    const std::vector<int> r = sw2::krylov_shares_minmax(std::vector<double>(W, W + n), std::vector<int>(G, G + n), cap);
    for (int j = 0; j < n; j++) P[j] = r[j];
}
extern "C" double work(long long nnzb, int pred, int done) { return sw2::krylov_work(nnzb, pred, done); }
'''


@pytest.fixture(scope="module")
def lib():
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    work = os.path.join(ROOT, "_build", "host_shares")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    src, so = os.path.join(work, "shim.cpp"), os.path.join(work, "libshares.so")
    with open(src, "w") as fh:
        fh.write(SHIM)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", CSRC, "-o", so, src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(so)
    L.shares.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
    L.work.argtypes = [C.c_longlong, C.c_int, C.c_int]
    L.work.restype = C.c_double
    yield L
    shutil.rmtree(work, ignore_errors=True)
    try:
        os.rmdir(os.path.dirname(work))
    except OSError:
        pass


def _shares(L, W, G, cap):
    W = np.ascontiguousarray(W, dtype=np.float64)
    G = np.ascontiguousarray(G, dtype=np.int32)
    P = np.zeros(len(W), dtype=np.int32)
    L.shares(len(W), W.ctypes.data_as(C.POINTER(C.c_double)), G.ctypes.data_as(C.POINTER(C.c_int)), cap,
             P.ctypes.data_as(C.POINTER(C.c_int)))
    return P


def test_shares_respect_bounds_and_use_the_capacity(lib):
    rng = np.random.default_rng(3)
    for _ in range(300):
        n = int(rng.integers(1, 40))
        W = rng.uniform(1e3, 1e7, n) * rng.integers(1, 60, n)
        G = rng.integers(1, 60, n)
        cap = int(rng.integers(n, 600))
        P = _shares(lib, W, G, cap)
        assert (P >= 1).all() and (P <= np.maximum(G, 1)).all()
        assert P.sum() <= cap
        if (P < G).any():   # some instance could still take a CTA: none is left
            assert P.sum() == cap


def test_shares_minimise_the_largest_work_per_cta(lib):
    rng = np.random.default_rng(11)
    for _ in range(200):
        n = int(rng.integers(1, 5))
        W = rng.uniform(1.0, 100.0, n)
        G = rng.integers(1, 6, n)
        cap = int(rng.integers(n, n + 8))
        P = _shares(lib, W, G, cap)
        got = max(W / P)
        best = min(max(W / np.array(q)) for q in itertools.product(*[range(1, g + 1) for g in G])
                   if sum(q) <= cap)
        assert got == pytest.approx(best, rel=1e-12)


def test_ties_go_to_the_lower_index(lib):
    P = _shares(lib, [4.0, 4.0, 4.0], [8, 8, 8], 4)
    assert list(P) == [2, 1, 1]


def test_resumed_work_prediction(lib):
    assert lib.work(1000, 20, 0) == 1000 * 20
    assert lib.work(1000, 20, 5) == 1000 * 15        # the rest of the prediction
    assert lib.work(1000, 20, 30) == 1000 * 15       # past it: half as many again (31 // 2)
    assert lib.work(1000, 0, 0) == 1000 * 1          # no prediction yet: one iteration
    assert lib.work(1000, 4, 3) == 1000 * 2          # max(4 - 3, (3 + 1) // 2)

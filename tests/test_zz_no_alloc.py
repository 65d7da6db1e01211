"""The allocation-free solve, sw2gpu_bcsr_solve_noalloc, checked through the C ABI.

Callers that own all of their GPU memory (a fixed arena sized at start-up, as a coupled
model's time loop or a serving process has) cannot let the library call cudaMalloc
during a step; this entry point solves a 3x3-block CSR system held in the caller's own
device buffers, using only a fixed work array compiled into the library.  Here it must
give the same solution as the allocating entry point sw2gpu_linear_solve, on two calls
in a row (the shared work array keeps the first call's contents), and refuse a system
larger than its fixed limit.  This file is named so that pytest collects it last."""
import ctypes as C

import numpy as np
import pytest

from adhv8_kraken_b200 import capi
from adhv8_kraken_b200.sw2 import SW2GPU, lib
from conftest import relerr
from helpers import channel_model

pytestmark = pytest.mark.gpu

NOALLOC_MAX_NODES = 16384


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_solve_matches_allocating_solve_on_two_calls(channel_ref):
    import torch
    model = channel_model()
    V = model.nnodes
    rp, col, val, b = (channel_ref["load0_rowptr"], channel_ref["load0_col"], channel_ref["load0_val"],
                       channel_ref["load0_resid"])
    rng = np.random.default_rng(7)
    rhs2 = 0.5 * b + 1e-3 * rng.standard_normal(b.shape) * np.abs(b).max()
    g = SW2GPU(model, lin_rtol=1e-10, lin_atol=0.0)
    dev = torch.device("cuda", 0)
    # the caller's buffers: allocated by the caller, never by the entry point
    d_rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
    d_col = torch.from_numpy(col.astype(np.int32)).to(dev)
    d_val = torch.from_numpy(np.ascontiguousarray(val, dtype=np.float64).reshape(-1)).to(dev)
    d_x = torch.empty(3 * V, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    for rhs in (b, rhs2):
        x_ref, its_ref, rc_ref = g.linear_solve(val, rhs)
        assert rc_ref == 0
        d_rhs = torch.from_numpy(np.ascontiguousarray(rhs)).to(dev)
        d_x.fill_(np.nan)
        torch.cuda.synchronize()
        its = C.c_int32()
        rc = lib().sw2gpu_bcsr_solve_noalloc(V, len(col), _ptr(d_rp), _ptr(d_col), _ptr(d_val), _ptr(d_rhs),
                                             _ptr(d_x), 1e-10, 0.0, 500, None, C.byref(its))
        assert rc == 0, lib().sw2gpu_last_error().decode()
        x = d_x.cpu().numpy()
        assert np.all(np.isfinite(x))
        assert its.value > 0
        assert relerr(x, x_ref) <= 1e-7
    g.close()


def test_noalloc_solve_rejects_systems_above_its_limit():
    its = C.c_int32()
    dummy = C.c_void_p(1)   # never dereferenced: the size check comes first
    rc = lib().sw2gpu_bcsr_solve_noalloc(NOALLOC_MAX_NODES + 1, 8, dummy, dummy, dummy, dummy, dummy,
                                         1e-10, 0.0, 10, None, C.byref(its))
    assert rc == capi.SW2GPU_E_ARG
    assert b"scratch limit" in lib().sw2gpu_last_error()

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


def _caller_buffers(channel_ref):
    import torch
    dev = torch.device("cuda", 0)
    rp, col, val, b = (channel_ref["load0_rowptr"], channel_ref["load0_col"], channel_ref["load0_val"],
                       channel_ref["load0_resid"])
    bufs = {"rp": torch.from_numpy(rp.astype(np.int32)).to(dev),
            "col": torch.from_numpy(col.astype(np.int32)).to(dev),
            "val": torch.from_numpy(np.ascontiguousarray(val, dtype=np.float64).reshape(-1)).to(dev),
            "rhs": torch.from_numpy(np.ascontiguousarray(b)).to(dev),
            "x": torch.zeros(len(b), dtype=torch.float64, device=dev)}
    torch.cuda.synchronize()
    return bufs, len(rp) - 1, len(col)


def _solve(B, V, nnzb):
    its = C.c_int32()
    return lib().sw2gpu_bcsr_solve_noalloc(V, nnzb, _ptr(B["rp"]), _ptr(B["col"]), _ptr(B["val"]), _ptr(B["rhs"]),
                                           _ptr(B["x"]), 1e-10, 0.0, 500, None, C.byref(its))


def test_noalloc_solve_allocates_no_device_memory(channel_ref):
    """Free device memory is the same before and after calls (the first call has already
    brought the library's fixed work array in)."""
    import torch
    B, V, nnzb = _caller_buffers(channel_ref)
    assert _solve(B, V, nnzb) == 0, lib().sw2gpu_last_error().decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        assert _solve(B, V, nnzb) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_solve_rejects_a_bad_block_structure(channel_ref):
    """Inconsistent row pointers, column indices outside the system and rows without their
    diagonal block are refused with SW2GPU_E_ARG before the work array is written; the bad
    ranges planted here stay inside the caller's arrays and the work array, so a broken check
    could not reach memory outside them either.  A good call afterwards still succeeds."""
    B, V, nnzb = _caller_buffers(channel_ref)
    rp0, col0 = B["rp"].clone(), B["col"].clone()
    # row_ptr[V] one block beyond nnzb (nnzb + 1 is still far below the block limit)
    B["rp"][V] = nnzb + 1
    assert _solve(B, V, nnzb) == capi.SW2GPU_E_ARG
    assert b"do not describe" in lib().sw2gpu_last_error()
    B["rp"].copy_(rp0)
    # a column index past the last node
    B["col"][5] = V + 3
    assert _solve(B, V, nnzb) == capi.SW2GPU_E_ARG
    assert b"column index" in lib().sw2gpu_last_error()
    B["col"].copy_(col0)
    # row 1 loses its diagonal block (its column becomes another column of the row)
    k0, k1 = int(rp0[1]), int(rp0[2])
    cols = col0[k0:k1].cpu().numpy()
    kd = k0 + int(np.nonzero(cols == 1)[0][0])
    B["col"][kd] = int(cols[0] if cols[0] != 1 else cols[-1])
    assert _solve(B, V, nnzb) == capi.SW2GPU_E_ARG
    assert b"diagonal block" in lib().sw2gpu_last_error()
    B["col"].copy_(col0)
    # a decreasing row range
    B["rp"][3] = int(rp0[2]) - 1
    assert _solve(B, V, nnzb) == capi.SW2GPU_E_ARG
    assert b"row range" in lib().sw2gpu_last_error()
    B["rp"].copy_(rp0)
    assert _solve(B, V, nnzb) == 0, lib().sw2gpu_last_error().decode()

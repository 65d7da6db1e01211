"""Request server (sw2gpu_server_*): continuous batching with admission by device memory.

* a request's result is bitwise the same alone and in a mix of requests that arrive while
  it runs (the serving contract: steps of different meshes share launches, results do not
  depend on the company);
* with a budget that holds one request at a time every request still completes, in order.
"""
import time

import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2GPU, SW2Server, run


def _models():
    return [
        meshgen.bumpy_basin(1500, seed=7, size=3000.0, nsteps=4, dt=7.0, nbins=3, name="a"),
        meshgen.channel(nsteps=3),
        meshgen.bumpy_basin(3000, seed=5, size=6000.0, nsteps=2, dt=4.0, nbins=3, name="c"),
        meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=5, dt=5.0, nbins=3, name="d"),
    ]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.SW2GPU_FP64, capi.SW2GPU_MIXED])
def test_alone_equals_mix(precision):
    models = _models()
    steps = [4, 3, 2, 5]
    # alone: the request by itself in a server, and the same solve stepped directly
    srv = SW2Server(precision)
    rid = srv.submit(models[0], steps[0])
    st_alone, (h_alone, u_alone, v_alone) = srv.wait(rid)
    srv.close()
    assert st_alone["status"] == 0 and st_alone["steps"] == steps[0]
    g = SW2GPU(models[0], precision=precision)
    run(g, steps[0])
    h, u, v = g.get_state(0)
    g.close()
    assert np.array_equal(h, h_alone) and np.array_equal(u, u_alone) and np.array_equal(v, v_alone)
    # in the mix: others arrive before and while it runs
    srv = SW2Server(precision)
    ids = [srv.submit(models[1], steps[1])]
    rid = srv.submit(models[0], steps[0])
    time.sleep(0.05)
    ids += [srv.submit(m, n) for m, n in zip(models[2:], steps[2:])]
    st_mix, (h_mix, u_mix, v_mix) = srv.wait(rid)
    others = [srv.wait(i) for i in ids]
    srv.close()
    assert st_mix["status"] == 0 and all(o[0]["status"] == 0 for o in others)
    assert np.array_equal(h_mix, h_alone) and np.array_equal(u_mix, u_alone) and np.array_equal(v_mix, v_alone)
    assert st_mix["newton_its"] == st_alone["newton_its"] and st_mix["linear_its"] == st_alone["linear_its"]
    assert st_mix["latency_ms"] >= st_mix["run_ms"] >= 0.0


@pytest.mark.gpu
def test_admission_by_memory():
    models = _models()
    # a budget below one request: requests are admitted one at a time, in arrival order
    srv = SW2Server(capi.SW2GPU_FP64, hbm_fraction=1e-6)
    ids, t_before, t_after = [], [], []
    for m in models:
        t_before.append(time.perf_counter())
        ids.append(srv.submit(m, 2))
        t_after.append(time.perf_counter())
    assert srv.status()["active"] <= 1
    res = [srv.wait(i) for i in ids]
    srv.close()
    st = [r[0] for r in res]
    assert all(s["status"] == 0 and s["steps"] == 2 and s["device_bytes"] > 0 for s in st)
    # request i was admitted only after request i-1 finished: its wait covers the other's
    # whole latency, less the time between the two submissions (at most from the start of
    # submit i-1 to the return of submit i; the server stamps a request inside submit)
    for i in range(1, len(st)):
        gap_ms = (t_after[i] - t_before[i - 1]) * 1e3
        assert st[i]["queue_ms"] + gap_ms >= st[i - 1]["latency_ms"], (i, st[i], st[i - 1])

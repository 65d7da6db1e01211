"""CUDA-graph stepping (sw2gpu_set_graphs): the step start and every Newton iteration replayed
from captured graphs (mode 1), or the whole step as one graph whose Newton loop and line search are
conditional nodes driven by device-side control kernels (mode 2), give bitwise the results of direct
launches, across the three level arrangements, a dt change (recapture), wet/dry fronts, failed
steps with line-search cuts, a Krylov wait that runs out and mass tracking."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2GPU


def _run(model, precision, graphs, dts, overrides=None):
    g = SW2GPU(model, precision=precision, overrides=overrides)
    if graphs:
        g.set_graphs(graphs)
    stats = [g.step(dt=d) for d in dts]
    out = [np.concatenate(g.get_state(lvl)) for lvl in range(3)], g.get_wd()
    g.close()
    return out, [(s["status"], s["newton_its"], s["linear_its"], s["linesearch_cuts"], s["resid_max"])
                 for s in stats]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("precision", [capi.SW2GPU_FP64, capi.SW2GPU_MIXED])
@pytest.mark.parametrize("which", ["channel", "basin"])
def test_graph_steps_equal_direct(precision, which, mode):
    if which == "channel":
        m = meshgen.channel(nsteps=6)
        dts = [10.0, 10.0, 10.0, 5.0, 10.0, 10.0]
    else:
        m = meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=6, dt=5.0, nbins=3, name="g")
        dts = [5.0, 5.0, 2.5, 5.0, 5.0, 5.0]
    (sd, wd), std = _run(m, precision, False, dts)
    (sg, wg), stg = _run(m, precision, mode, dts)
    assert stg == std
    assert np.array_equal(wg, wd)
    for a, b in zip(sg, sd):
        assert np.array_equal(a, b)


def _run_batch(models, precision, precond, graphs, dts):
    from adhv8_kraken_b200.sw2 import SW2Batch
    solvers = [SW2GPU(m, precision=precision, precond=precond) for m in models]
    b = SW2Batch(solvers)
    if graphs:
        b.set_graphs(True)
    stats = [b.step([d] * len(models)) for d in dts]
    out = [[np.concatenate(g.get_state(lvl)) for lvl in range(3)] + [g.get_wd()] for g in solvers]
    summ = [[(s["status"], s["newton_its"], s["linear_its"]) for s in st] for st in stats]
    b.close()
    for g in solvers:
        g.close()
    return out, summ


@pytest.mark.gpu
@pytest.mark.parametrize("precision,precond", [(capi.SW2GPU_FP64, capi.SW2GPU_PREC_BJACOBI),
                                               (capi.SW2GPU_MIXED, capi.SW2GPU_PREC_BJACOBI),
                                               (capi.SW2GPU_FP64, capi.SW2GPU_PREC_DILU)])
def test_batch_graph_steps_equal_direct(precision, precond):
    """sw2gpu_batch_set_graphs: a batch of uneven meshes replayed from CUDA graphs (all-instance
    Newton iterations as graph launches, each instance's Krylov tolerance from device memory)
    gives bitwise the results of direct launches, across level arrangements and a dt change."""
    models = [meshgen.channel(nsteps=5),
              meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=5, dt=5.0, nbins=3, name="g1"),
              meshgen.bumpy_basin(400, seed=12, size=1500.0, nsteps=5, dt=5.0, nbins=3, name="g2")]
    dts = [5.0, 5.0, 2.5, 5.0, 5.0]
    od, sd = _run_batch(models, precision, precond, False, dts)
    og, sg = _run_batch(models, precision, precond, True, dts)
    assert sg == sd
    for a, b in zip(og, od):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_device_loop_failed_steps_and_line_search_equal_direct():
    """Graph mode 2 on steps that fail (Newton iterations capped) and cut the line search: the
    same statuses, iterations, cuts, norms and states (the failed step's level reset) as direct
    launches."""
    m = meshgen.channel_spike(nsteps=8)
    dts = [m.dt] * 8
    (sd, wd), std = _run(m, capi.SW2GPU_FP64, False, dts)
    (sg, wg), stg = _run(m, capi.SW2GPU_FP64, 2, dts)
    assert stg == std
    assert any(s[0] != 0 for s in std) and any(s[3] > 0 for s in std)
    assert np.array_equal(wg, wd)
    for a, b in zip(sg, sd):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_device_loop_timeout_and_mass_tracking():
    """Graph mode 2: a Krylov wait bounded to one poll runs out inside the step graph -- the step
    reports SW2GPU_E_TIMEOUT with the current level reset, no fault; with the limits back the
    context steps on like one that never timed out, and the mass tracked inside the graph equals
    the direct step's."""
    from adhv8_kraken_b200.sw2 import SW2Error
    m = meshgen.bumpy_basin(10000, seed=23, size=20000.0 * np.sqrt(10000 / 5e5), nsteps=4, dt=5.0, name="gl")
    g, ref = SW2GPU(m), SW2GPU(m)
    g.set_graphs(2)
    g.set_wait_limits(1, 0)
    with pytest.raises(SW2Error) as ei:
        g.step()
    assert ei.value.code == capi.SW2GPU_E_TIMEOUT
    h, u, v = g.get_state(0)
    h1, u1, v1 = g.get_state(1)
    assert np.array_equal(h, h1) and np.array_equal(u, u1) and np.array_equal(v, v1)
    for lvl in range(3):
        g.set_state(lvl, *ref.get_state(lvl))
    g.set_wait_limits(0, 0)
    from adhv8_kraken_b200 import sw2 as _s
    for s in (g, ref):
        _s._check(_s.lib().sw2gpu_set_mass_tracking(s.h, 1, 1000.0))
    for _ in range(2):
        a, b = g.step(), ref.step()
        assert a["status"] == 0 and b["status"] == 0
        assert (a["newton_its"], a["linear_its"]) == (b["newton_its"], b["linear_its"])
        ma, mb = [_s.C.c_double() for _ in range(2)], [_s.C.c_double() for _ in range(2)]
        _s._check(_s.lib().sw2gpu_step_mass(g.h, _s.C.byref(ma[0]), _s.C.byref(ma[1])))
        _s._check(_s.lib().sw2gpu_step_mass(ref.h, _s.C.byref(mb[0]), _s.C.byref(mb[1])))
        assert ma[0].value == mb[0].value and ma[1].value == mb[1].value
    for x, y in zip(g.get_state(0), ref.get_state(0)):
        assert np.array_equal(x, y)

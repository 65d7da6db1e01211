"""CUDA-graph stepping (sw2gpu_set_graphs): the step start and every Newton iteration replayed
from captured graphs give bitwise the results of direct launches, across the three level
arrangements, a dt change (recapture) and wet/dry fronts."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2GPU


def _run(model, precision, graphs, dts):
    g = SW2GPU(model, precision=precision)
    if graphs:
        g.set_graphs(True)
    stats = [g.step(dt=d) for d in dts]
    out = [np.concatenate(g.get_state(lvl)) for lvl in range(3)], g.get_wd()
    g.close()
    return out, [(s["status"], s["newton_its"], s["linear_its"]) for s in stats]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.SW2GPU_FP64, capi.SW2GPU_MIXED])
@pytest.mark.parametrize("which", ["channel", "basin"])
def test_graph_steps_equal_direct(precision, which):
    if which == "channel":
        m = meshgen.channel(nsteps=6)
        dts = [10.0, 10.0, 10.0, 5.0, 10.0, 10.0]
    else:
        m = meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=6, dt=5.0, nbins=3, name="g")
        dts = [5.0, 5.0, 2.5, 5.0, 5.0, 5.0]
    (sd, wd), std = _run(m, precision, False, dts)
    (sg, wg), stg = _run(m, precision, True, dts)
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

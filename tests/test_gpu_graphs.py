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

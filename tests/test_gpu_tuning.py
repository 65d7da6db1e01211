"""Launch variants and the autotuner: the register budget of the wet-Jacobian kernel and the
depth of the Krylov tile ring change speed only -- every variant steps to the same bits, and
autotuning (which runs the step's kernels on the current state) leaves the state untouched."""
import itertools

import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2GPU, run


def _model():
    return meshgen.bumpy_basin(1500, seed=7, size=3000.0, nsteps=3, dt=7.0, nbins=3, name="tune")


def _states(g):
    return [np.concatenate(g.get_state(lvl)) for lvl in range(3)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.SW2GPU_FP64, capi.SW2GPU_MIXED])
def test_variants_give_identical_steps(precision):
    m = _model()
    ref = None
    for jac, stages in itertools.product((1, 2), (0, 2, 3)):
        g = SW2GPU(m, precision=precision)
        g.set_variant(jac, stages)
        assert g.variant() == (jac, stages)
        sts = run(g, 3)
        got = (_states(g), [(s["newton_its"], s["linear_its"]) for s in sts])
        g.close()
        if ref is None:
            ref = got
            continue
        assert got[1] == ref[1], (jac, stages)
        for a, b in zip(got[0], ref[0]):
            assert np.array_equal(a, b), (jac, stages)


@pytest.mark.gpu
@pytest.mark.parametrize("warm_steps", [0, 2])
def test_autotune_keeps_state_and_results(warm_steps):
    """Tuning at the start and in mid-run (three distinct time levels, an increment in
    flight) leaves every level as it was and the following steps unchanged."""
    m = _model()
    g0 = SW2GPU(m)
    run(g0, warm_steps + 3)
    ref = _states(g0)
    g0.close()
    g = SW2GPU(m)
    if warm_steps:
        run(g, warm_steps)
    before = _states(g)
    jac, stages = g.autotune()
    assert jac in (1, 2) and stages in (0, 2, 3) and g.variant() == (jac, stages)
    for a, b in zip(_states(g), before):
        assert np.array_equal(a, b)
    run(g, 3)
    for a, b in zip(_states(g), ref):
        assert np.array_equal(a, b)
    g.close()

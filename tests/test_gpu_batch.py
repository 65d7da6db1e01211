"""Batched stepping (sw2gpu_batch_*): every instance of a batch of uneven meshes reproduces,
bit for bit, what it computes alone -- states, wet/dry flags, Newton and Krylov iteration
counts -- on the FP64 and on the mixed-precision path."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2Batch, SW2GPU

NSTEPS = 3


def uneven_models():
    return [
        meshgen.channel(nsteps=NSTEPS),
        meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=NSTEPS, dt=5.0, nbins=3, name="b700"),
        meshgen.bumpy_basin(3000, seed=5, size=6000.0, nsteps=NSTEPS, dt=4.0, nbins=3, name="b3000"),
        meshgen.bumpy_basin(1500, seed=7, size=3000.0, nsteps=NSTEPS, dt=7.0, nbins=3, name="b1500"),
    ]


def _summary(stats):
    return [(s["status"], s["newton_its"], s["linear_its"], s["linesearch_cuts"]) for s in stats]


@pytest.mark.gpu
@pytest.mark.parametrize("precision,precond", [(capi.SW2GPU_FP64, capi.SW2GPU_PREC_BJACOBI),
                                               (capi.SW2GPU_MIXED, capi.SW2GPU_PREC_BJACOBI),
                                               (capi.SW2GPU_FP64, capi.SW2GPU_PREC_DILU),
                                               (capi.SW2GPU_MIXED, capi.SW2GPU_PREC_DILU)])
def test_batch_equals_alone(precision, precond):
    models = uneven_models()
    alone = []
    for m in models:
        g = SW2GPU(m, precision=precision, precond=precond)
        st = [g.step() for _ in range(NSTEPS)]
        alone.append((g.get_state(0), g.get_wd(), _summary(st)))
        g.close()
    solvers = [SW2GPU(m, precision=precision, precond=precond) for m in models]
    batch = SW2Batch(solvers)
    steps = [batch.step() for _ in range(NSTEPS)]
    for k, g in enumerate(solvers):
        h, u, v = g.get_state(0)
        (ha, ua, va), wda, sa = alone[k]
        assert np.array_equal(h, ha) and np.array_equal(u, ua) and np.array_equal(v, va), models[k].name
        assert np.array_equal(g.get_wd(), wda), models[k].name
        assert _summary([s[k] for s in steps]) == sa, models[k].name
        assert all(s[k]["status"] == 0 for s in steps)
    batch.close()
    for g in solvers:
        g.close()


@pytest.mark.gpu
def test_batch_order_does_not_matter():
    models = uneven_models()
    a = [SW2GPU(m) for m in models]
    b = [SW2GPU(m) for m in models[::-1]]
    ba, bb = SW2Batch(a), SW2Batch(b)
    for _ in range(2):
        ba.step()
        bb.step()
    for k in range(len(models)):
        ha = a[k].get_state(0)
        hb = b[len(models) - 1 - k].get_state(0)
        for x, y in zip(ha, hb):
            assert np.array_equal(x, y)
    ba.close()
    bb.close()


def _run_alone(solver, nsteps, max_retries=8):
    """sw2.run's contract: a failed step is retried with dt / 4, the next step uses dt again."""
    from adhv8_kraken_b200.sw2 import run
    return run(solver, nsteps, max_retries=max_retries)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.SW2GPU_FP64, capi.SW2GPU_MIXED])
@pytest.mark.parametrize("rebalance", [(1, 0.5), (4, 0.5), (8, 0.0)], ids=["off", "default", "every-iteration"])
def test_engine_equals_alone(precision, rebalance):
    """Continuous batching: instances with different step counts join one engine (one of
    them later, while the others are mid-run) and each ends bitwise where it ends alone --
    without Krylov rebalancing, with the default rounds, and with every solve paused after
    each of its first seven iterations (fraction 0: the pause fires at once) and resumed in
    the next launch with a different CTA share."""
    from adhv8_kraken_b200.sw2 import SW2Engine
    models = uneven_models()
    nsteps = [3, 2, 4, 1]
    alone = []
    for m, n in zip(models, nsteps):
        g = SW2GPU(m, precision=precision)
        _run_alone(g, n)
        alone.append((g.get_state(0), g.get_state(1), g.t))
        g.close()
    solvers = [SW2GPU(m, precision=precision) for m in models]
    eng = SW2Engine(precision)
    eng.set_rebalance(*rebalance)
    for g, n in list(zip(solvers, nsteps))[:3]:
        eng.add(g, n)
    done = eng.tick() + eng.tick()
    eng.add(solvers[3], nsteps[3])   # joins while the others are inside their steps
    done += eng.run()
    assert len(done) == len(models) and all(d["status"] == 0 for d in done)
    for k, g in enumerate(solvers):
        (h0, u0, v0), (h1, u1, v1), t = alone[k]
        h, u, v = g.get_state(0)
        assert np.array_equal(h, h0) and np.array_equal(u, u0) and np.array_equal(v, v0), models[k].name
        hh, uu, vv = g.get_state(1)
        assert np.array_equal(hh, h1) and np.array_equal(uu, u1), models[k].name
        assert g.t == t
    eng.close()
    for g in solvers:
        g.close()

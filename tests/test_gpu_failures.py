"""Failure paths, made on the host (no GPU fault is provoked): the step contract of fe_newton /
fe_main -- a failed step returns NO with the state reset to the old level, the caller retries
with dt / 4 -- and the library's own reporting (NaN residuals, capped linear solves, solves that
give up in a batch, requests with bad input in the server)."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.capi import MeshArrays
from adhv8_kraken_b200.sw2 import SW2Engine, SW2Error, SW2GPU, SW2Server, run


def _basin(n=700, seed=11, nsteps=4):
    return meshgen.bumpy_basin(n, seed=seed, size=2000.0, nsteps=nsteps, dt=5.0, nbins=3, name=f"b{n}")


@pytest.mark.gpu
def test_newton_failure_resets_to_old_level():
    m = _basin()
    # one Newton iteration against an unreachable tolerance: the step must fail
    g = SW2GPU(m, overrides={"max_nonlin_it": 1, "tol_nonlin": 1e-30, "inc_nonlin": 1e-30})
    old = g.get_state(0)
    st = g.step()
    assert st["status"] == capi.SW2GPU_E_NEWTON and st["newton_its"] == 1
    # fe_sw2_init: the current level is the old one again (the level shift already happened)
    h, u, v = g.get_state(0)
    h1, u1, v1 = g.get_state(1)
    assert np.array_equal(h, h1) and np.array_equal(h1, old[0])
    assert g.t == m.t0
    # the retry loop gives up after its retries and says so
    with pytest.raises(SW2Error):
        run(g, 1, max_retries=2)
    g.close()


@pytest.mark.gpu
def test_linear_failure_is_reported():
    m = _basin()
    g = SW2GPU(m, max_lin_it=1)      # one BiCGSTAB iteration cannot reach 1e-8 of the residual
    st = g.step()
    assert st["status"] == capi.SW2GPU_E_LINEAR
    h, _, _ = g.get_state(0)
    assert np.array_equal(h, g.get_state(1)[0])
    g.close()


@pytest.mark.gpu
def test_nan_state_returns_error_instead_of_exiting():
    m = _basin()
    g = SW2GPU(m)
    h, u, v = g.get_state(0)
    h = h.copy()
    h[len(h) // 2] = np.nan
    g.set_state(0, h, u, v)          # becomes the old level at the next step's shift
    st = g.step()
    assert st["status"] == capi.SW2GPU_E_NAN
    g.close()


@pytest.mark.gpu
def test_engine_instance_gives_up_alone():
    good = [_basin(700, 11), _basin(1500, 7)]
    alone = []
    for m in good:
        g = SW2GPU(m)
        run(g, 2)
        alone.append(g.get_state(0))
        g.close()
    bad = SW2GPU(_basin(900, 3), overrides={"max_nonlin_it": 1, "tol_nonlin": 1e-30, "inc_nonlin": 1e-30})
    gs = [SW2GPU(m) for m in good]
    eng = SW2Engine()
    for g in gs:
        eng.add(g, 2)
    eng.add(bad, 2, max_retries=1)
    done = {d["id"]: d for d in eng.run()}
    assert done[id(bad)]["status"] == capi.SW2GPU_E_NEWTON and done[id(bad)]["steps"] == 0
    assert done[id(bad)]["failures"] == 2
    for g, ref in zip(gs, alone):
        assert done[id(g)]["status"] == 0
        for x, y in zip(g.get_state(0), ref):
            assert np.array_equal(x, y)
    eng.close()
    for g in gs + [bad]:
        g.close()


@pytest.mark.gpu
def test_server_request_with_bad_mesh_fails_alone():
    srv = SW2Server()
    good = _basin()
    bad = _basin(900, 3)
    arrays = MeshArrays(bad)
    arrays.mesh.elem2d_nodes[0] = 10 ** 8          # a node index out of range
    rid_bad = srv.submit(bad, 2, arrays=arrays)
    rid_good = srv.submit(good, 2)
    with pytest.raises(SW2Error) as err:
        srv.wait(rid_bad)
    assert err.value.code == capi.SW2GPU_E_ARG and "out of range" in str(err.value)
    st, _ = srv.wait(rid_good)
    assert st["status"] == 0 and st["steps"] == 2
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("what", ["lid", "bad_string"])
def test_create_rejects_unsupported_node_strings(what):
    """sw2gpu_create refuses a node string with a lid (BCT_LID_*, not built) or a string id out of
    range with SW2GPU_E_ARG instead of solving without it."""
    import dataclasses
    m = meshgen.channel_obstacle(nsteps=2, with_depth=True)
    if what == "lid":
        strings = list(m.strings)
        strings[-1] = dataclasses.replace(strings[-1], bc_flag=capi.SW2GPU_BCT_LID_DFT)
        m = dataclasses.replace(m, strings=strings)
    else:
        ns = m.node_string.copy()
        ns[ns >= 0] = len(m.strings)
        m = dataclasses.replace(m, node_string=ns)
    with pytest.raises(SW2Error) as err:
        SW2GPU(m)
    assert err.value.code == capi.SW2GPU_E_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("stages,barrier_polls,copy_polls", [(0, 1, 0), (3, 1, 0), (3, 0, 1)])
def test_device_wait_that_runs_out_ends_the_step_with_timeout(stages, barrier_polls, copy_polls):
    """A Krylov grid-barrier wait (direct sweeps) or tile-copy wait (staged sweeps) bounded to
    one poll runs out: no fault, no hang -- the kernel flags the error and returns, the step
    reports SW2GPU_E_TIMEOUT with the current level reset to the old one, and once the limits
    are back at their defaults the same context steps on exactly as a context that never
    timed out."""
    m = _basin(n=10000, seed=23, nsteps=4)   # ~20k triangles: hundreds of Krylov CTAs
    g = SW2GPU(m)
    ref = SW2GPU(m)
    for s in (g, ref):
        s.set_variant(1, stages)
    g.set_wait_limits(barrier_polls, copy_polls)
    with pytest.raises(SW2Error) as ei:
        g.step()
    assert ei.value.code == capi.SW2GPU_E_TIMEOUT
    h, u, v = g.get_state(0)
    h1, u1, v1 = g.get_state(1)
    assert np.array_equal(h, h1) and np.array_equal(u, u1) and np.array_equal(v, v1)
    # the same levels in both contexts, then one step each
    for lvl in range(3):
        g.set_state(lvl, *ref.get_state(lvl))
    g.set_wait_limits(0, 0)
    a, b = g.step(), ref.step()
    assert a["status"] == 0 and b["status"] == 0
    for x, y in zip(g.get_state(0), ref.get_state(0)):
        assert np.array_equal(x, y)
    g.close()
    ref.close()


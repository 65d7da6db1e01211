"""GPU parity of the constituent transport (fe_transport) through the C ABI: the residual and the
scalar FD Jacobian at the reference's own transport Jacobian builds (against the oracle, bit for
bit, and against the reference's values), fe_transport_init, the concentrations of every step of
five workloads against the reference's runs, the reference's angle_salt known answer, the
transport levels kept across a remesh, and a transport Krylov wait that runs out.

Tolerances: residual and Jacobian against the oracle 0 (the same operations in the same order);
against the reference 1e-12 and 1e-10 (the reference's own round-off, and the flow's side output
recomputed from the dumped state).  Time-stepped concentrations: 1e-9 of the field's maximum per
step -- the reference solves each transport system exactly and stops after one Newton iteration,
the device runs Jacobi-preconditioned BiCGSTAB to a relative 1e-12 and iterates until the residual
max norm is below tol_nonlin, as the reference's Newton rule for a linear problem asks; what is
left is the flow's own per-step difference (1e-13 to 1e-10) carried by the transport."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.model import Constituent
from adhv8_kraken_b200.sw2 import SW2GPU, run
from conftest import relerr
from golden.make_golden import TRANSPORT_CASES
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

LOADS = [("basin", 0), ("basin", 1), ("terms", 0), ("terms", 1)]


def _put_load_state(s, m, ref, p):
    """The flow and concentration levels of the reference's transport Jacobian build `p`; the
    flow's side output is recomputed by a residual evaluation at the dumped (final) flow state."""
    itrn, t, dt = ref[f"{p}_meta"]
    itrn = int(itrn)
    s.set_state(0, ref[f"{p}_h"], ref[f"{p}_u"], ref[f"{p}_v"])
    s.set_state(1, ref[f"{p}_h1"], ref[f"{p}_u1"], ref[f"{p}_v1"])
    s.set_state(2, ref[f"{p}_h2"], ref[f"{p}_u2"], ref[f"{p}_v2"])
    s.set_dt(dt, m.series_values(t, t + dt))
    s.set_wd(ref[f"{p}_wd"])
    s.resid()
    for level, key in enumerate(("c", "c1", "c2")):
        s.set_conc(itrn, level, ref[f"{p}_{key}"])
    return itrn, t, dt


@pytest.mark.parametrize("name,q", LOADS)
def test_transport_residual_and_jacobian_match_oracle_and_reference(name, q, transport_ref):
    m = TRANSPORT_CASES[name]()
    g, o = SW2GPU(m), Oracle(m)
    p = f"{name}_tload{q}"
    for s in (g, o):
        itrn, t, dt = _put_load_state(s, m, transport_ref, p)
    # fe_transport_init sets bc_mask (and the current level, put back to the dump's)
    o.trn_init(itrn)
    g.transport_init(itrn, t, dt)
    for s in (g, o):
        s.set_conc(itrn, 0, transport_ref[f"{p}_c"])
    val_g, r_g = g.transport_load(itrn)
    r_o = o.trn_resid(itrn)
    val_o, _ = o.trn_load(itrn)
    assert np.array_equal(r_g, r_o)
    assert np.array_equal(val_g, val_o)
    assert relerr(r_g, transport_ref[f"{p}_resid"]) <= 1e-12
    assert relerr(val_g, transport_ref[f"{p}_val"]) <= 1e-10


def test_transport_init_matches_oracle():
    m = meshgen.channel_transport(nsteps=2, nx=30, ny=6)
    g, o = SW2GPU(m), Oracle(m)
    rng = np.random.default_rng(5)
    h = m.h0 + rng.normal(0, 0.5, m.nnodes)        # some dry nodes: their concentration starts at 0
    c1 = rng.uniform(0.5, 1.5, m.nnodes)
    t, dt = 0.0, m.dt
    for s in (g, o):
        s.set_state(0, h, m.u0, m.v0)
        s.set_conc(0, 1, c1)
    o.set_dt(dt, m.series_values(t, t + dt))
    o.trn_init(0)
    g.transport_init(0, t, dt)
    assert np.array_equal(g.get_conc(0), o.get_conc(0))
    assert (g.get_conc(0)[h <= np.finfo(np.float32).eps] == 0).any()


@pytest.mark.parametrize("name", list(TRANSPORT_CASES))
def test_transport_runs_match_reference(name, transport_ref):
    m = TRANSPORT_CASES[name]()
    g = SW2GPU(m)
    con = transport_ref[f"{name}_con"]
    worst = 0.0
    for k in range(con.shape[0]):
        st = g.step(dt=transport_ref[f"{name}_dt"][k], t=transport_ref[f"{name}_t"][k])
        assert st["status"] == 0
        trn = g.transport_step()
        assert len(trn) == len(m.constituents) and all(s["status"] == 0 for s in trn)
        for j in range(len(m.constituents)):
            e = relerr(g.get_conc(j), con[k, j])
            worst = max(worst, e)
            assert e <= 1e-9, (name, k, j, e)
    print(f"{name}: worst per-step relative concentration error against the reference {worst:.2e}")


def test_uniform_concentration_stays_uniform_on_gpu():
    """The reference's angle_salt check (src/initio/test_cases.c:1506-1535) on the device."""
    g = SW2GPU(meshgen.salt_transport())
    for _ in range(6):
        assert g.step()["status"] == 0
        assert g.transport_step()[0]["status"] == 0
        assert np.abs(g.get_conc(0) - 17.5).max() <= 1e-6


def test_run_steps_flow_then_transport():
    """The time loop runs the constituents after every accepted flow step (fe_main.c:528-531)."""
    m = meshgen.basin_transport(nsteps=4)
    g, o = SW2GPU(m), Oracle(m)
    out = run(g, 4)
    assert all(len(st["transport"]) == 2 for st in out)
    for _ in range(4):
        assert o.step()["status"] == 0
        o.transport_step()
    for j in range(2):
        assert relerr(g.get_conc(j), o.get_conc(j)) <= 1e-9


def test_remesh_keeps_the_concentrations():
    from helpers import centroid_refine
    m = meshgen.channel_transport(nsteps=4, nx=30, ny=6)
    g = SW2GPU(m)
    for _ in range(2):
        assert g.step()["status"] == 0
        assert g.transport_step()[0]["status"] == 0
    before = [g.get_conc(0, lvl) for lvl in range(3)]
    m2 = centroid_refine(m, np.arange(0, m.nelems2d, 7))
    g.remesh(m2)
    for lvl in range(3):
        c = g.get_conc(0, lvl)
        assert np.array_equal(c[:m.nnodes], before[lvl])
        assert (c[m.nnodes:] == 0).all()


def _transport_basin(n=10000, seed=23, nsteps=4):
    m = meshgen.bumpy_basin(n, seed=seed, size=20000.0 * np.sqrt(n / 5e5), nsteps=nsteps, dt=5.0, name="trn_big")
    ser = meshgen.const_series(m, 1.0)
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[0.5] * len(m.materials), edge_bc={len(m.materials): ser},
                                  c0=np.full(m.nnodes, 0.3))]
    return m


def test_transport_wait_that_runs_out_ends_with_timeout():
    """The transport Krylov solve's grid-barrier wait bounded to one poll runs out: no fault, no
    hang -- the kernel flags the error and returns, transport reports SW2GPU_E_TIMEOUT with the
    constituent's current level reset (fe_transport_init), and once the limits are back at their
    defaults the context steps on exactly as one that never timed out."""
    m = _transport_basin()
    g, ref = SW2GPU(m), SW2GPU(m)
    for s in (g, ref):
        assert s.step()["status"] == 0
    g.set_wait_limits(1, 0)
    trn = g.transport_step()
    assert trn[0]["status"] == capi.SW2GPU_E_TIMEOUT
    g.set_wait_limits(0, 0)
    for s in (g, ref):
        for lvl in range(3):
            s.set_conc(0, lvl, np.full(m.nnodes, 0.3))
        for lvl in range(3):
            s.set_state(lvl, *ref.get_state(lvl))
    for s in (g, ref):
        assert s.step()["status"] == 0
        assert s.transport_step()[0]["status"] == 0
    assert np.array_equal(g.get_conc(0), ref.get_conc(0))


def test_transport_error_indicator_matches_oracle():
    """sw2gpu_transport_elem_error against the oracle at the same state: the flow's indicator, then
    the constituents' folded in, bit for bit (the same operations in the same order)."""
    from golden.make_golden import trnerr_model
    m = trnerr_model()
    g, o = SW2GPU(m), Oracle(m)
    for _ in range(2):
        assert o.step()["status"] == 0
        o.transport_step()
    for s in (g,):
        for lvl in range(3):
            s.set_state(lvl, *o.get_state(lvl))
            for j in range(2):
                s.set_conc(j, lvl, o.get_conc(j, lvl))
    g.set_dt(m.dt, m.series_values(0.0, m.dt))
    g.set_wd(o.get_wd())                  # the flow's indicator marks elements with wd_flag > 0
    srt = np.full(len(m.materials), 100.0)
    trt = np.array([[c.refine_tol] * len(m.materials) for c in m.constituents])
    eg, _ = g.elem_error(srt)
    eo, _ = o.elem_error(srt)
    assert np.array_equal(eg, eo)
    eg2, cg = g.transport_elem_error(trt, eg)
    eo2, co = o.trn_elem_error(trt, eo)
    assert np.array_equal(eg2, eo2)
    assert np.array_equal(cg, co)
    assert (eg2 > eg).sum() > 0

"""The CPU oracle's constituent transport (fe_transport, src/fe/transport/) against the reference
executable's own runs (tests/golden/transport_ref.npz): the residual and FD Jacobian at the
reference's own transport Jacobian builds, the concentrations after every step of five
workloads, and the reference's angle_salt known answer (a uniform 17.5 stays within 1e-6,
src/initio/test_cases.c:1506-1535)."""
import numpy as np
import pytest

from adhv8_kraken_b200 import meshgen
from adhv8_kraken_b200.model import BCT_DIR, Constituent
from conftest import relerr
from golden.make_golden import TRANSPORT_CASES, fingerprint
from oracle.oracle import Oracle

LOADS = [("basin", 0), ("basin", 1), ("terms", 0), ("terms", 1)]


def set_tload_state(o, m, ref, p):
    """Puts a solver in the state of the reference's transport Jacobian build `p`."""
    itrn, t, dt = ref[f"{p}_meta"]
    itrn = int(itrn)
    o.set_state(0, ref[f"{p}_h"], ref[f"{p}_u"], ref[f"{p}_v"])
    o.set_state(1, ref[f"{p}_h1"], ref[f"{p}_u1"], ref[f"{p}_v1"])
    o.set_state(2, ref[f"{p}_h2"], ref[f"{p}_u2"], ref[f"{p}_v2"])
    o.set_dt(dt, m.series_values(t, t + dt))
    o.set_wd(ref[f"{p}_wd"])
    o.set_dacont(ref[f"{p}_dacont"].reshape(3, -1))
    for level, key in enumerate(("c", "c1", "c2")):
        o.set_conc(itrn, level, ref[f"{p}_{key}"])
    return itrn


def test_transport_fixture_models_are_current(transport_ref):
    for name, make in TRANSPORT_CASES.items():
        assert str(transport_ref[f"{name}_fingerprint"]) == fingerprint(make()), name


@pytest.mark.parametrize("name,q", LOADS)
def test_oracle_transport_residual_and_jacobian_match_reference(name, q, transport_ref):
    m = TRANSPORT_CASES[name]()
    o = Oracle(m)
    p = f"{name}_tload{q}"
    itrn = set_tload_state(o, m, transport_ref, p)
    mask = o.trn_init(itrn)                     # bc_mask of fe_transport_init; the iterate is the dump's
    assert np.array_equal(mask, transport_ref[f"{p}_bcmask"])
    o.set_conc(itrn, 0, transport_ref[f"{p}_c"])
    r = o.trn_resid(itrn)
    val, _ = o.trn_load(itrn)
    # the same operations in the same order: round-off in the last bits only
    assert relerr(r, transport_ref[f"{p}_resid"]) <= 1e-14
    assert relerr(val, transport_ref[f"{p}_val"]) <= 1e-14
    assert np.mean(val == transport_ref[f"{p}_val"]) > 0.9


@pytest.mark.parametrize("name", list(TRANSPORT_CASES))
def test_oracle_transport_runs_match_reference(name, transport_ref):
    m = TRANSPORT_CASES[name]()
    o = Oracle(m)
    con = transport_ref[f"{name}_con"]
    assert (transport_ref[f"{name}_attempts"] == 1).all()
    # wet decks: the same arithmetic; wet/dry basins: the flow's own 1e-13 differences, carried
    tol = 1e-12 if name in ("channel", "outflow", "salt") else 1e-9
    for k in range(con.shape[0]):
        st = o.step(dt=transport_ref[f"{name}_dt"][k], t=transport_ref[f"{name}_t"][k])
        assert st["status"] == 0
        sts = o.transport_step()
        assert all(s["status"] == 0 for s in sts) and len(sts) == len(m.constituents)
        for j in range(len(m.constituents)):
            assert relerr(o.get_conc(j), con[k, j]) <= tol, (name, k, j)


def test_uniform_concentration_stays_uniform(transport_ref):
    """The reference's angle_salt check: |c - 17.5| <= 1e-6 after every step, in the reference's
    own run and in the oracle's."""
    assert np.abs(transport_ref["salt_con"] - 17.5).max() <= 1e-6
    o = Oracle(meshgen.salt_transport())
    for _ in range(6):
        assert o.step()["status"] == 0
        assert o.transport_step()[0]["status"] == 0
        assert np.abs(o.get_conc(0) - 17.5).max() <= 1e-6


def test_oracle_rejects_held_concentration_on_an_edge_string():
    """DB TRN on an edge string: the reference's boundary residual would read the string's unset
    NB TRN series (fe_2d_transport_boundary_resid.c:186-199)."""
    m = meshgen.channel_transport(nsteps=2, nx=10, ny=2)
    con = m.constituents[0]
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[0.5], node_bc={1: next(iter(con.node_bc.values()))})]
    assert m.transport_tables()[2][0, 1] == BCT_DIR
    with pytest.raises(ValueError):
        Oracle(m)


def test_oracle_transport_error_indicator_matches_reference():
    """The adaption error indicator of a model with constituents: the flow's (ssw_2d_calculate_
    elem_error), then the constituents' folded in (scon_calculate_elem2d_error), as fe_main calls
    them (src/fe/fe_main.c:625-628); element values and each constituent's nodal values after every
    step within 1e-9 of the reference's (the states' own differences)."""
    import os
    from conftest import GOLDEN
    from golden.make_golden import trnerr_model
    ref = dict(np.load(os.path.join(GOLDEN, "trnerr_ref.npz")))
    m = trnerr_model()
    assert str(ref["fingerprint"]) == fingerprint(m)
    o = Oracle(m)
    srt = np.full(len(m.materials), 100.0)                       # MP SRT of the deck writer
    trt = np.array([[c.refine_tol] * len(m.materials) for c in m.constituents])
    for k in range(1, 5):
        assert o.step()["status"] == 0
        assert all(s["status"] == 0 for s in o.transport_step())
        ee, _ = o.elem_error(srt)
        ee2, cerr = o.trn_elem_error(trt, ee)
        assert (ee2 > ee).sum() > len(ee) // 2 and (ee2 == ee).sum() > 0   # both indicators decide some
        assert relerr(ee2, ref[f"step{k}_elem_error"]) <= 1e-9
        for j in range(2):
            assert relerr(cerr[j], ref[f"step{k}_con_error"][j]) <= 1e-9

"""The CPU oracle against fixtures produced by the reference executable itself."""
import os

import numpy as np
import pytest

from golden.make_golden import fingerprint
from helpers import basin_model, channel_model, field_errors, fields, set_load_state
from conftest import GOLDEN, relerr
from oracle.oracle import Oracle


def test_fixture_models_are_current(channel_ref, basin_ref):
    assert str(channel_ref["fingerprint"]) == fingerprint(channel_model())
    assert str(basin_ref["fingerprint"]) == fingerprint(basin_model())


@pytest.mark.parametrize("case", ["channel", "basin"])
def test_oracle_residual_and_jacobian_match_reference(case, channel_ref, basin_ref):
    model, ref = (channel_model(), channel_ref) if case == "channel" else (basin_model(), basin_ref)
    o = Oracle(model)
    set_load_state(o, model, ref)
    o.resid()
    val, r = o.load()
    rp, col = o.pattern()
    assert np.array_equal(rp, ref["load0_rowptr"]) and np.array_equal(col, ref["load0_col"])
    # residual: same arithmetic as the reference up to the summation round-off
    assert relerr(r, ref["load0_resid"]) <= 1e-13
    # Jacobian: central differences amplify residual round-off by 1/eps ~ 1e8
    assert relerr(val, ref["load0_val"]) <= 1e-7
    if case == "channel":
        assert relerr(val, ref["load0_val"]) == 0.0 and relerr(r, ref["load0_resid"]) == 0.0


def test_oracle_channel_run_matches_reference(channel_ref):
    m = channel_model()
    o = Oracle(m)
    for k in range(20):
        st = o.step(dt=channel_ref["dt"][k], t=channel_ref["t"][k])
        assert st["status"] == 0
        assert st["newton_its"] == channel_ref["newton_its"][k]
        if k + 1 in (1, 5, 10, 20):
            got = fields(*o.get_state(0))
            exp = fields(channel_ref[f"step{k+1}_h"], channel_ref[f"step{k+1}_u"], channel_ref[f"step{k+1}_v"])
            for f, e in field_errors(got, exp).items():
                assert e <= 1e-10, (k, f, e)


def test_oracle_basin_run_matches_reference(basin_ref):
    m = basin_model()
    o = Oracle(m)
    for k in range(8):
        st = o.step(dt=basin_ref["dt"][k], t=basin_ref["t"][k])
        assert st["status"] == 0
        assert st["newton_its"] == basin_ref["newton_its"][k]
        got = fields(*o.get_state(0))
        exp = fields(basin_ref[f"step{k+1}_h"], basin_ref[f"step{k+1}_u"], basin_ref[f"step{k+1}_v"])
        for f, e in field_errors(got, exp).items():
            assert e <= 1e-10, (k, f, e)
        assert np.array_equal(o.get_wd(), basin_ref[f"step{k+1}_wd"])


def test_oracle_lake_at_rest_stays_at_rest():
    """Flat water surface over a bumpy bed with no inflow: the reference's lake-at-rest
    invariant (src/initio/test_cases.c:288-340) -- velocities stay ~0, surface stays flat."""
    from adhv8_kraken_b200 import meshgen
    m = meshgen.bumpy_basin(400, seed=5, size=1500.0, nsteps=3, dt=20.0, nbins=1, q_start=0.0, q_peak=0.0)
    o = Oracle(m)
    for _ in range(3):
        assert o.step()["status"] == 0
    h, u, v = o.get_state(0)
    wet = h > 0.05
    assert np.abs(u[wet]).max() < 1e-6 and np.abs(v[wet]).max() < 1e-6
    assert np.abs((h + m.z - 2.0)[wet]).max() < 1e-7


@pytest.mark.parametrize("case", ["channel", "basin"])
def test_oracle_grid_mass_matches_reference(case, mass_ref, basin_ref):
    """tl_find_grid_mass_elem2d and the per-step mass flux of tl_find_grid_mass_error_elem2d,
    restated, against the reference's own values after every step (wet/dry clipped mass with
    the negative-depth correction; boundary flux with the reference's edge length quirk)."""
    from adhv8_kraken_b200 import meshgen
    m = meshgen.channel(nsteps=6) if case == "channel" else basin_model()
    assert str(mass_ref[f"{case}_fingerprint"]) == fingerprint(m)
    o = Oracle(m)
    mass0 = o.grid_mass(0)
    assert relerr(mass0, mass_ref[f"{case}_mass0"][0]) <= 1e-14
    acc = 0.0
    for k, dt in enumerate(mass_ref[f"{case}_dt"], 1):
        src = mass_ref if case == "channel" else basin_ref
        pre = "channel_step" if case == "channel" else "step"
        o.set_state(0, src[f"{pre}{k}_h"], src[f"{pre}{k}_u"], src[f"{pre}{k}_v"])
        mass = o.grid_mass(0)
        acc += o.mass_flux(dt)
        err = abs(mass - acc - mass0)
        assert relerr(mass, mass_ref[f"{case}_mass"][k - 1]) <= 1e-14, k
        assert abs(acc - mass_ref[f"{case}_mass_flux_total"][k - 1]) <= 1e-13 * mass0, k
        assert abs(err - mass_ref[f"{case}_mass_error"][k - 1]) <= 1e-13 * mass0, k


@pytest.mark.parametrize("case", ["ovh", "outflow", "terms", "rain", "obstacle", "combined"])
def test_oracle_boundary_variants_match_reference(case):
    """NB OVH inflow (elevation + velocity, fe_sw2_boundary_resid.c:398-440 with fe_sw2_1d_hvel),
    a free NB OF outflow edge (:227-240, fe_sw2_1d_implicit_flow), a wet/dry basin with every
    optional body term (temporal alpha, EVS / EEV 1-3 eddy viscosity, Coriolis) and one with a
    water source (NB SOURCE, fe_sw2_body_resid.c:728-754), and interior nodes held by a DB OVH node
    string (values set at fe_sw2_init.c:37-85, rows zeroed at fe_sw2_body_resid.c:1239-1256), and
    all of them at once on the wet/dry basin (with the Dirichlet values imposed on the hot start
    as the reference's reader does, ssw.c:452-545):
    residual and FD Jacobian at the first load, then 6 steps (for the source, also the grid mass
    and the accumulated mass flux)."""
    import os
    from adhv8_kraken_b200 import meshgen
    from conftest import GOLDEN
    ovh_ref = dict(np.load(os.path.join(GOLDEN, f"{case}_ref.npz")))
    m = {"ovh": meshgen.channel_ovh, "outflow": meshgen.channel_outflow,
         "terms": meshgen.basin_all_terms, "rain": meshgen.basin_rain,
         "obstacle": lambda nsteps: meshgen.channel_obstacle(nsteps=nsteps, with_depth=True),
         "combined": meshgen.basin_combined}[case](nsteps=6)
    assert str(ovh_ref["fingerprint"]) == fingerprint(m)
    o = Oracle(m)
    set_load_state(o, m, ovh_ref)
    o.resid()
    val, r = o.load()
    assert relerr(r, ovh_ref["load0_resid"]) <= 1e-13
    assert relerr(val, ovh_ref["load0_val"]) <= 1e-7
    o = Oracle(m)
    mass0, acc = o.grid_mass(0), 0.0
    for k in range(6):
        t, dt = ovh_ref["t"][k], ovh_ref["dt"][k]
        st = o.step(dt=dt, t=t)
        assert st["status"] == 0 and st["newton_its"] == ovh_ref["newton_its"][k]
        got = fields(*o.get_state(0))
        exp = fields(ovh_ref[f"step{k+1}_h"], ovh_ref[f"step{k+1}_u"], ovh_ref[f"step{k+1}_v"])
        for f, e in field_errors(got, exp).items():
            assert e <= 1e-10, (k, f, e)
        if "mass" in ovh_ref:   # sources count in the mass flux at the step's series values
            acc += o.mass_flux(dt, m.series_values(t, t + dt))
            assert relerr(o.grid_mass(0), ovh_ref["mass"][k]) <= 1e-12, k
            assert abs(acc - ovh_ref["mass_flux_total"][k]) <= 1e-12 * mass0, k


def test_oracle_transport_side_output_matches_reference(basin_ref):
    """elem_rhs_dacont_extra_terms (fe_sw2_body_resid.c:353-355, :400, :1214: the continuity
    parts of shock capturing and SUPG kept per element vertex for transport) after steps of the
    wet/dry basin, against the reference's own array."""
    import os
    from conftest import GOLDEN
    ref = dict(np.load(os.path.join(GOLDEN, "dacont_ref.npz")))
    m = basin_model()
    assert str(ref["fingerprint"]) == fingerprint(m)
    o = Oracle(m)
    for k in range(8):
        assert o.step(dt=basin_ref["dt"][k], t=basin_ref["t"][k])["status"] == 0
        if k + 1 in (1, 4, 8):
            assert relerr(o.dacont(), ref[f"step{k+1}_dacont"]) <= 1e-10, k


@pytest.mark.parametrize("what", ["lid", "bad_string"])
def test_oracle_rejects_unsupported_node_strings(what):
    """A node string with a lid (BCT_LID_*, pressure under a lid in fe_sw2_body_resid.c:154-177,
    not built) or a string id out of range is refused at creation, not ignored."""
    import dataclasses
    from adhv8_kraken_b200 import capi, meshgen
    m = meshgen.channel_obstacle(nsteps=2, with_depth=True)
    if what == "lid":
        strings = list(m.strings)
        strings[-1] = dataclasses.replace(strings[-1], bc_flag=capi.SW2GPU_BCT_LID_DFT)
        m = dataclasses.replace(m, strings=strings)
    else:
        ns = m.node_string.copy()
        ns[ns >= 0] = len(m.strings)
        m = dataclasses.replace(m, node_string=ns)
    with pytest.raises(ValueError):
        Oracle(m)


def _errind_states(basin_ref, k):
    m = basin_model()
    h0, u0, v0 = m.initial_state()
    prev = (h0, u0, v0) if k == 1 else tuple(basin_ref[f"step{k-1}_{f}"] for f in "huv")
    cur = tuple(basin_ref[f"step{k}_{f}"] for f in "huv")
    return m, cur, prev, basin_ref[f"step{k}_wd"]


@pytest.mark.parametrize("k", [1, 4, 8])
def test_oracle_error_indicator_matches_reference(basin_ref, k):
    """The adaption error indicator (ssw_2d_calculate_elem_error) of the oracle against the
    reference's own grid->elem_error and nodal error after basin steps 1, 4 and 8, from the
    reference's states: within 1e-14 relative (a few ulps: on this Delaunay mesh the shape
    gradients differ from the reference's by round-off, as the residual pin shows)."""
    ref = dict(np.load(os.path.join(GOLDEN, "errind_ref.npz")))
    m, cur, prev, wd = _errind_states(basin_ref, k)
    o = Oracle(m)
    o.set_state(0, *cur)
    o.set_state(1, *prev)
    o.set_dt(m.dt, m.series_values(0.0, m.dt))
    o.set_wd(wd)
    ee, ne = o.elem_error(np.full(len(m.materials), 100.0))   # MP SRT 100 in every generated deck
    assert relerr(ee, ref[f"step{k}_elem_error"]) <= 1e-14
    assert relerr(ne, ref[f"step{k}_node_error"]) <= 1e-14
    assert np.array_equal(ee == 0.5, ref[f"step{k}_elem_error"] == 0.5)   # the wet/dry elements held

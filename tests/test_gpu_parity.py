"""GPU parity: the B200 library through its C ABI against the oracle and the
reference fixtures.  Tolerances (relative to the field's max magnitude):
residual 1e-12, Jacobian 1e-7 (central differences amplify round-off by ~1e8),
time-stepped state 1e-10 per step (h, uh, vh), Newton iterations within +-1."""
import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.sw2 import SW2Error, SW2GPU, run
from conftest import relerr
from helpers import basin_model, channel_model, field_errors, fields, scale_model, set_load_state
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["channel", "basin"])
def test_residual_and_jacobian_match_reference(case, channel_ref, basin_ref):
    model, ref = (channel_model(), channel_ref) if case == "channel" else (basin_model(), basin_ref)
    g = SW2GPU(model)
    set_load_state(g, model, ref)
    g.resid()
    rp, col, val, r = g.load()
    assert np.array_equal(rp, ref["load0_rowptr"]) and np.array_equal(col, ref["load0_col"])
    assert relerr(r, ref["load0_resid"]) <= 1e-12
    assert relerr(val, ref["load0_val"]) <= 1e-7


def test_residual_and_jacobian_match_oracle_on_random_wet_dry_states():
    model = basin_model()
    rng = np.random.default_rng(3)
    for trial in range(3):
        h = model.h0 + rng.normal(0, 0.05, model.nnodes)
        u = rng.normal(0, 0.2, model.nnodes)
        v = rng.normal(0, 0.2, model.nnodes)
        ho = model.h0 + rng.normal(0, 0.05, model.nnodes)
        g, o = SW2GPU(model), Oracle(model)
        for s in (g, o):
            s.set_state(0, h, u, v)
            s.set_state(1, ho, 0.5 * u, 0.5 * v)
            s.set_state(2, ho, 0.25 * u, 0.25 * v)
            s.set_dt(5.0, model.series_values(0.0, 5.0))
        wd = o.wdflag()
        g.set_wd(wd)
        assert (wd > 0).sum() > 50
        rg, ro = g.resid(), o.resid()
        assert relerr(rg, ro) <= 1e-12, trial
        _, _, vg, rg2 = g.load()
        vo, ro2 = o.load()
        assert relerr(rg2, ro2) <= 1e-12
        assert relerr(vg.reshape(-1), vo.reshape(-1)) <= 1e-7
        hg, ug, vvg = g.get_state(0)
        ho_, uo_, vo_ = o.get_state(0)
        assert np.array_equal(ug, uo_) and np.array_equal(vvg, vo_)   # dry-node velocity zeroing


def test_linear_solve_matches_direct_solve(channel_ref):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    model = channel_model()
    g = SW2GPU(model, lin_rtol=1e-10, lin_atol=0.0)
    V = model.nnodes
    A = sp.bsr_matrix((channel_ref["load0_val"], channel_ref["load0_col"], channel_ref["load0_rowptr"]),
                      shape=(3 * V, 3 * V)).tocsc()
    b = channel_ref["load0_resid"]
    x, its, rc = g.linear_solve(channel_ref["load0_val"], b)
    assert rc == 0 and its > 0
    assert relerr(x, spla.spsolve(A, b)) <= 1e-7


def test_band_linear_solve_is_the_exact_solve(channel_ref):
    """SW2GPU_PREC_BAND factors the scaled system exactly: its solution is the direct solve's to
    round-off (the reference's OP BLK 1 profile LU gives the same), one reported iteration."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    model = channel_model()
    g = SW2GPU(model, precond=capi.SW2GPU_PREC_BAND)
    V = model.nnodes
    A = sp.bsr_matrix((channel_ref["load0_val"], channel_ref["load0_col"], channel_ref["load0_rowptr"]),
                      shape=(3 * V, 3 * V)).tocsc()
    b = channel_ref["load0_resid"]
    x, its, rc = g.linear_solve(channel_ref["load0_val"], b)
    assert rc == 0 and its == 1
    assert relerr(x, spla.spsolve(A, b)) <= 1e-10


def test_band_solve_rejects_mixed_precision():
    with pytest.raises(SW2Error):
        SW2GPU(channel_model(), precision=capi.SW2GPU_MIXED, precond=capi.SW2GPU_PREC_BAND)


def test_band_runs_match_reference(channel_ref, basin_ref):
    """Whole time steps with the exact banded solve follow the reference like the Krylov path."""
    _run_against(channel_model(), channel_ref, 20, (1, 5, 10, 20), precond=capi.SW2GPU_PREC_BAND)
    _run_against(basin_model(), basin_ref, 8, range(1, 9), wd=True, precond=capi.SW2GPU_PREC_BAND)


def test_dilu_linear_solve_matches_direct_solve(channel_ref):
    """Block D-ILU BiCGSTAB (SW2GPU_PREC_DILU) solves the reference's load to the direct solve."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    model = channel_model()
    g = SW2GPU(model, precond=capi.SW2GPU_PREC_DILU, lin_rtol=1e-10, lin_atol=0.0)
    V = model.nnodes
    A = sp.bsr_matrix((channel_ref["load0_val"], channel_ref["load0_col"], channel_ref["load0_rowptr"]),
                      shape=(3 * V, 3 * V)).tocsc()
    b = channel_ref["load0_resid"]
    x, its, rc = g.linear_solve(channel_ref["load0_val"], b)
    assert rc == 0 and its > 0
    assert relerr(x, spla.spsolve(A, b)) <= 1e-7


@pytest.mark.parametrize("precision,tol", [(capi.SW2GPU_FP64, 1e-10), (capi.SW2GPU_MIXED, 1e-8)])
def test_dilu_runs_match_reference(channel_ref, basin_ref, scale_ref, precision, tol):
    """Whole time steps with block D-ILU BiCGSTAB against the reference: the channel, the wet/dry
    basin and the benchmark generator's basin, at the bounds of the block-Jacobi path."""
    kw = dict(precision=precision, tol=tol, precond=capi.SW2GPU_PREC_DILU)
    _run_against(channel_model(), channel_ref, 20, (1, 5, 10, 20), **kw)
    _run_against(basin_model(), basin_ref, 8, range(1, 9), wd=precision == capi.SW2GPU_FP64, **kw)
    _run_against(_scale_model_checked(scale_ref), scale_ref, 10, range(1, 11), wd=precision == capi.SW2GPU_FP64, **kw)


def _run_against(model, ref, nsteps, check_every, precision=capi.SW2GPU_FP64, tol=1e-10, wd=False, **kw):
    g = SW2GPU(model, precision=precision, **kw)
    worst = 0.0
    for k in range(nsteps):
        st = g.step(dt=ref["dt"][k], t=ref["t"][k])
        assert st["status"] == 0, st
        assert abs(st["newton_its"] - int(ref["newton_its"][k])) <= 1, (k, st["newton_its"], ref["newton_its"][k])
        if (k + 1) in check_every:
            got = fields(*g.get_state(0))
            exp = fields(ref[f"step{k+1}_h"], ref[f"step{k+1}_u"], ref[f"step{k+1}_v"])
            for f, e in field_errors(got, exp).items():
                worst = max(worst, e)
                assert e <= tol, (k, f, e)
            if wd:
                assert np.array_equal(g.get_wd(), ref[f"step{k+1}_wd"])
    return worst


def test_channel_run_matches_reference(channel_ref):
    _run_against(channel_model(), channel_ref, 20, (1, 5, 10, 20))


def test_basin_run_matches_reference(basin_ref):
    _run_against(basin_model(), basin_ref, 8, range(1, 9), wd=True)


def test_mixed_precision_channel_within_1e8(channel_ref):
    _run_against(channel_model(), channel_ref, 20, (1, 5, 10, 20), precision=capi.SW2GPU_MIXED, tol=1e-8)


@pytest.fixture(scope="module")
def scale_ref():
    import os
    from conftest import GOLDEN
    return dict(np.load(os.path.join(GOLDEN, "scale_ref.npz")))


def _scale_model_checked(ref):
    from golden.make_golden import fingerprint
    m = scale_model()
    assert str(ref["fingerprint"]) == fingerprint(m)   # the generator still makes the recorded problem
    return m


def test_bench_generator_basin_fp64_matches_reference_every_step(scale_ref):
    """The benchmark's own generator (seed 2024, 32 Manning bins, 40 bumps with dry tops, inflow
    ramp) at ~20k triangles against the reference over 10 steps: plain FP64 within 1e-10 per
    step in depth and unit discharge, Newton iterations within +-1, identical wet/dry flags."""
    m = _scale_model_checked(scale_ref)
    worst = _run_against(m, scale_ref, 10, range(1, 11), wd=True)
    assert worst <= 1e-10


def test_bench_generator_basin_mixed_matches_reference_every_step(scale_ref):
    """The mixed path (FP32 Jacobian storage, SpMV and preconditioner inside the FP64 Newton
    loop) on the same problem, against the reference's states (not against the GPU's own FP64
    run): within 1e-8 per step, Newton iterations within +-1."""
    m = _scale_model_checked(scale_ref)
    _run_against(m, scale_ref, 10, range(1, 11), precision=capi.SW2GPU_MIXED, tol=1e-8)


def test_reruns_are_bitwise_identical():
    model = basin_model()
    outs = []
    for _ in range(2):
        g = SW2GPU(model)
        for _ in range(3):
            assert g.step()["status"] == 0
        outs.append(np.concatenate(g.get_state(0)))
    assert np.array_equal(outs[0], outs[1])


VARIANTS = {"ovh": meshgen.channel_ovh, "outflow": meshgen.channel_outflow, "terms": meshgen.basin_all_terms,
            "rain": meshgen.basin_rain,
            "obstacle": lambda nsteps: meshgen.channel_obstacle(nsteps=nsteps, with_depth=True),
            "combined": meshgen.basin_combined}


@pytest.mark.parametrize("case", sorted(VARIANTS))
def test_boundary_and_term_variants_match_reference(case):
    """The reference fixtures of an inflow given as water elevation and velocity (NB OVH), a free
    outflow edge (NB OF), a wet/dry basin with every optional body term (temporal alpha, EVS /
    EEV 1-3 eddy viscosity, Coriolis), a water source (NB SOURCE) and interior nodes held by a
    DB OVH string, and all of them at once on the wet/dry basin: residual and Jacobian at the
    first load, then 6 steps, each state within 1e-10 and Newton iterations within +-1."""
    import os
    from conftest import GOLDEN
    from golden.make_golden import fingerprint
    ref = dict(np.load(os.path.join(GOLDEN, f"{case}_ref.npz")))
    model = VARIANTS[case](nsteps=6)
    assert str(ref["fingerprint"]) == fingerprint(model)
    g = SW2GPU(model)
    set_load_state(g, model, ref)
    g.resid()
    rp, col, val, r = g.load()
    assert np.array_equal(rp, ref["load0_rowptr"]) and np.array_equal(col, ref["load0_col"])
    assert relerr(r, ref["load0_resid"]) <= 1e-12
    assert relerr(val, ref["load0_val"]) <= 1e-7
    _run_against(model, ref, 6, range(1, 7))


@pytest.mark.parametrize("case", ["channel", "basin", "rain", "combined"])
def test_mass_balance_on_device_matches_reference(case, mass_ref, basin_ref):
    """The device's grid mass (tl_find_grid_mass_elem2d) and per-step mass flux (sources minus
    boundary outflow, tl_find_grid_mass_error_elem2d) at the reference's own state after every
    step, against the reference's values: the channel (inflow and tailwater edges), the wet/dry
    basin (dry corners), the basin with rain, and the all-features basin (rain, NB OVH and NB OF
    edges, Dirichlet nodes).  The device adds its terms in a fixed tree
    order, the reference in element order: 1e-12 relative to the initial mass."""
    import os
    from conftest import GOLDEN
    from golden.make_golden import fingerprint
    if case in ("rain", "combined"):
        model = (meshgen.basin_rain if case == "rain" else meshgen.basin_combined)(nsteps=6)
        ref = dict(np.load(os.path.join(GOLDEN, f"{case}_ref.npz")))
        assert str(ref["fingerprint"]) == fingerprint(model)
        dts, masses, totals, pre, src = ref["dt"], ref["mass"], ref["mass_flux_total"], "step", ref
        ref_mass0 = ref["mass0"][0]
    else:
        model = meshgen.channel(nsteps=6) if case == "channel" else basin_model()
        assert str(mass_ref[f"{case}_fingerprint"]) == fingerprint(model)
        dts, masses, totals = (mass_ref[f"{case}_{k}"] for k in ("dt", "mass", "mass_flux_total"))
        pre, src = ("channel_step", mass_ref) if case == "channel" else ("step", basin_ref)
        ref_mass0 = mass_ref[f"{case}_mass0"][0]
    g = SW2GPU(model)
    mass0 = g.grid_mass(0)
    assert relerr(mass0, ref_mass0) <= 1e-12
    t, acc = model.t0, 0.0
    for k, dt in enumerate(dts, 1):
        g.set_state(0, src[f"{pre}{k}_h"], src[f"{pre}{k}_u"], src[f"{pre}{k}_v"])
        g.set_dt(dt, model.series_values(t, t + dt))
        t += dt
        acc += g.mass_flux()
        assert relerr(g.grid_mass(0), masses[k - 1]) <= 1e-12, k
        assert abs(acc - totals[k - 1]) <= 1e-12 * mass0, k
    assert g.grid_mass(0) == g.grid_mass(0)   # fixed-order reduction: the same bits every call


def test_transport_side_output_matches_reference(basin_ref):
    """elem_rhs_dacont_extra_terms (the continuity parts of shock capturing and SUPG per element
    vertex, kept for transport) after steps 1, 4 and 8 of the wet/dry basin, against the
    reference's own array.  The output is built from depth gradients and amplifies differences of
    the state by up to ~1e3 (measured on the oracle with seeded noise), and the device holds the
    state within 1e-10 of the reference's: 1e-7 relative to the array's largest magnitude (a
    missing or wrong term is an O(1) error)."""
    import os
    from conftest import GOLDEN
    from golden.make_golden import fingerprint
    ref = dict(np.load(os.path.join(GOLDEN, "dacont_ref.npz")))
    model = basin_model()
    assert str(ref["fingerprint"]) == fingerprint(model)
    g = SW2GPU(model)
    with pytest.raises(SW2Error):
        g.dacont()                      # off until asked for
    g.set_dacont(True)
    for k in range(8):
        assert g.step(dt=basin_ref["dt"][k], t=basin_ref["t"][k])["status"] == 0
        if k + 1 in (1, 4, 8):
            got = g.dacont().reshape(3, model.nelems2d)
            assert relerr(got, ref[f"step{k+1}_dacont"]) <= 1e-7, k


@pytest.mark.parametrize("k", [1, 4, 8])
def test_device_error_indicator_matches_oracle_and_reference(basin_ref, k):
    """The adaption error indicator computed on the device from the reference's states after basin
    steps 1, 4 and 8: bit-identical to the oracle, and within 1e-14 of the reference's own
    grid->elem_error and nodal error (shape-gradient round-off, as for the residual)."""
    import os
    from conftest import GOLDEN
    from oracle.oracle import Oracle
    ref = dict(np.load(os.path.join(GOLDEN, "errind_ref.npz")))
    m = basin_model()
    h0, u0, v0 = m.initial_state()
    prev = (h0, u0, v0) if k == 1 else tuple(basin_ref[f"step{k-1}_{f}"] for f in "huv")
    cur = tuple(basin_ref[f"step{k}_{f}"] for f in "huv")
    tol = np.full(len(m.materials), 100.0)
    out = []
    for s in (SW2GPU(m), Oracle(m)):
        s.set_state(0, *cur)
        s.set_state(1, *prev)
        s.set_dt(m.dt, m.series_values(0.0, m.dt))
        s.set_wd(basin_ref[f"step{k}_wd"])
        out.append(s.elem_error(tol))
    (eg, ng), (eo, no) = out
    assert np.array_equal(eg, eo) and np.array_equal(ng, no)
    assert relerr(eg, ref[f"step{k}_elem_error"]) <= 1e-14
    assert relerr(ng, ref[f"step{k}_node_error"]) <= 1e-14


def test_mass_reduced_inside_the_step_equals_the_on_demand_diagnostics():
    """With mass tracking on, every accepted step reduces the grid mass and the step's mass flux
    inside the step; the values are bitwise those of sw2gpu_grid_mass / sw2gpu_mass_flux called
    right after the step (the reference's SOUT MERROR path), on the rain basin with a source."""
    m = meshgen.basin_rain(nsteps=4)
    g = SW2GPU(m)
    g.set_mass_tracking(True)
    with pytest.raises(SW2Error):
        g.step_mass()                 # no accepted step yet
    for _ in range(4):
        assert g.step()["status"] == 0
        mass, flux = g.step_mass()
        assert mass == g.grid_mass(0) and flux == g.mass_flux()
    g.close()


def test_wind_and_wave_stress_residual_and_steps_match_oracle():
    """Wave radiation stress (nodal Sxx, Sxy, Syy) on top of the wind stress on the wet/dry basin:
    the device's element stresses, residual and three steps against the oracle; turning the
    waves off again gives the wind-only residual back bit for bit."""
    m = basin_model()
    rng = np.random.Generator(np.random.PCG64(31))
    nm = len(m.materials)
    flags = np.zeros(nm, np.int32)
    att = np.ones(nm)
    sx, sy = rng.normal(0.0, 0.2, m.nnodes), rng.normal(0.0, 0.2, m.nnodes)
    rads = [rng.normal(0.0, 0.05, m.nnodes) for _ in range(3)]
    g, o = SW2GPU(m), Oracle(m)
    for s in (g, o):
        s.set_wind(flags, att, sx, sy)
        s.set_dt(m.dt, m.series_values(0.0, m.dt))
    o.wdflag()
    g.set_wd(o.get_wd())
    wind_only = g.resid()
    for s in (g, o):
        s.set_waves(*rads)
    assert relerr(g.resid(), o.resid()) <= 1e-12
    g.set_waves(None)
    assert np.array_equal(g.resid(), wind_only)
    g.set_waves(*rads)
    for _ in range(3):
        a, b = g.step(), o.step()
        assert a["status"] == 0 and b["status"] == 0 and abs(a["newton_its"] - b["newton_its"]) <= 1
        errs = field_errors(fields(*g.get_state(0)), fields(*o.get_state(0)))
        assert max(errs.values()) <= 1e-10, errs


def test_wind_stress_residual_and_steps_match_oracle():
    """Wind surface stress (both stress forms, per-material attenuation) on the wet/dry basin:
    the device residual and three steps against the oracle with the same nodal winds."""
    m = basin_model()
    rng = np.random.Generator(np.random.PCG64(29))
    nm = len(m.materials)
    flags = np.array([k % 2 for k in range(nm)], np.int32)
    att = np.linspace(1.0, 0.6, nm)
    sx, sy = rng.normal(0.0, 0.2, m.nnodes), rng.normal(0.0, 0.2, m.nnodes)
    g, o = SW2GPU(m), Oracle(m)
    for s in (g, o):
        s.set_wind(flags, att, sx, sy)
        s.set_dt(m.dt, m.series_values(0.0, m.dt))
    o.wdflag()
    g.set_wd(o.get_wd())
    assert relerr(g.resid(), o.resid()) <= 1e-12
    for _ in range(3):
        a, b = g.step(), o.step()
        assert a["status"] == 0 and b["status"] == 0 and abs(a["newton_its"] - b["newton_its"]) <= 1
        errs = field_errors(fields(*g.get_state(0)), fields(*o.get_state(0)))
        assert max(errs.values()) <= 1e-10, errs

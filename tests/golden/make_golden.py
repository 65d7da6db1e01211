"""Generates the golden fixtures of this directory by running the reference AdH
executable (built from the reference sources by ``oracle/ref/build_ref.py``).

Run in a container where the reference sources are present::

    python oracle/ref/build_ref.py && python tests/golden/make_golden.py

Fixtures (numpy ``.npz``):

* ``channel_ref.npz`` -- the rectangular channel (100 x 20 squares, 4,000 triangles,
  NB VEL inflow 0.5 m^2/s, NB OTW tailwater, dt = 10 s), 20 steps: Newton iterations
  of every step, the state after steps 1, 5, 10, 20, and the state / residual /
  Jacobian (sorted BCSR) at the first fe_sw2_load call.
* ``basin_ref.npz`` -- a seeded Delaunay basin with dry bump tops (wet/dry fronts),
  8 steps: Newton iterations, state and wd flags after every step, and the first
  fe_sw2_load state / residual / Jacobian.
* ``ovh_ref.npz`` -- the channel with its inflow given as NB OVH (elevation + velocity),
  6 steps: Newton iterations, state after every step, and the first fe_sw2_load state /
  residual / Jacobian.
* ``outflow_ref.npz`` -- the channel with a free outflow edge (NB OF) east, 6 steps, recorded
  like ``ovh_ref.npz``.
* ``terms_ref.npz`` -- a wet/dry basin with every optional body term on (temporal alpha, EVS
  and EEV modes 1-3 eddy viscosity, Coriolis), 6 steps, recorded like ``ovh_ref.npz``.
* ``rain_ref.npz`` -- the basin with a water source (NB SOURCE) on one material string, 6 steps,
  recorded like ``ovh_ref.npz`` plus the grid mass diagnostics after every step.
* ``obstacle_ref.npz`` -- the channel with a line of interior nodes held at zero velocity and 1 m
  depth (DB OVH node string), 6 steps, recorded like ``ovh_ref.npz``.
* ``combined_ref.npz`` -- every supported feature at once on the wet/dry basin (all optional body
  terms, rain, NB OVH inflow, NB OF outflow, a DB OVH node group), 6 steps, recorded like
  ``rain_ref.npz``.
* ``dacont_ref.npz`` -- the reference's transport side output elem_rhs_dacont_extra_terms
  (continuity parts of shock capturing and SUPG per element vertex) after steps 1, 4 and 8 of
  the basin run.
* ``scale_ref.npz`` -- the generator of the 1M-triangle benchmark basin (seed 2024, 32 Manning
  bins, 40 bumps with dry tops, inflow ramp 1 -> 5 m^2/s over 30 steps, dt 5 s) at 10k points
  (~20k triangles, the domain scaled to keep the element size), 10 steps: Newton iterations,
  state and wd flags after every step.
* ``errind_ref.npz`` -- the reference's adaption error indicator (ssw_2d_calculate_elem_error,
  src/structs/ssw_2d.c:424-500: grid->elem_error and its nodal average) after steps 1, 4 and 8
  of the basin run, whose states are in ``basin_ref.npz``.
* ``transport_ref.npz`` -- constituent transport after every flow step (fe_transport) on five
  workloads of ``adhv8_kraken_b200.meshgen``: the channel with a held inflow concentration
  (DB TRN) and diffusion, the wet/dry basin with two constituents (NB TRN at the inflow and the
  tailwater, per-material diffusion), the all-terms basin (temporal alpha, EEV diffusion), the
  free-outflow channel and the uniform-17.5 channel of the reference's angle_salt check:
  concentrations after every step, and for the two basins the inputs and results of the first
  two transport Jacobian builds.
* ``trnerr_ref.npz`` -- the adaption error indicator of the two-constituent basin (MP TRT 0.05 and
  2.0) after each of 4 steps: grid->elem_error with the constituents' indicator folded in after
  the flow's, and each constituent's nodal indicator con[k].error.
* ``mass_ref.npz`` -- the reference's grid mass diagnostics (src/tools/tl_grid_mass.c) after
  every step of 6 channel steps and of the 8 basin steps: initial and current mass, mass error
  and accumulated mass flux, with the channel's state after every step (the basin's states are
  in ``basin_ref.npz``).

Each fixture stores a fingerprint of the generated model so a generator change is
detected instead of silently comparing different problems.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from adhv8_kraken_b200 import meshgen  # noqa: E402
from oracle.ref_run import run_reference  # noqa: E402


def fingerprint(m) -> str:
    h = hashlib.sha256()
    for a in (m.x, m.y, m.z, m.tri, m.tri_mat, m.edges, m.edge_string, m.h0, m.u0, m.v0):
        h.update(np.ascontiguousarray(a).tobytes())
    if m.constituents:
        for a in m.transport_tables():
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(np.ascontiguousarray(m.node_string).tobytes())
    return h.hexdigest()


def pattern(m):
    """Sorted BCSR pattern of the model (element and edge node pairs)."""
    rows = [set() for _ in range(m.nnodes)]
    for t in m.tri:
        for a in t:
            rows[a].update(int(b) for b in t)
    for e in m.edges:
        for a in e:
            rows[a].update(int(b) for b in e)
    rp = np.zeros(m.nnodes + 1, np.int32)
    cols = []
    for i, r in enumerate(rows):
        c = sorted(r)
        cols.extend(c)
        rp[i + 1] = rp[i] + len(c)
    return rp, np.array(cols, np.int32)


def ref_jacobian_to_bcsr(m, L):
    rp, col = pattern(m)
    V = m.nnodes
    val = np.zeros((len(col), 3, 3))
    diag = L["diag"].reshape(V, 3, 3)
    vals = L["vals"].reshape(-1, 3, 3)
    k = 0
    for i in range(V):
        lookup = {int(c): rp[i] + n for n, c in enumerate(col[rp[i]:rp[i + 1]])}
        val[lookup[i]] = diag[i]
        for _ in range(L["rowsz"][i]):
            val[lookup[int(L["cols"][k])]] = vals[k]
            k += 1
    return rp, col, val


def load_record(m, L, prefix):
    rp, col, val = ref_jacobian_to_bcsr(m, L)
    out = {}
    for key in ("h", "u", "v", "h1", "u1", "v1", "h2", "u2", "v2", "resid"):
        out[f"{prefix}_{key}"] = L[key]
    out[f"{prefix}_wd"] = L["wd"]
    out[f"{prefix}_t"] = np.array([L["t"], L["dt"]])
    out[f"{prefix}_rowptr"] = rp
    out[f"{prefix}_col"] = col
    out[f"{prefix}_val"] = val
    return out


def channel():
    m = meshgen.channel()
    ref = run_reference(m, nsteps=20, loads=1)
    out = {"fingerprint": np.array(fingerprint(m)),
           "newton_its": np.array([s["newton_its"] for s in ref["steps"]], np.int32),
           "t": np.array([s["t"] for s in ref["steps"]]), "dt": np.array([s["dt"] for s in ref["steps"]])}
    for k in (1, 5, 10, 20):
        s = ref["steps"][k - 1]
        out[f"step{k}_h"], out[f"step{k}_u"], out[f"step{k}_v"] = s["h"], s["u"], s["v"]
    out.update(load_record(m, ref["loads"][0], "load0"))
    np.savez_compressed(os.path.join(HERE, "channel_ref.npz"), **out)


def basin_model():
    return meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=8, dt=5.0, nbins=3, name="basin")


def basin():
    m = basin_model()
    ref = run_reference(m, nsteps=8, loads=1)
    out = {"fingerprint": np.array(fingerprint(m)),
           "newton_its": np.array([s["newton_its"] for s in ref["steps"]], np.int32),
           "t": np.array([s["t"] for s in ref["steps"]]), "dt": np.array([s["dt"] for s in ref["steps"]])}
    for k, s in enumerate(ref["steps"], 1):
        out[f"step{k}_h"], out[f"step{k}_u"], out[f"step{k}_v"] = s["h"], s["u"], s["v"]
        out[f"step{k}_wd"] = s["wd"]
    out.update(load_record(m, ref["loads"][0], "load0"))
    np.savez_compressed(os.path.join(HERE, "basin_ref.npz"), **out)


def ovh(m=None, fname="ovh_ref.npz", mass=False):
    m = meshgen.channel_ovh(nsteps=6) if m is None else m
    ref = run_reference(m, nsteps=6, loads=1, mass=mass)
    out = {"fingerprint": np.array(fingerprint(m)),
           "newton_its": np.array([s["newton_its"] for s in ref["steps"]], np.int32),
           "t": np.array([s["t"] for s in ref["steps"]]), "dt": np.array([s["dt"] for s in ref["steps"]])}
    for k, s in enumerate(ref["steps"], 1):
        out[f"step{k}_h"], out[f"step{k}_u"], out[f"step{k}_v"] = s["h"], s["u"], s["v"]
    out.update(load_record(m, ref["loads"][0], "load0"))
    if mass:
        for key in ("mass0", "mass", "mass_error", "mass_flux_total"):
            out[key] = np.array([s[key] for s in ref["steps"]])
    np.savez_compressed(os.path.join(HERE, fname), **out)


def scale_model(nsteps=10):
    """The benchmark basin's generator at 10k points (bench.py scales the domain with the
    square root of the point count, so the element size is that of the 1M-triangle mesh)."""
    import math
    points = 10000
    return meshgen.bumpy_basin(points, seed=2024, size=20000.0 * math.sqrt(points / 5e5), nsteps=nsteps, dt=5.0,
                               name="scale")


def scale():
    m = scale_model()
    ref = run_reference(m, nsteps=10)
    out = {"fingerprint": np.array(fingerprint(m)),
           "newton_its": np.array([s["newton_its"] for s in ref["steps"]], np.int32),
           "attempts": np.array([s["attempts"] for s in ref["steps"]], np.int32),
           "t": np.array([s["t"] for s in ref["steps"]]), "dt": np.array([s["dt"] for s in ref["steps"]]),
           "op_blk": np.array(m.params.nblock, np.int32)}
    for k, s in enumerate(ref["steps"], 1):
        out[f"step{k}_h"], out[f"step{k}_u"], out[f"step{k}_v"] = s["h"], s["u"], s["v"]
        out[f"step{k}_wd"] = s["wd"].astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "scale_ref.npz"), **out)


def errind():
    m = basin_model()
    ref = run_reference(m, nsteps=8, error=True)
    out = {"fingerprint": np.array(fingerprint(m))}
    for k in (1, 4, 8):
        out[f"step{k}_elem_error"] = ref["steps"][k - 1]["elem_error"]
        out[f"step{k}_node_error"] = ref["steps"][k - 1]["node_error"]
        out[f"step{k}_h"] = ref["steps"][k - 1]["h"]
    np.savez_compressed(os.path.join(HERE, "errind_ref.npz"), **out)


def dacont():
    m = basin_model()
    ref = run_reference(m, nsteps=8, dacont=True)
    out = {"fingerprint": np.array(fingerprint(m))}
    for k in (1, 4, 8):
        out[f"step{k}_dacont"] = ref["steps"][k - 1]["dacont"]
    np.savez_compressed(os.path.join(HERE, "dacont_ref.npz"), **out)


def mass():
    out = {}
    for name, m, n in (("channel", meshgen.channel(nsteps=6), 6), ("basin", basin_model(), 8)):
        ref = run_reference(m, nsteps=n, mass=True)
        out[f"{name}_fingerprint"] = np.array(fingerprint(m))
        out[f"{name}_dt"] = np.array([s["dt"] for s in ref["steps"]])
        for key in ("mass0", "mass", "mass_error", "mass_flux_total"):
            out[f"{name}_{key}"] = np.array([s[key] for s in ref["steps"]])
        if name == "channel":
            for k, s in enumerate(ref["steps"], 1):
                out[f"channel_step{k}_h"], out[f"channel_step{k}_u"], out[f"channel_step{k}_v"] = s["h"], s["u"], s["v"]
    np.savez_compressed(os.path.join(HERE, "mass_ref.npz"), **out)


TRANSPORT_CASES = {"channel": lambda: meshgen.channel_transport(nsteps=6),
                   "basin": lambda: meshgen.basin_transport(nsteps=8),
                   "terms": lambda: meshgen.terms_transport(nsteps=6),
                   "outflow": lambda: meshgen.outflow_transport(nsteps=6),
                   "salt": lambda: meshgen.salt_transport(nsteps=6)}


def transport():
    """Constituent transport after every flow step (fe_transport): each case's concentrations
    after every step, and for the wet/dry basins the inputs and results of the first two
    transport Jacobian builds (fe_transport_load): the three concentration and flow levels,
    wd_flag, the flow's side output, bc_mask, the residual and the scalar Jacobian over the
    sorted pattern."""
    out = {}
    for name, make in TRANSPORT_CASES.items():
        m = make()
        nl = 2 if name in ("basin", "terms") else 0
        ref = run_reference(m, tloads=nl)
        out[f"{name}_fingerprint"] = np.array(fingerprint(m))
        out[f"{name}_t"] = np.array([s["t"] for s in ref["steps"]])
        out[f"{name}_dt"] = np.array([s["dt"] for s in ref["steps"]])
        out[f"{name}_attempts"] = np.array([s["attempts"] for s in ref["steps"]], np.int32)
        out[f"{name}_con"] = np.stack([np.stack(s["con"]) for s in ref["steps"]])     # [step, ntrn, V]
        rp, col = pattern(m)
        for q, L in enumerate(ref["tloads"][:nl]):
            p = f"{name}_tload{q}"
            for key in ("c", "c1", "c2", "h", "u", "v", "h1", "u1", "v1", "h2", "u2", "v2", "resid", "dacont"):
                out[f"{p}_{key}"] = L[key]
            out[f"{p}_wd"] = L["wd"]
            out[f"{p}_bcmask"] = (L["bcmask"] == 1).astype(np.int32)
            out[f"{p}_meta"] = np.array([L["itrn"], L["t"], L["dt"]])
            val = np.zeros(len(col))
            k = 0
            for i in range(m.nnodes):
                lookup = {int(c): rp[i] + n for n, c in enumerate(col[rp[i]:rp[i + 1]])}
                val[lookup[i]] = L["diag"][i]
                for _ in range(L["rowsz"][i]):
                    c = int(L["cols"][k])
                    if c >= 0:
                        val[lookup[c]] += L["vals"][k]
                    k += 1
            out[f"{p}_val"] = val
    np.savez_compressed(os.path.join(HERE, "transport_ref.npz"), **out)


def trnerr_model():
    """The two-constituent wet/dry basin with MP TRT 0.05 and 2.0: the constituents set most
    elements' indicator, the flow the rest."""
    m = meshgen.basin_transport(nsteps=4)
    m.constituents[0].refine_tol = 0.05
    m.constituents[1].refine_tol = 2.0
    return m


def trnerr():
    """The adaption error indicator of a model with constituents after every step: grid->elem_error
    (the flow's, then the constituents' folded in, src/fe/fe_main.c:625-628) and each constituent's
    nodal con[k].error (scon_calculate_elem2d_error)."""
    m = trnerr_model()
    ref = run_reference(m, error=True)
    out = {"fingerprint": np.array(fingerprint(m))}
    for k, st in enumerate(ref["steps"], 1):
        out[f"step{k}_elem_error"] = st["elem_error"]
        out[f"step{k}_con_error"] = np.stack(st["con_error"])
    np.savez_compressed(os.path.join(HERE, "trnerr_ref.npz"), **out)


if __name__ == "__main__":
    import sys as _sys
    which = _sys.argv[1:] or ["channel", "basin", "ovh", "outflow", "terms", "rain", "obstacle", "combined", "dacont",
                              "mass", "scale", "errind", "transport", "trnerr"]
    if "channel" in which:
        channel()
    if "basin" in which:
        basin()
    if "ovh" in which:
        ovh()
    if "outflow" in which:
        ovh(meshgen.channel_outflow(nsteps=6), "outflow_ref.npz")
    if "terms" in which:
        ovh(meshgen.basin_all_terms(nsteps=6), "terms_ref.npz")
    if "rain" in which:
        ovh(meshgen.basin_rain(nsteps=6), "rain_ref.npz", mass=True)
    if "obstacle" in which:
        ovh(meshgen.channel_obstacle(nsteps=6, with_depth=True), "obstacle_ref.npz")
    if "combined" in which:
        ovh(meshgen.basin_combined(nsteps=6), "combined_ref.npz", mass=True)
    if "dacont" in which:
        dacont()
    if "mass" in which:
        mass()
    if "scale" in which:
        scale()
    if "errind" in which:
        errind()
    if "transport" in which:
        transport()
    if "trnerr" in which:
        trnerr()
    for f in ("channel_ref.npz", "basin_ref.npz", "ovh_ref.npz", "outflow_ref.npz", "terms_ref.npz", "rain_ref.npz",
              "obstacle_ref.npz", "combined_ref.npz", "dacont_ref.npz", "mass_ref.npz", "scale_ref.npz",
              "errind_ref.npz", "transport_ref.npz", "trnerr_ref.npz"):
        if os.path.exists(os.path.join(HERE, f)):
            print(f, os.path.getsize(os.path.join(HERE, f)))

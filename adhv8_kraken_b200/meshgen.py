"""Seeded synthetic SW2 problems.

The reference publishes no benchmark meshes, so every workload is generated here
from a seed.  Two families:

* :func:`channel` -- the rectangular channel: ``nx x ny`` squares, each split
  into two triangles along the (i,j)-(i+1,j+1) diagonal, bed sloping along +x,
  unit-discharge inflow (``NB VEL``) on the west edge and a tailwater level
  (``NB OTW``) on the east edge.
* :func:`bumpy_basin` -- Delaunay triangulation of seeded uniform points in a
  square, bed = planar slope + Gaussian bumps, flat initial water surface (dry
  bump tops give wet/dry fronts), per-element log-normal Manning n quantised into
  ``nbins`` material classes, inflow hydrograph on the west edge and a tailwater
  level on the east edge.

Nodes are ordered along a Morton (Z-order) curve so that element gathers on the
GPU and the block solver of the reference CPU path both see local data.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .model import (BCT_PRS_NEU, BCT_VEL_NEU, NORMAL, Material, Params, Series,
                    StringSpec, SW2Model)


def _morton_order(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Permutation that sorts points along a 2D Z-order curve (16 bits per axis)."""
    span = max(float(x.max() - x.min()), float(y.max() - y.min()), 1e-30)
    ix = np.clip(((x - x.min()) / span * 65535.0).astype(np.uint64), 0, 65535)
    iy = np.clip(((y - y.min()) / span * 65535.0).astype(np.uint64), 0, 65535)

    def spread(v):
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v

    code = spread(ix) | (spread(iy) << np.uint64(1))
    return np.argsort(code, kind="stable")


def channel(nx: int = 100, ny: int = 20, length: float = 1000.0, width: float = 200.0,
            slope: float = 1e-4, manning: float = 0.025, q_in: float = 0.5, h_out: float = 1.0,
            h0: float = 1.0, dt: float = 10.0, nsteps: int = 20, tol_nonlin: float = 1e-8,
            name: str = "channel") -> SW2Model:
    """Rectangular channel (4,000 triangles and 2,121 nodes at the default 100 x 20).

    Nodes are numbered column by column (y fastest), which keeps the reference's
    profile LU bandwidth at ``3 (ny + 2)``.
    """
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    x = (ii * (length / nx)).ravel().astype(np.float64)
    y = (jj * (width / ny)).ravel().astype(np.float64)
    z = -slope * x
    nid = lambda i, j: i * (ny + 1) + j
    tri = []
    for i in range(nx):
        for j in range(ny):
            a, b, c, d = nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)
            tri.append((a, b, c))
            tri.append((a, c, d))
    tri = np.array(tri, dtype=np.int32)
    west = [(nid(0, j + 1), nid(0, j)) for j in range(ny)]
    east = [(nid(nx, j), nid(nx, j + 1)) for j in range(ny)]
    edges = np.array(west + east, dtype=np.int32)
    strings = [StringSpec("mat", manning_n=manning),
               StringSpec("edge", bc_flag=BCT_VEL_NEU, isigma=0),
               StringSpec("edge", bc_flag=BCT_PRS_NEU, isigma=1)]
    edge_string = np.array([1] * ny + [2] * ny, dtype=np.int32)
    t_end = (nsteps + 10) * dt
    series = [Series(np.array([0.0, t_end]), np.array([q_in, q_in])),
              Series(np.array([0.0, t_end]), np.array([-slope * length + h_out] * 2))]
    V = x.shape[0]
    return SW2Model(x=x, y=y, z=z, tri=tri, tri_mat=np.zeros(tri.shape[0], np.int32),
                    edges=edges, edge_string=edge_string,
                    node_string=np.full(V, NORMAL, np.int32), strings=strings,
                    materials=[Material(evs=(0.0, 0.0, 0.0))], series=series,
                    params=Params(tol_nonlin=tol_nonlin), h0=np.full(V, h0), u0=np.zeros(V),
                    v0=np.zeros(V), dt=dt, nsteps=nsteps, name=name)


def basin_all_terms(nsteps: int = 6) -> SW2Model:
    """A small wet/dry basin with every optional body term on: temporal weight alpha = 0.5
    (OP TEM), and per material EVS eddy viscosity with Coriolis, EEV modes 1 and 2, and EEV
    mode 3 with Coriolis."""
    from .model import Material
    m = bumpy_basin(700, seed=11, size=2000.0, nsteps=nsteps, dt=5.0, nbins=4, name="terms")
    m.params = dataclasses.replace(m.params, tau_temporal=0.5)
    m.materials = [Material(evs=(6.0, 2.0, 1.0), coriolis=30.0), Material(eev_coef=0.4, eev_mode=1),
                   Material(eev_coef=0.4, eev_mode=2), Material(eev_coef=0.4, eev_mode=3, coriolis=-20.0)]
    return m


def basin_rain(nsteps: int = 6, rate: float = 2e-4) -> SW2Model:
    """The small wet/dry basin with a water source (NB SOURCE, `rate` m/s of rain) on its first
    material string."""
    from .model import BCT_WATER_SOURCE
    m = bumpy_basin(700, seed=11, size=2000.0, nsteps=nsteps, dt=5.0, nbins=3, name="rain")
    t_end = (nsteps + 10) * m.dt
    m.series = list(m.series) + [Series(np.array([0.0, t_end]), np.array([rate, rate]))]
    m.strings = list(m.strings)
    m.strings[0] = dataclasses.replace(m.strings[0], bc_flag=BCT_WATER_SOURCE, isigma=len(m.series) - 1)
    return m


def basin_combined(nsteps: int = 6, rate: float = 2e-4, u_in: float = 0.2) -> SW2Model:
    """Every supported feature at once, for interactions: the all-terms wet/dry basin (temporal
    alpha, EVS with Coriolis, EEV modes 1-3) with rain on its first material, an NB OVH inflow
    west (water elevation 2 m, velocity (u_in, 0)), a free NB OF outflow east, and an interior
    node with its element neighbours held at zero velocity and their mean initial depth (DB OVH)."""
    from .model import BCT_OUTFLOW, BCT_OVH_NEU, BCT_VEL_PRS_DIR, BCT_WATER_SOURCE
    m = basin_all_terms(nsteps=nsteps)
    m.name = "combined"
    t_end = (nsteps + 10) * m.dt
    ns = len(m.series)
    const = lambda val: Series(np.array([0.0, t_end]), np.array([val, val]))
    # held nodes: the node nearest the basin centre and every node sharing an element with it
    c = int(np.argmin(np.hypot(m.x - 1000.0, m.y - 1000.0)))
    held = np.unique(m.tri[(m.tri == c).any(axis=1)].ravel())
    m.series = list(m.series) + [const(rate), const(u_in), const(0.0), const(2.0),
                                 const(float(np.mean(m.h0[held])))]
    strings = list(m.strings)
    nmat = len(m.materials)
    strings[0] = dataclasses.replace(strings[0], bc_flag=BCT_WATER_SOURCE, isigma=ns)
    strings[nmat] = StringSpec("edge", bc_flag=BCT_OVH_NEU, ivx=ns + 1, ivy=ns + 2, isigma=ns + 3)
    strings[nmat + 1] = StringSpec("edge", bc_flag=BCT_OUTFLOW)
    strings.append(StringSpec("node", bc_flag=BCT_VEL_PRS_DIR, ivx=ns + 2, ivy=ns + 2, iu0=ns + 4))
    m.strings = strings
    node_string = m.node_string.copy()
    node_string[held] = len(strings) - 1
    m.node_string = node_string
    return m


def channel_obstacle(nsteps: int = 6, with_depth: bool = False) -> SW2Model:
    """The channel with a short line of interior nodes across mid-channel held at zero velocity
    (DB OVL), or at zero velocity and 1 m depth (DB OVH, `with_depth`): a small obstacle in the
    flow.  The reference itself ends with a segmentation fault on the DB OVL form (its edge
    elements generated for DB OVL assume the string lies on the domain boundary)."""
    from .model import BCT_VEL_DIR, BCT_VEL_PRS_DIR
    m = channel(nsteps=nsteps)
    t_end = (nsteps + 10) * m.dt
    ns = len(m.series)
    m.series = list(m.series) + [Series(np.array([0.0, t_end]), np.array([0.0, 0.0])),
                                 Series(np.array([0.0, t_end]), np.array([0.0, 0.0])),
                                 Series(np.array([0.0, t_end]), np.array([1.0, 1.0]))]
    m.strings = list(m.strings) + [StringSpec("node", bc_flag=BCT_VEL_PRS_DIR if with_depth else BCT_VEL_DIR,
                                              ivx=ns, ivy=ns + 1, iu0=ns + 2)]
    pick = (np.abs(m.x - 500.0) < 1.0) & (m.y > 60.0) & (m.y < 140.0)   # a short line across mid-channel
    ns_arr = m.node_string.copy()
    ns_arr[pick] = len(m.strings) - 1
    m.node_string = ns_arr
    m.name = "channel_obstacle"
    return m


def channel_spike(nsteps: int = 12, peak: float = 20.0, max_nonlin_it: int = 5) -> SW2Model:
    """The rectangular channel with a one-step inflow spike (0.5 -> `peak` -> 0.5 m^2/s over
    [40, 50] s) and at most `max_nonlin_it` Newton iterations: the step that meets the spike
    fails, is retried with dt / 4 (twice), and the time loop then recovers the nominal dt by
    doubling it after every accepted step (the reference's tc_end, src/tools/tc_end.c:55-66);
    the run ends with the time loop's shortened last steps."""
    m = channel(nsteps=nsteps, name="spike")
    t_end = (nsteps + 10) * m.dt
    m.series = [Series(np.array([0.0, 40.0, 45.0, 50.0, t_end]), np.array([0.5, 0.5, peak, 0.5, 0.5])),
                m.series[1]]
    m.params = dataclasses.replace(m.params, max_nonlin_it=max_nonlin_it)
    return m


def channel_ovh(nsteps: int = 6, u_in: float = 0.5, **kw) -> SW2Model:
    """The channel with its inflow given as NB OVH instead of NB VEL: water elevation 1 m above
    the datum (the west bed) and velocity (u_in, 0) on the west edge; NB OTW tailwater east."""
    from .model import BCT_OVH_NEU
    m = channel(nsteps=nsteps, **kw)
    t_end = (nsteps + 10) * m.dt
    ns = len(m.series)
    m.series = list(m.series) + [Series(np.array([0.0, t_end]), np.array([u_in, u_in])),
                                 Series(np.array([0.0, t_end]), np.array([0.0, 0.0])),
                                 Series(np.array([0.0, t_end]), np.array([1.0, 1.0]))]
    m.strings = list(m.strings)
    m.strings[1] = StringSpec("edge", bc_flag=BCT_OVH_NEU, ivx=ns, ivy=ns + 1, isigma=ns + 2)
    m.name = "channel_ovh"
    return m


def channel_outflow(nsteps: int = 6, **kw) -> SW2Model:
    """The channel with a free outflow edge (NB OF: implicit flow, no tailwater) east."""
    from .model import BCT_OUTFLOW
    m = channel(nsteps=nsteps, **kw)
    m.strings = list(m.strings)
    m.strings[2] = StringSpec("edge", bc_flag=BCT_OUTFLOW)
    m.name = "channel_outflow"
    return m


def bumpy_basin(npoints: int, seed: int, size: float = 20000.0, slope: float = 5e-4,
                nbumps: int = 40, wse0: float = 2.0, n_median: float = 0.03, n_sigma: float = 0.3,
                nbins: int = 32, q_start: float = 1.0, q_peak: float = 5.0, ramp_steps: int = 30,
                dt: float = 5.0, nsteps: int = 100, drying_limit: float = 0.1,
                tol_nonlin: float = 1e-6, name: str = "basin") -> SW2Model:
    """Seeded Delaunay basin with bumps (triangle count is about ``2 * npoints``).

    * bed: ``z = -slope * x + sum_k A_k exp(-|p - c_k|^2 / (2 s_k^2))`` with
      ``A_k ~ U[0.5, 3]`` m, ``s_k ~ U[200, 1500]`` m (scaled with ``size``),
      centres uniform;
    * initial water surface flat at ``wse0``: depth ``h = wse0 - z`` (negative
      where the bed is above the water, the reference's convention for dry land);
    * Manning n ~ LogNormal(ln n_median, n_sigma) per element, quantised to
      ``nbins`` geometric bins, one material (and one ``FR MNG`` string) per bin;
    * west edge: unit-discharge inflow ramping linearly ``q_start -> q_peak`` over
      ``ramp_steps`` steps, then held; east edge: tailwater level ``wse0``.
    """
    from scipy.spatial import Delaunay

    rng = np.random.Generator(np.random.PCG64(seed))
    nb = max(8, int(round(math.sqrt(npoints) / 2)))        # points per side
    s = np.linspace(0.0, size, nb + 1)[:-1]
    bx = np.concatenate([s, np.full(nb, size), s[::-1] + size / nb, np.zeros(nb)])
    by = np.concatenate([np.zeros(nb), s, np.full(nb, size), s[::-1] + size / nb])
    nin = max(npoints - bx.shape[0], 16)
    margin = size / nb * 0.25
    ix = rng.uniform(margin, size - margin, nin)
    iy = rng.uniform(margin, size - margin, nin)
    x = np.concatenate([bx, ix])
    y = np.concatenate([by, iy])
    order = _morton_order(x, y)
    x, y = x[order].copy(), y[order].copy()
    tri = Delaunay(np.stack([x, y], axis=1)).simplices.astype(np.int32)
    # counter-clockwise orientation and no slivers
    x1, x2, x3 = x[tri[:, 0]], x[tri[:, 1]], x[tri[:, 2]]
    y1, y2, y3 = y[tri[:, 0]], y[tri[:, 1]], y[tri[:, 2]]
    cross = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)
    tri[cross < 0] = tri[cross < 0][:, [0, 2, 1]]
    cross = np.abs(cross)
    tri = tri[cross > 1e-6 * (size / math.sqrt(npoints)) ** 2]
    # drop points no triangle uses (every node must carry a diagonal block)
    used = np.zeros(x.shape[0], bool)
    used[tri.ravel()] = True
    if not used.all():
        remap = np.cumsum(used) - 1
        tri = remap[tri].astype(np.int32)
        x, y = x[used].copy(), y[used].copy()
    # renumber elements by the Morton code of their centroid
    cx = x[tri].mean(axis=1)
    cy = y[tri].mean(axis=1)
    tri = tri[_morton_order(cx, cy)]
    scale = size / 20000.0
    amp = rng.uniform(0.5, 3.0, nbumps)
    wid = rng.uniform(200.0, 1500.0, nbumps) * scale
    cxb = rng.uniform(0.0, size, nbumps)
    cyb = rng.uniform(0.0, size, nbumps)
    # bumps fade out within 10% of the west (inflow) and east (tailwater) edges:
    # a dry node on a NB VEL edge makes the inflow velocity q n / max(h_avg, eps)
    # unbounded (src/fe/sw2/fe_sw2_boundary_resid.c:212-219) and no time step converges
    xs = np.minimum(x, size - x) / size
    taper = np.clip((xs - 0.05) / 0.05, 0.0, 1.0)
    taper = taper * taper * (3.0 - 2.0 * taper)
    z = -slope * x
    for a, w, u, v in zip(amp, wid, cxb, cyb):
        z = z + taper * a * np.exp(-((x - u) ** 2 + (y - v) ** 2) / (2.0 * w * w))
    h0 = wse0 - z
    # per-element roughness classes
    n_elem = np.exp(rng.normal(math.log(n_median), n_sigma, tri.shape[0]))
    lo, hi = n_median * math.exp(-3 * n_sigma), n_median * math.exp(3 * n_sigma)
    edges_b = np.geomspace(lo, hi, nbins + 1)
    tri_mat = np.clip(np.searchsorted(edges_b, n_elem) - 1, 0, nbins - 1).astype(np.int32)
    bin_n = np.sqrt(edges_b[:-1] * edges_b[1:])
    # boundary edges (west: inflow, east: tailwater), oriented as in the mesh
    tol = 1e-9 * size
    # edges used by one triangle only, as (min, max) node pairs
    pairs = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    pairs.sort(axis=1)
    uniq, cnt = np.unique(pairs, axis=0, return_counts=True)
    bedges = [(int(a), int(b)) for a, b in uniq[cnt == 1]]
    west = sorted([k for k in bedges if x[k[0]] < tol and x[k[1]] < tol], key=lambda k: y[k[0]] + y[k[1]])
    east = sorted([k for k in bedges if x[k[0]] > size - tol and x[k[1]] > size - tol],
                  key=lambda k: y[k[0]] + y[k[1]])
    edges = np.array(west + east, dtype=np.int32)
    strings = [StringSpec("mat", manning_n=float(n)) for n in bin_n]
    strings += [StringSpec("edge", bc_flag=BCT_VEL_NEU, isigma=0),
                StringSpec("edge", bc_flag=BCT_PRS_NEU, isigma=1)]
    edge_string = np.array([nbins] * len(west) + [nbins + 1] * len(east), dtype=np.int32)
    t_end = (nsteps + 10) * dt
    ramp = ramp_steps * dt
    series = [Series(np.array([0.0, ramp, max(t_end, ramp + dt)]), np.array([q_start, q_peak, q_peak])),
              Series(np.array([0.0, t_end]), np.array([wse0, wse0]))]
    V = x.shape[0]
    params = Params(tol_nonlin=tol_nonlin, drying_limit=drying_limit, nblock=max(1, V // 2000))
    return SW2Model(x=x, y=y, z=z, tri=tri, tri_mat=tri_mat, edges=edges, edge_string=edge_string,
                    node_string=np.full(V, NORMAL, np.int32), strings=strings,
                    materials=[Material(evs=(0.0, 0.0, 0.0)) for _ in range(nbins)], series=series,
                    params=params, h0=h0, u0=np.zeros(V), v0=np.zeros(V), dt=dt, nsteps=nsteps, name=name)


def ensemble_member(seed: int, tri_lo: float = 5e3, tri_hi: float = 2e5, nsteps: int = 50,
                    name: str = "member") -> SW2Model:
    """One instance of the batched ensemble: triangle count log-uniform in
    [tri_lo, tri_hi], Manning median U[0.015, 0.05], inflow peak U[1, 8] m^2/s,
    dt U[2, 10] s, its own bathymetry seed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    T = math.exp(rng.uniform(math.log(tri_lo), math.log(tri_hi)))
    n_med = rng.uniform(0.015, 0.05)
    q_peak = rng.uniform(1.0, 8.0)
    dt = rng.uniform(2.0, 10.0)
    sub = int(rng.integers(0, 2**31 - 1))
    size = 20000.0 * math.sqrt(T / 1.0e6)
    return bumpy_basin(int(T / 2), sub, size=size, n_median=n_med, q_peak=q_peak, dt=dt,
                       nsteps=nsteps, name=f"{name}{seed}")


# ---------------------------------------------------------------------------------------------
# constituent transport workloads (fe_transport after every flow step)

def const_series(m: SW2Model, value: float) -> int:
    """Appends a constant series to the model; returns its id."""
    t_end = m.t0 + (m.nsteps + 10) * m.dt
    m.series = list(m.series) + [Series(np.array([m.t0, t_end]), np.array([value, value]))]
    return len(m.series) - 1


def channel_transport(nsteps: int = 6, nx: int = 100, ny: int = 20) -> SW2Model:
    """The channel carrying a constituent (reference concentration 1): a Gaussian patch at
    x = 300 m drifting east, the west column of nodes held at 2 (DB TRN node string) and
    diffusion d_m = 0.5 m^2/s."""
    from .model import Constituent
    m = channel(nx=nx, ny=ny, nsteps=nsteps, name="trn_channel")
    ser = const_series(m, 2.0)
    m.strings = list(m.strings) + [StringSpec("node")]
    sid = len(m.strings) - 1
    node_string = m.node_string.copy()
    node_string[m.x == 0.0] = sid
    m.node_string = node_string
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[0.5], node_bc={sid: ser},
                                  c0=np.exp(-((m.x - 300.0) / 100.0) ** 2))]
    return m


def basin_transport(nsteps: int = 8, nbins: int = 3) -> SW2Model:
    """The small wet/dry basin carrying two constituents through its fronts: the first
    (reference concentration 2, diffusion 0.1 / 1 / 3 m^2/s by material) enters with the NB VEL
    inflow at 3 (NB TRN, 1.5 in the reference's normalised units) and leaves through the NB OTW
    tailwater, which also brings in 0.25 where it flows back; the second (reference 1, no
    diffusion, no boundary condition) starts as a smooth field."""
    from .model import Constituent
    m = bumpy_basin(700, seed=11, size=2000.0, nsteps=nsteps, dt=5.0, nbins=nbins, name="trn_basin")
    s_in, s_out = const_series(m, 3.0), const_series(m, 0.5)
    e_in, e_out = nbins, nbins + 1
    c0 = 0.5 + 0.4 * np.sin(m.x / 300.0) * np.cos(m.y / 250.0)
    m.constituents = [Constituent(ref_conc=2.0, diffusion=[0.1, 1.0, 3.0][:nbins], edge_bc={e_in: s_in, e_out: s_out},
                                  c0=c0),
                      Constituent(ref_conc=1.0, c0=1.0 + 0.5 * np.cos(m.x / 400.0))]
    return m


def terms_transport(nsteps: int = 6) -> SW2Model:
    """The all-terms basin (temporal alpha 0.5; EVS with Coriolis and EEV modes 1-3: transport
    then takes its diffusion from the estimated eddy viscosity) with one constituent entering
    at the inflow (NB TRN) and diffusion 2 m^2/s on the EVS material."""
    from .model import Constituent
    m = basin_all_terms(nsteps=nsteps)
    m.name = "trn_terms"
    s_in = const_series(m, 1.0)
    nmat = len(m.materials)
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[2.0, 0.0, 0.0, 0.0], edge_bc={nmat: s_in},
                                  c0=0.2 + 0.1 * np.cos(m.y / 200.0))]
    return m


def outflow_transport(nsteps: int = 6) -> SW2Model:
    """The channel with a free outflow (NB OF) east and a constituent entering with the NB VEL
    inflow west at 0.8 (NB TRN), from a linear initial profile."""
    from .model import Constituent
    m = channel_outflow(nsteps=nsteps)
    m.name = "trn_outflow"
    s_in = const_series(m, 0.8)
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[1.0], edge_bc={1: s_in}, c0=m.x / 1000.0)]
    return m


def salt_transport(nsteps: int = 6) -> SW2Model:
    """Known answer of the reference's own angle_salt check (write_testcase_error_salt,
    src/initio/test_cases.c:1506-1535: |c - 17.5| <= 1e-6 everywhere): the channel with a
    constituent at 17.5 everywhere, entering at 17.5 through the inflow and the tailwater.  A
    uniform concentration stays uniform only if the transport residual is consistent with the
    flow's discrete continuity equation, which the side output elem_rhs_dacont_extra_terms
    provides; it holds where the flow is wet everywhere."""
    from .model import Constituent
    m = channel(nsteps=nsteps, name="trn_salt")
    s = const_series(m, 17.5)
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[1.0], edge_bc={1: s, 2: s},
                                  c0=np.full(m.nnodes, 17.5))]
    return m

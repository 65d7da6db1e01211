"""SW2 model description: mesh, strings, materials, series and solver parameters.

This is the host-side mirror of what AdH reads from its ``.2dm``/``.bc``/``.hot``
files for a 2D shallow-water (SW2) run.  The same :class:`SW2Model` object is

* flattened into the C-ABI structs of ``include/sw2gpu.h`` (see ``capi.py``), and
* written out as AdH input files (:meth:`SW2Model.write_adh`) so that the
  reference executable can run the identical problem.

Conventions follow AdH:

* node ordering and 0-based ids internally; files are written 1-based;
* every 2D element carries a material id; material ``m`` is bound to string ``m``
  (``MTS m m``), which carries the Manning coefficient (``FR MNG``);
* boundary edges (1D elements) carry an edge string whose ``ol_flow.bc_flag`` is
  ``BCT_VEL_NEU`` (card ``NB VEL``) or ``BCT_PRS_NEU`` (card ``NB OTW``)
  (``src/initio/read_bc_NB.c:62-81``);
* the per-node unknowns are ordered ``[u, v, h]`` (``src/fe/sw2/fe_sw2_resid.c:127-130``).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

# --- AdH constants (src/include/define.h) ---------------------------------------
NORMAL = -1                 # define.h:364
UNSET_INT = -3              # define.h:448
UNSET_FLT = -9999999.9      # define.h:449
BCT_PRS_DIR = 7             # define.h:381
BCT_VEL_DIR = 8             # define.h:382
BCT_DIR = 1                 # define.h:375  (DB TRN, a constituent's held concentration)
BCT_NEU = 3                 # define.h:377  (NB TRN, a constituent's inflow concentration)
BCT_PRS_NEU = 9             # define.h:383  (NB OTW, tailwater)
BCT_VEL_NEU = 10            # define.h:384  (NB VEL, unit discharge)
BCT_WATER_SOURCE = 12       # define.h:386
BCT_VEL_PRS_DIR = 16        # define.h:403
BCT_OUTFLOW = 4             # define.h:378
BCT_OVH_NEU = 18            # define.h:406  (NB OVH, tailwater elevation + velocities)
BCT_DIS_NEU = 24            # define.h:412
DBL_EPSILON = np.finfo(np.float64).eps
FLT_EPSILON = float(np.finfo(np.float32).eps)


@dataclasses.dataclass
class Series:
    """Piecewise-linear time series (AdH ``SERIES BC``/``SERIES DT``)."""
    times: np.ndarray
    values: np.ndarray

    def value_avg(self, t1: float, t2: float) -> float:
        """Average of the series over [t1, t2] (trapezoid areas, linear interpolation).

        Restates ``sseries_set_values_average`` (``src/structs/sseries.c:566-613``):
        the boundary data a step sees is the mean of the series over the step.
        Outside the table the end segments are extrapolated linearly, as AdH's
        ``tc_eval_series`` does for the interval search.
        """
        t = self.times
        v = self.values
        if t2 <= t1:
            return self.value_at(t1)
        # integrate the piecewise-linear function exactly
        pts = [t1] + [x for x in t if t1 < x < t2] + [t2]
        area = 0.0
        for a, b in zip(pts[:-1], pts[1:]):
            area += 0.5 * (self.value_at(a) + self.value_at(b)) * (b - a)
        return area / (t2 - t1)

    def value_at(self, tt: float) -> float:
        t = self.times
        v = self.values
        if len(t) == 1:
            return float(v[0])
        i = int(np.searchsorted(t, tt, side="right") - 1)
        i = min(max(i, 0), len(t) - 2)
        w = (tt - t[i]) / (t[i + 1] - t[i])
        return float(v[i] + w * (v[i + 1] - v[i]))


@dataclasses.dataclass
class Material:
    """SW2 material (``MP EVS`` / ``MP EEV`` / ``MP COR``; src/initio/read_bc_MP.c:29-160)."""
    evs: Optional[Sequence[float]] = (0.0, 0.0, 0.0)   # xx, yy, xy eddy viscosity (EVSF)
    eev_coef: float = 0.0                              # estimated eddy viscosity (EEVF)
    eev_mode: int = 0                                  # 0 = not used, 1..3 = EEV modes
    coriolis: float = 0.0                              # latitude in degrees (MP COR)


@dataclasses.dataclass
class StringSpec:
    """One AdH string (``str_values[i]``); only the fields the SW2 step reads."""
    kind: str                       # "mat" | "edge" | "node"
    bc_flag: int = UNSET_INT        # ol_flow.bc_flag
    isigma: int = -1                # series id (0-based) for NB VEL / NB OTW / source
    ivx: int = -1
    ivy: int = -1
    iu0: int = -1
    manning_n: Optional[float] = None   # FR MNG


@dataclasses.dataclass
class Constituent:
    """A general transported constituent (``CN CON``, src/initio/read_bc_CN.c:14-18), carried by
    the 2D flow (fe_transport, src/fe/transport/fe_transport.c:31-113).

    ``ref_conc`` is the reference concentration property[0]: boundary values are divided by it
    (fe_transport_init.c:47, fe_2d_transport_boundary_resid.c:74) while the hot-start values are
    taken as given (ssw.c, the ``ICON`` data set).  ``diffusion[m]`` is material m's ``MP DF``
    coefficient d_m (0 when absent).  ``node_bc`` maps a node string to the series it holds the
    concentration at (``DB TRN``, BCT_DIR); ``edge_bc`` an edge string to the series of the
    concentration of the water that enters through it (``NB TRN``, BCT_NEU)."""
    ref_conc: float = 1.0
    diffusion: Sequence[float] = ()
    node_bc: Dict[int, int] = dataclasses.field(default_factory=dict)
    edge_bc: Dict[int, int] = dataclasses.field(default_factory=dict)
    c0: Optional[np.ndarray] = None                  # initial concentration (None: 0)
    refine_tol: float = 1.0                          # MP TRT, every material (adaption indicator)


@dataclasses.dataclass
class Params:
    """Model and solver parameters (defaults: src/structs/smodel_defaults.c:130-160)."""
    gravity: float = 9.8
    density: float = 1000.0
    viscosity: float = 9.8e-7
    manning_units: float = 1.0      # MP MUC
    drying_limit: float = 0.0       # MP DTL (lower == upper limit)
    tau_temporal: float = 0.0       # OP TEM (0 = implicit Euler)
    tau_pg: float = 0.5             # OP TPG
    tol_nonlin: float = 1e-8        # IP NTL
    inc_nonlin: float = UNSET_FLT   # IP ITL (unset = residual test only)
    max_nonlin_it: int = 10         # IP NIT
    max_lin_it: int = 500           # IP MIT
    max_linesearch_cuts: int = 5    # solv_initialize.c:56
    nblock: int = 1                 # OP BLK (reference CPU solver only)


@dataclasses.dataclass
class SW2Model:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    tri: np.ndarray                  # int32 [T, 3], counter-clockwise
    tri_mat: np.ndarray              # int32 [T], 0-based material id (== material string)
    edges: np.ndarray                # int32 [E, 2] boundary edges with a NB string
    edge_string: np.ndarray          # int32 [E]
    node_string: np.ndarray          # int32 [V], NORMAL or string id
    strings: List[StringSpec]
    materials: List[Material]
    series: List[Series]             # BC series, indexed by StringSpec.isigma etc.
    params: Params
    h0: np.ndarray
    u0: np.ndarray
    v0: np.ndarray
    dt: float = 1.0
    nsteps: int = 1
    t0: float = 0.0
    name: str = "sw2"
    constituents: List[Constituent] = dataclasses.field(default_factory=list)

    # ------------------------------------------------------------------ sizes
    @property
    def nnodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def nelems2d(self) -> int:
        return int(self.tri.shape[0])

    @property
    def nelems1d(self) -> int:
        return int(self.edges.shape[0])

    # ------------------------------------------------------------ derived data
    def roughness_heights(self) -> np.ndarray:
        """Equivalent roughness height per string (``fterms.eqrheight``).

        Manning's n is converted once with k_s = (8.25 sqrt(g) n / k_n)^6
        (``src/friction/fr_manningsn_to_rheight.c:16-30``, applied at
        ``src/structs/sstr_value.c:297``); strings without a friction card keep
        ``UNSET_FLT`` (zero drag, ``src/fe/sw2/fe_sw2_get_roughness.c:44-49``).
        """
        g = self.params.gravity
        kn = self.params.manning_units
        out = np.full(len(self.strings), UNSET_FLT, dtype=np.float64)
        for i, s in enumerate(self.strings):
            if s.manning_n is not None:
                n = s.manning_n
                out[i] = 0.0 if n < 1e-8 else math.pow(8.25 * math.sqrt(g) * n / kn, 6.0)
        return out

    def initial_state(self):
        """The state every time level starts from: the hot start (h0, u0, v0) with the Dirichlet
        node strings' values imposed.  Restates the reference's hot-start reader, which forces the
        initial condition to meet the Dirichlet boundary conditions and then starts the old and
        older levels from it (``src/structs/ssw.c:452-545``); the series are taken at ``t0``."""
        h, u, v = (np.array(a, dtype=np.float64) for a in (self.h0, self.u0, self.v0))
        for sid, st in enumerate(self.strings):
            if st.kind != "node" or st.bc_flag not in (BCT_PRS_DIR, BCT_VEL_DIR, BCT_VEL_PRS_DIR):
                continue
            nodes = self.node_string == sid
            if st.bc_flag in (BCT_VEL_DIR, BCT_VEL_PRS_DIR):
                u[nodes] = self.series[st.ivx].value_at(self.t0)
                v[nodes] = self.series[st.ivy].value_at(self.t0)
            if st.bc_flag in (BCT_PRS_DIR, BCT_VEL_PRS_DIR):
                h[nodes] = self.series[st.iu0].value_at(self.t0)
        return h, u, v

    def transport_tables(self):
        """The constituents as the transport interface takes them: reference concentrations
        [ntrn], MP DF diffusion [ntrn, nmats], per string the constituent's bc flag (0, BCT_DIR
        for DB TRN, BCT_NEU for NB TRN) and its series [ntrn, nstrings], and the initial
        concentrations [ntrn, nnodes] (ICON, 0 when absent)."""
        n, M, S, V = len(self.constituents), len(self.materials), len(self.strings), self.nnodes
        refc = np.array([c.ref_conc for c in self.constituents], dtype=np.float64)
        dm = np.zeros((n, M))
        bc = np.zeros((n, S), np.int32)
        ser = np.full((n, S), -1, np.int32)
        c0 = np.zeros((n, V))
        for k, con in enumerate(self.constituents):
            for m in range(min(M, len(con.diffusion))):
                dm[k, m] = con.diffusion[m]
            for s_id, sr in con.node_bc.items():
                bc[k, s_id], ser[k, s_id] = BCT_DIR, sr
            for s_id, sr in con.edge_bc.items():
                bc[k, s_id], ser[k, s_id] = BCT_NEU, sr
            if con.c0 is not None:
                c0[k] = con.c0
        return refc, dm, bc, ser, c0

    def series_values(self, t1: float, t2: float) -> np.ndarray:
        """Step-averaged value of every BC series over [t1, t2]."""
        return np.array([s.value_avg(t1, t2) for s in self.series], dtype=np.float64)

    def edge_parent(self) -> np.ndarray:
        """2D element adjacent to each boundary edge (``elem1d_find_elem2d``)."""
        key = {}
        for e, (a, b, c) in enumerate(self.tri):
            for p, q in ((a, b), (b, c), (c, a)):
                key[(min(p, q), max(p, q))] = e
        return np.array([key[(min(p, q), max(p, q))] for p, q in self.edges], dtype=np.int32)

    # --------------------------------------------------------------- AdH files
    def write_adh(self, directory: str, name: Optional[str] = None, nsteps: Optional[int] = None) -> str:
        """Write ``name.2dm``, ``name.bc`` and ``name.hot`` for the reference executable."""
        name = name or self.name
        nsteps = self.nsteps if nsteps is None else nsteps
        os.makedirs(directory, exist_ok=True)
        base = os.path.join(directory, name)
        p = self.params
        with open(base + ".2dm", "w") as f:
            f.write("MESH2D\n")
            for e, (a, b, c) in enumerate(self.tri):
                f.write(f"E3T {e + 1} {a + 1} {b + 1} {c + 1} {int(self.tri_mat[e]) + 1}\n")
            for i in range(self.nnodes):
                f.write(f"ND {i + 1} {_f(self.x[i])} {_f(self.y[i])} {_f(self.z[i])}\n")
        nmat = len(self.materials)
        tf = self.t0 + nsteps * self.dt
        with open(base + ".bc", "w") as f:
            w = f.write
            w(f"OP SW2\nOP TRN {len(self.constituents)}\n")
            w(f"OP BLK {p.nblock}\nOP PRE 1\nOP INC 40\n")
            w(f"OP TEM {_f(p.tau_temporal)}\nOP TPG {_f(p.tau_pg)}\n")
            w(f"IP NTL {_f(p.tol_nonlin)}\n")
            if p.inc_nonlin != UNSET_FLT:
                w(f"IP ITL {_f(p.inc_nonlin)}\n")
            w(f"IP NIT {p.max_nonlin_it}\nIP MIT {p.max_lin_it}\n")
            for m, mat in enumerate(self.materials):
                w(f"MTS {m + 1} {m + 1}\n")
                w(f"MP ML {m + 1} 0\nMP SRT {m + 1} 100\n")
                if mat.eev_mode:
                    w(f"MP EEV {m + 1} {_f(mat.eev_coef)} {mat.eev_mode}\n")
                else:
                    xx, yy, xy = mat.evs
                    w(f"MP EVS {m + 1} {_f(xx)} {_f(yy)} {_f(xy)}\n")
                if mat.coriolis != 0.0:
                    w(f"MP COR {m + 1} {_f(mat.coriolis)}\n")
            for k, con in enumerate(self.constituents):          # read_bc_CN.c:14-18, read_bc_MP.c:180-184
                w(f"CN CON {k + 1} {_f(con.ref_conc)}\n")
                for m in range(nmat):
                    dm = con.diffusion[m] if m < len(con.diffusion) else 0.0
                    w(f"MP DF {m + 1} {k + 1} {_f(dm)}\n")
                    w(f"MP TRT {m + 1} {k + 1} {_f(con.refine_tol)}\n")   # read_bc_MP.c:203-210
            if p.drying_limit > 0:
                w(f"MP DTL {_f(p.drying_limit)}\n")
            w(f"MP G {_f(p.gravity)}\nMP RHO {_f(p.density)}\nMP MU {_f(p.viscosity)}\nMP MUC {_f(p.manning_units)}\n")
            for s_id, s in enumerate(self.strings):
                if s.manning_n is not None:
                    w(f"FR MNG {s_id + 1} {_f(s.manning_n)}\n")
            # series: ids 1..nser are BC series, then the DT and output series
            nser = len(self.series)
            for k, s in enumerate(self.series):
                w(f"SERIES BC {k + 1} {len(s.times)} 0 0 0 0\n")
                for t, v in zip(s.times, s.values):
                    w(f"{_f(float(t))} {_f(float(v))}\n")
            w(f"SERIES DT {nser + 1} 2 0 0 0 0\n{_f(self.t0)} {_f(self.dt)}\n{_f(tf + 10 * self.dt)} {_f(self.dt)}\n")
            w(f"SERIES AWRITE {nser + 2} 1 0 0 0 0\n{_f(self.t0)} {_f(tf)} {_f(self.dt)} 0\n")
            w(f"TC T0 {_f(self.t0)} 0\nTC TF {_f(tf)} 0\n")
            for s_id, s in enumerate(self.strings):
                if s.kind == "mat" and s.bc_flag == BCT_WATER_SOURCE:   # read_bc_NB.c:83-88
                    w(f"NB SOURCE {s_id + 1} {s.isigma + 1}\n")
                # DB OVL: the reference then adds edge elements of its own along the string
                # (BCT_DB_VEL, src/tools/create_dbovl_elem1d.c) that this model does not carry
                if s.kind == "node" and s.bc_flag == BCT_VEL_DIR:        # read_bc_DB.c:41-48
                    w(f"DB OVL {s_id + 1} {s.ivx + 1} {s.ivy + 1}\n")
                elif s.kind == "node" and s.bc_flag == BCT_VEL_PRS_DIR:  # read_bc_DB.c:49-58
                    w(f"DB OVH {s_id + 1} {s.ivx + 1} {s.ivy + 1} {s.iu0 + 1}\n")
                if s.kind == "edge":
                    if s.bc_flag == BCT_VEL_NEU:
                        w(f"NB VEL {s_id + 1} {s.isigma + 1}\n")
                    elif s.bc_flag == BCT_PRS_NEU:
                        w(f"NB OTW {s_id + 1} {s.isigma + 1}\n")
                    elif s.bc_flag == BCT_OVH_NEU:   # read_bc_NB.c:94-103: vx, vy, elevation series
                        w(f"NB OVH {s_id + 1} {s.ivx + 1} {s.ivy + 1} {s.isigma + 1}\n")
                    elif s.bc_flag == BCT_OUTFLOW:   # read_bc_NB.c:21-27
                        w(f"NB OF {s_id + 1}\n")
                    else:
                        raise ValueError(f"unsupported edge bc flag {s.bc_flag}")
            for k, con in enumerate(self.constituents):          # read_bc_DB.c:59-65, read_bc_NB.c:119-125
                for s_id, ser in sorted(con.node_bc.items()):
                    w(f"DB TRN {s_id + 1} {k + 1} {ser + 1}\n")
                for s_id, ser in sorted(con.edge_bc.items()):
                    w(f"NB TRN {s_id + 1} {k + 1} {ser + 1}\n")
            for (a, b), s_id in zip(self.edges, self.edge_string):
                w(f"EGS {a + 1} {b + 1} {s_id + 1}\n")
            for i in np.nonzero(self.node_string >= 0)[0]:
                w(f"NDS {i + 1} {int(self.node_string[i]) + 1}\n")
            w("END\n")
        with open(base + ".hot", "w") as f:
            T = self.nelems2d
            f.write(f'DATASET\nOBJTYPE "mesh2d"\nBEGSCL\nND {self.nnodes}\nNC {T}\nNAME "ioh"\n')
            f.write(f"TIMEUNITS seconds\nTS 0 {_f(self.t0)}\n")
            for v in self.h0:
                f.write(f"{_f(float(v))}\n")
            f.write("ENDDS\n")
            f.write(f'DATASET\nOBJTYPE "mesh2d"\nBEGVEC\nND {self.nnodes}\nNC {T}\nNAME "iov"\n')
            f.write(f"TIMEUNITS seconds\nTS 0 {_f(self.t0)}\n")
            for a, b in zip(self.u0, self.v0):
                f.write(f"{_f(float(a))} {_f(float(b))} 0.0\n")
            f.write("ENDDS\n")
            for k, con in enumerate(self.constituents):          # ssw.c: NAME ICON <id>
                if con.c0 is None:
                    continue
                f.write(f'DATASET\nOBJTYPE "mesh2d"\nBEGSCL\nND {self.nnodes}\nNC {T}\nNAME "icon" {k + 1}\n')
                f.write(f"TIMEUNITS seconds\nTS 0 {_f(self.t0)}\n")
                for v in con.c0:
                    f.write(f"{_f(float(v))}\n")
                f.write("ENDDS\n")
        return base


def _f(v) -> str:
    """Shortest round-trip decimal for a float (exact when AdH parses it back)."""
    return repr(float(v))


def geometry(model: SW2Model):
    """Per-element geometry, restating ``get_triangle_linear_djac_nrml_gradPhi``
    (``src/elem/element_djac_nrml_gradPhi.c:193-273``) and the 1D edge length
    and outward normal (``:15-27``, ``src/elem/elem1d_outward_nrml.c:7-66``).

    Returns ``djac[T]``, ``grad[T, 3, 2]``, ``edge_djac[E]``, ``edge_nrml[E, 2]``.
    """
    x, y = model.x, model.y
    n = model.tri
    x1, x2, x3 = x[n[:, 0]], x[n[:, 1]], x[n[:, 2]]
    y1, y2, y3 = y[n[:, 0]], y[n[:, 1]], y[n[:, 2]]
    s1x, s1y = x2 - x1, y2 - y1
    s2x, s2y = x3 - x1, y3 - y1
    cross = s1x * s2y - s2x * s1y
    grad = np.empty((n.shape[0], 3, 2))
    grad[:, 0, 0] = (s1y - s2y) / cross
    grad[:, 0, 1] = (s2x - s1x) / cross
    grad[:, 1, 0] = s2y / cross
    grad[:, 1, 1] = -s2x / cross
    grad[:, 2, 0] = -s1y / cross
    grad[:, 2, 1] = s1x / cross
    djac = cross * 0.5
    e = model.edges
    if e.shape[0]:
        ex1, ex2 = x[e[:, 0]], x[e[:, 1]]
        ey1, ey2 = y[e[:, 0]], y[e[:, 1]]
        dx, dy = ex2 - ex1, ey2 - ey1
        L = np.sqrt(dx * dx + dy * dy)
        nx, ny = dy / L, -dx / L
        par = model.edge_parent()
        cx = (x[n[par, 0]] + x[n[par, 1]] + x[n[par, 2]]) * (1.0 / 3.0)
        cy = (y[n[par, 0]] + y[n[par, 1]] + y[n[par, 2]]) * (1.0 / 3.0)
        flip = ((cx - ex1) * nx + (cy - ey1) * ny) > 0.0
        nx = np.where(flip, -nx, nx)
        ny = np.where(flip, -ny, ny)
        edge_djac = L
        edge_nrml = np.stack([nx, ny], axis=1)
    else:
        edge_djac = np.zeros(0)
        edge_nrml = np.zeros((0, 2))
    return djac, grad, edge_djac, edge_nrml

"""The device element physics (adhv8_kraken_b200/csrc/sw2_physics.cuh, the code every residual and
Jacobian kernel runs) compiled as host C++ and checked element by element against the oracle:
fully wet and wet/dry elements, unperturbed and with the Jacobian's +-eps perturbations, on a basin
with wet/dry fronts and every optional term switched on (temporal alpha, eddy viscosity, Coriolis),
on one with a water source, and on elements holding Dirichlet nodes (DB OVH); and the boundary-edge
residual (NB VEL inflow, NB OTW tailwater, NB OF free outflow, NB OVH elevation + velocity) edge by
edge.
Runs on CPU, so a change to the physics is checked on every CPU run; the GPU parity tests check
the same code as compiled for sm_100a."""
import ctypes as C
import dataclasses
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from adhv8_kraken_b200 import capi, meshgen
from adhv8_kraken_b200.model import BCT_PRS_DIR, BCT_VEL_DIR, BCT_VEL_PRS_DIR, BCT_WATER_SOURCE, Material
from oracle.oracle import Oracle
from oracle.oracle import lib as oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "adhv8_kraken_b200", "csrc")

SHIM = r"""
#include <algorithm>
#include <cmath>
using std::fabs; using std::fmax; using std::log; using std::pow; using std::sqrt;
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__
#include "sw2_physics.cuh"
#include "sw2_mass.cuh"
using namespace sw2;

// xyz: x[3], y[3], z[3]; lv: h, u, v at the current, old and older levels (3 values each);
// geo: djac, gx0, gy0, gx1, gy1, gx2, gy2; phys: g, dll, dul, alpha, tau_pg, dt;
// mat: ks, ev_st, ev_tr, eev_coef, cor_speed, water_src; dflag: the vertices' Dirichlet flags;
// dac: null, or the transport side output (continuity parts of shock capturing and SUPG);
// ws: null, or the element's wind surface stress (x, y);
// pre: evaluate the way the wet Jacobian kernel does (fully wet elements, perturbed calls only):
// the parts the perturbation leaves unchanged precomputed once per element (WetPre) from the
// unperturbed iterate, as the kernel's staging warp forms them, and the column's `fix` mask
extern "C" void host_elem_resid(const double* xyz, const double* lv, const double* geo, int wd, int pvar, int pnode,
                                double dx, const double* phys, const double* mat, int eev_mode, int has_source,
                                int pre, const int* dflag, double* out, double* dac, const double* ws) {
    ElemIn in;
    in.wsx = ws ? ws[0] : 0.0;   // the element's wind surface stress
    in.wsy = ws ? ws[1] : 0.0;
    for (int i = 0; i < 3; i++) {
        in.x[i] = xyz[i]; in.y[i] = xyz[3 + i]; in.z[i] = xyz[6 + i];
        in.h[i] = lv[i]; in.u[i] = lv[3 + i]; in.v[i] = lv[6 + i];
        in.ho[i] = lv[9 + i]; in.uo[i] = lv[12 + i]; in.vo[i] = lv[15 + i];
        in.hoo[i] = lv[18 + i]; in.uoo[i] = lv[21 + i]; in.voo[i] = lv[24 + i];
        in.gx[i] = geo[1 + 2 * i]; in.gy[i] = geo[2 + 2 * i];
    }
    in.djac = geo[0];
    double hc[3], uc[3], vc[3];
    for (int i = 0; i < 3; i++) { hc[i] = in.h[i]; uc[i] = in.u[i]; vc[i] = in.v[i]; }
    if (pvar == kPertH) hc[pnode] += dx;
    else if (pvar == kPertU) uc[pnode] += dx;
    else if (pvar == kPertV) vc[pnode] += dx;
    const PhysParams P{phys[0], phys[1], phys[2], phys[3], phys[4], phys[5]};
    MatParams M{};
    M.ks = mat[0]; M.ev_st = mat[1]; M.ev_tr = mat[2]; M.eev_coef = mat[3]; M.cor_speed = mat[4];
    M.water_src = mat[5]; M.eev_mode = eev_mode; M.has_source = has_source;
    double er[3][3];
    if (pre) {
        WetPre wp;
        wet_levels(in, P, wp.L);
        wet_depth(in, in.h, P, M, wp.D);
        wet_pre_velocity(in, wp);
        const unsigned others = (7u & ~(1u << pnode)) << kFixNode;
        const unsigned fix = pvar == kPertU ? (kFixH | kFixV | others)
                           : pvar == kPertV ? (kFixH | kFixU | others) : (kFixU | kFixV | (7u << kFixNode));
        elem_resid_impl<true, true>(in, hc, uc, vc, wd, pvar, P, M, dflag, er, &wp, fix);
    } else {
        sw2_elem_resid(in, hc, uc, vc, wd, pvar, P, M, dflag, er, dac);
    }
    for (int i = 0; i < 3; i++)
        for (int q = 0; q < 3; q++) out[3 * i + q] = er[i][q];
}

// huv: h, u, v at the edge's two nodes (2 values each); geo: djac, nx, ny; zb: the nodes' beds;
// value: the string's series value (unit discharge or water elevation); bv: NB OVH velocity
extern "C" void host_edge_resid(const double* huv, const double* geo, const double* zb, int kind, double value,
                                const double* bv, int pvar, int pnode, double dx, const double* phys,
                                const int* dflag, double* out) {
    EdgeIn in;
    for (int i = 0; i < 2; i++) { in.h[i] = huv[i]; in.u[i] = huv[2 + i]; in.v[i] = huv[4 + i]; }
    if (pvar == kPertH) in.h[pnode] += dx;
    else if (pvar == kPertU) in.u[pnode] += dx;
    else if (pvar == kPertV) in.v[pnode] += dx;
    in.djac = geo[0]; in.nx = geo[1]; in.ny = geo[2]; in.z0 = zb[0]; in.z1 = zb[1];
    in.bvx = bv[0]; in.bvy = bv[1];
    const PhysParams P{phys[0], phys[1], phys[2], phys[3], phys[4], phys[5]};
    double er[2][3];
    sw2_edge_resid(in, kind, value, pvar, P, dflag, er);
    for (int i = 0; i < 2; i++)
        for (int q = 0; q < 3; q++) out[3 * i + q] = er[i][q];
}

// grid mass and one step's mass flux from the per-element / per-edge terms of sw2_mass.cuh,
// added in element order (the device adds the same terms in a fixed tree order)
static void corners(const int* tri, const double* x, const double* y, const double* h, int e, double* ex, double* ey,
                    double* eh) {
    for (int i = 0; i < 3; i++) { const int n = tri[3 * e + i]; ex[i] = x[n]; ey[i] = y[n]; eh[i] = h[n]; }
}

extern "C" double host_grid_mass(int T, const int* tri, const double* x, const double* y, const double* h,
                                 const double* djac, double density) {
    double mass = 0.0, ex[3], ey[3], eh[3];
    for (int e = 0; e < T; e++) {
        corners(tri, x, y, h, e, ex, ey, eh);
        mass += elem_mass(ex, ey, eh, djac[e]);
    }
    return mass * density;
}

// rate[e]: the element's source rate, or NaN for an element without a source;
// edges: node pairs with their outward normals nrm (nx, ny per edge)
extern "C" double host_mass_flux(int T, const int* tri, const double* x, const double* y, const double* h,
                                 const double* u, const double* v, const double* djac, const double* rate, int E,
                                 const int* edges, const double* nrm, double djac0, double density, double dt) {
    double body = 0.0, edge = 0.0, ex[3], ey[3], eh[3];
    for (int e = 0; e < T; e++) {
        if (rate[e] != rate[e]) continue;
        corners(tri, x, y, h, e, ex, ey, eh);
        body += elem_source_mass(ex, ey, eh, djac[e], rate[e], dt, density);
    }
    for (int j = 0; j < E; j++) {
        const int a = edges[2 * j], b = edges[2 * j + 1];
        const double nx = nrm[2 * j], ny = nrm[2 * j + 1];
        edge -= edge_outflow_term(djac0, density, dt, h[a], h[b], u[a] * nx + v[a] * ny, u[b] * nx + v[b] * ny);
    }
    return body + edge;
}
"""


@pytest.fixture(scope="module")
def host_physics():
    if shutil.which("g++") is None or not os.path.isdir("/usr/local/cuda/include"):
        pytest.skip("no host C++ compiler or CUDA headers")
    work = os.path.join(ROOT, "_build", "host_physics")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    src, lib = os.path.join(work, "shim.cpp"), os.path.join(work, "libhostphys.so")
    with open(src, "w") as fh:
        fh.write(SHIM)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", CSRC, "-I", "/usr/local/cuda/include",
                        "-o", lib, src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(lib)
    yield L
    shutil.rmtree(work, ignore_errors=True)
    try:
        os.rmdir(os.path.dirname(work))
    except OSError:
        pass


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fd_eps(x):   # NUM_DIFF_EPSILON (src/include/macro.h:669-673)
    p = 1.4901161193847656e-08
    e = abs(x) * (1.0 + p) - abs(x)
    return p if e < p else e


def _dirichlet_flags(m):
    """Per node: the device's Dirichlet flag (bit0 PRS_DIR, bit1 VEL_DIR, bit2 VEL_PRS_DIR)."""
    code = {BCT_PRS_DIR: 1, BCT_VEL_DIR: 2, BCT_VEL_PRS_DIR: 4}
    per_string = np.array([code.get(s.bc_flag, 0) if s.kind == "node" else 0 for s in m.strings] + [0], np.int32)
    return per_string[np.where(m.node_string >= 0, m.node_string, len(m.strings))]


def _element_wind(m, flags, att, sx, sy, density):
    """Element wind stress as swind_elem2d_get_local_stress forms it (vertex sum in order, then
    windatt^2 / (3 density)); flag 1 is Wu's drag law (winds_proc_wu) of the nodal value."""
    def wu(g, xs, ys):
        wmag = math.sqrt(math.pow(xs, 2.0) + math.pow(ys, 2.0) + 1e-10)
        cd = (0.8 + 0.065 * wmag) * .001
        return 1.225 * cd * xs * wmag, 1.225 * cd * ys * wmag
    out = np.zeros((m.nelems2d, 2))
    for e, nodes in enumerate(m.tri):
        k = int(m.tri_mat[e])
        wx = wy = 0.0
        for n in nodes:
            a, b = (sx[n], sy[n]) if flags[k] == 0 else wu(m.params.gravity, sx[n], sy[n])
            wx += a
            wy += b
        f = math.pow(att[k], 2.0) / (3 * density)
        out[e] = (wx * f, wy * f)
    return out


def _element_wave(o, m, rxx, rxy, ryy):
    """Element wave radiation stress as swave_elem2d_get_local_stress forms it (CSTORM_WSID off):
    -sum_i (dphi_i/dx Sxx_i + dphi_i/dy Sxy_i), -sum_i (dphi_i/dx Sxy_i + dphi_i/dy Syy_i)."""
    out = np.zeros((m.nelems2d, 2))
    for e, nodes in enumerate(m.tri):
        _, g6 = o.geometry(e)
        sx = sy = 0.0
        for i, n in enumerate(nodes):
            gx, gy = g6[2 * i], g6[2 * i + 1]
            sx -= (gx * rxx[n] + gy * rxy[n])
            sy -= (gx * rxy[n] + gy * ryy[n])
        out[e] = (sx, sy)
    return out


@pytest.mark.parametrize("case", ["all_terms", "terms_fixture", "rain", "obstacle", "combined", "wind", "wave"])
def test_device_physics_matches_oracle_on_host(host_physics, case):
    wind = None
    if case == "combined":
        m = meshgen.basin_combined(nsteps=4)
    elif case == "terms_fixture":   # the all-terms reference fixture's model (EEV mode 3, southern Coriolis)
        m = meshgen.basin_all_terms(nsteps=4)
    elif case == "rain":
        m = meshgen.basin_rain(nsteps=4)
    elif case == "obstacle":
        m = meshgen.channel_obstacle(nsteps=4, with_depth=True)
    elif case in ("wind", "wave"):   # surface stress on fully wet elements: both wind forms; wind + waves
        m = meshgen.bumpy_basin(900, seed=5, size=2500.0, nsteps=4, dt=5.0, nbins=3, name="wind")
    else:
        base = meshgen.bumpy_basin(900, seed=5, size=2500.0, nsteps=4, dt=5.0, nbins=3, name="physics")
        m = dataclasses.replace(
            base, params=dataclasses.replace(base.params, tau_temporal=0.5),
            materials=[Material(evs=(6.0, 2.0, 1.0), coriolis=30.0)] + [Material(eev_coef=0.4, eev_mode=k) for k in (1, 2)])
    o = Oracle(m)
    if case == "wind":
        wrng = np.random.Generator(np.random.PCG64(17))
        flags = np.array([0, 1, 0], np.int32)
        att = np.array([1.0, 0.8, 0.5])
        sx = wrng.normal(0.0, 0.3, m.nnodes)
        sy = wrng.normal(0.0, 0.3, m.nnodes)
        o.set_wind(flags, att, sx, sy)
        wind = _element_wind(m, flags, att, sx, sy, m.params.density)
    if case == "wave":
        wrng = np.random.Generator(np.random.PCG64(19))
        flags = np.array([0, 0, 1], np.int32)
        att = np.array([1.0, 0.9, 0.7])
        sx = wrng.normal(0.0, 0.3, m.nnodes)
        sy = wrng.normal(0.0, 0.3, m.nnodes)
        rads = [wrng.normal(0.0, 0.05, m.nnodes) for _ in range(3)]
        o.set_wind(flags, att, sx, sy)
        o.set_waves(*rads)
        wind = _element_wind(m, flags, att, sx, sy, m.params.density) + _element_wave(o, m, *rads)
    for _ in range(2):   # distinct time levels and moving wet/dry fronts
        assert o.step()["status"] == 0
    series = m.series_values(o.t, o.t + m.dt)
    o.set_dt(m.dt, series)
    o.wdflag()
    wd = o.get_wd()
    arrays = capi.MeshArrays(m)
    prm = capi.make_params(m)
    levels = [o.get_state(k) for k in range(3)]
    phys = np.array([prm.gravity, prm.drying_lower_limit, prm.drying_upper_limit, prm.tau_temporal, prm.tau_pg, m.dt])
    ks = np.ctypeslib.as_array(arrays.mesh.str_rough_height, shape=(len(m.strings),))
    rng = np.random.Generator(np.random.PCG64(3))
    h0 = levels[0][0]
    tri = m.tri
    dflag = _dirichlet_flags(m)
    if case in ("obstacle", "combined"):   # every element holding a Dirichlet node
        fringe = np.nonzero((dflag[tri] != 0).any(axis=1))[0]
    else:                    # wet/dry fronts
        fringe = np.nonzero((wd != 0) | (h0[tri] <= 0.0).any(axis=1))[0]
    picks = np.concatenate([fringe[:150], rng.choice(m.nelems2d, 150, replace=False)])
    assert fringe.size > 0
    worst, wet_columns = 0.0, 0
    for ie in picks:
        nodes = tri[ie]
        xyz = np.concatenate([m.x[nodes], m.y[nodes], m.z[nodes]])
        lv = np.concatenate([levels[k][j][nodes] for k in range(3) for j in range(3)])
        djac, g6 = o.geometry(int(ie))
        geo = np.concatenate([[djac], g6])
        k = int(m.tri_mat[ie])
        mt = m.materials[k]
        xx, yy = mt.evs[0] + prm.viscosity, mt.evs[1] + prm.viscosity
        st = m.strings[k]   # material k's string
        source = st.bc_flag == BCT_WATER_SOURCE
        mat = np.array([ks[k], abs(xx - yy), min(xx, yy), mt.eev_coef,
                        math.sin(math.pi / 180.0 * mt.coriolis) * 2.0 * 7.2722e-5,
                        float(series[st.isigma]) if source else 0.0])
        df = np.ascontiguousarray(dflag[nodes], np.int32)
        fully_wet = wd[ie] == 0 and all((levels[k][0][nodes] > 0).all() for k in range(3))
        cases = [(-1, 0, 0.0, 0)]
        for pvar, arr in ((1, levels[0][1]), (2, levels[0][2]), (5, levels[0][0])):
            b = int(rng.integers(0, 3))
            eps = _fd_eps(arr[nodes[b]])
            cases += [(pvar, b, eps, 1), (pvar, b, -eps, -1)]
        ws = None if wind is None else np.ascontiguousarray(wind[ie])
        for pvar, b, dx, sign in cases:
            dev, ref, dac = np.zeros(9), np.zeros(9), np.zeros(3)
            host_physics.host_elem_resid(_dp(xyz), _dp(lv), _dp(geo), int(wd[ie]), pvar, b, C.c_double(dx), _dp(phys),
                                         _dp(mat), mt.eev_mode, int(source), 0,
                                         df.ctypes.data_as(C.POINTER(C.c_int)), _dp(dev), _dp(dac),
                                         None if ws is None else _dp(ws))
            oracle_lib().orc_body_resid(o.h, int(ie), abs(dx), b, pvar, sign, _dp(ref))
            if fully_wet and pvar != -1:   # the wet Jacobian kernel's evaluation of the same column
                pre = np.zeros(9)
                host_physics.host_elem_resid(_dp(xyz), _dp(lv), _dp(geo), 0, pvar, b, C.c_double(dx), _dp(phys),
                                             _dp(mat), mt.eev_mode, int(source), 1,
                                             df.ctypes.data_as(C.POINTER(C.c_int)), _dp(pre), None,
                                             None if ws is None else _dp(ws))
                assert np.array_equal(pre, ref), (int(ie), pvar, b, sign, pre, ref)
                wet_columns += 1
            # the transport side output of the same call (elem_rhs_dacont_extra_terms)
            assert np.array_equal(dac, o.dacont()[:, ie]), (int(ie), pvar, dac, o.dacont()[:, ie])
            scale = max(np.abs(ref).max(), 1e-300)
            err = float(np.abs(dev - ref).max() / scale)
            worst = max(worst, err)
            assert err <= 1e-12, (int(ie), pvar, b, sign, err, dev, ref)
    assert worst <= 1e-12
    assert wet_columns > 0   # the precomputed-parts path ran


@pytest.mark.parametrize("case", ["tailwater", "outflow", "ovh"])
def test_device_edge_physics_matches_oracle_on_host(host_physics, case):
    from adhv8_kraken_b200.model import BCT_OUTFLOW, BCT_OVH_NEU, BCT_PRS_NEU, BCT_VEL_NEU
    m = {"tailwater": meshgen.channel, "outflow": meshgen.channel_outflow, "ovh": meshgen.channel_ovh}[case](nsteps=4)
    o = Oracle(m)
    assert o.step()["status"] == 0
    series = m.series_values(o.t, o.t + m.dt)
    o.set_dt(m.dt, series)
    prm = capi.make_params(m)
    phys = np.array([prm.gravity, prm.drying_lower_limit, prm.drying_upper_limit, prm.tau_temporal, prm.tau_pg, m.dt])
    h, u, v = o.get_state(0)
    kinds = {BCT_VEL_NEU: 1, BCT_PRS_NEU: 2, BCT_OUTFLOW: 3, BCT_OVH_NEU: 4}
    dflag = _dirichlet_flags(m)
    worst = 0.0
    seen = set()
    for ie, (a, b) in enumerate(m.edges):
        st = m.strings[int(m.edge_string[ie])]
        seen.add(st.bc_flag)
        value = float(series[st.isigma]) if st.isigma >= 0 else 0.0
        bv = np.array([float(series[st.ivx]), float(series[st.ivy])]) if st.bc_flag == BCT_OVH_NEU else np.zeros(2)
        zb = np.array([m.z[a], m.z[b]])
        df = np.ascontiguousarray(dflag[[a, b]], np.int32)
        huv = np.array([h[a], h[b], u[a], u[b], v[a], v[b]])
        cases = [(-1, 0, 0.0, 0)]
        for pvar, arr in ((1, u), (2, v), (5, h)):
            for nd in (0, 1):
                eps = _fd_eps(arr[(a, b)[nd]])
                cases += [(pvar, nd, eps, 1), (pvar, nd, -eps, -1)]
        for pvar, nd, dx, sign in cases:
            dev, ref, geo = np.zeros(6), np.zeros(6), np.zeros(3)
            oracle_lib().orc_edge_resid(o.h, ie, abs(dx), nd, pvar, sign, _dp(ref), _dp(geo))
            host_physics.host_edge_resid(_dp(huv), _dp(geo), _dp(zb), kinds[st.bc_flag], C.c_double(value), _dp(bv),
                                         pvar, nd, C.c_double(dx), _dp(phys), df.ctypes.data_as(C.POINTER(C.c_int)),
                                         _dp(dev))
            err = float(np.abs(dev - ref).max() / max(np.abs(ref).max(), 1e-300))
            worst = max(worst, err)
            assert err <= 1e-12, (ie, pvar, nd, sign, err, dev, ref)
    assert worst <= 1e-12
    assert {"tailwater": BCT_PRS_NEU, "outflow": BCT_OUTFLOW, "ovh": BCT_OVH_NEU}[case] in seen


@pytest.mark.parametrize("case", ["basin", "rain", "channel"])
def test_device_mass_terms_match_oracle_on_host(host_physics, case):
    """Grid mass (tl_find_grid_mass_elem2d, with its h < 0 corner clip and dry corners counted
    as positive mass) and one step's mass flux (water sources, boundary outflow) from the
    device's per-element terms, added in element order: bit-identical to the oracle after every
    step of a wet/dry basin, a basin with rain and the channel with its inflow and tailwater
    edges."""
    from helpers import basin_model
    m = {"basin": basin_model, "rain": lambda: meshgen.basin_rain(nsteps=6), "channel": lambda: meshgen.channel(nsteps=6)}[case]()
    o = Oracle(m)
    tri = np.ascontiguousarray(m.tri, np.int32)
    djac = np.array([o.geometry(e)[0] for e in range(m.nelems2d)])
    edges = np.ascontiguousarray(m.edges, np.int32).reshape(-1, 2)
    nrm, elen = np.zeros((len(edges), 2)), np.zeros(len(edges))
    for j in range(len(edges)):   # the oracle's edge geometry: length and outward normal
        geo = np.zeros(3)
        oracle_lib().orc_edge_resid(o.h, j, 1e-8, 0, -1, 0, _dp(np.zeros(6)), _dp(geo))
        elen[j], nrm[j] = geo[0], geo[1:]
    djac0 = float(elen[0]) if len(edges) else 0.0
    assert (case != "channel") or len(edges) > 0
    rho = m.params.density
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    host_physics.host_grid_mass.restype = C.c_double
    host_physics.host_mass_flux.restype = C.c_double
    saw_negative = False
    for k in range(6):
        t, dt = o.t, m.dt
        assert o.step()["status"] == 0
        series = m.series_values(t, t + dt)
        h, u, v = (np.ascontiguousarray(a) for a in o.get_state(0))
        saw_negative |= bool((h < 0).any())
        got = host_physics.host_grid_mass(m.nelems2d, ip(tri), _dp(m.x), _dp(m.y), _dp(h), _dp(djac), C.c_double(rho))
        assert got == o.grid_mass(0), (k, got, o.grid_mass(0))
        rate = np.full(m.nelems2d, np.nan)
        for e in range(m.nelems2d):
            st = m.strings[int(m.tri_mat[e])]
            if st.bc_flag == BCT_WATER_SOURCE:
                rate[e] = series[st.isigma]
        assert (case != "rain") or np.isfinite(rate).any()
        flux = host_physics.host_mass_flux(m.nelems2d, ip(tri), _dp(m.x), _dp(m.y), _dp(h), _dp(u), _dp(v), _dp(djac),
                                           _dp(rate), len(edges), ip(edges), _dp(nrm), C.c_double(djac0),
                                           C.c_double(rho), C.c_double(dt))
        assert flux == o.mass_flux(dt, series), (k, flux, o.mass_flux(dt, series))
    if case == "basin":
        assert saw_negative   # the dry-corner branches ran

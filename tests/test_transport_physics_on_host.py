"""The device transport physics (adhv8_kraken_b200/csrc/trn_physics.cuh, the code the transport
residual and Jacobian kernels run) compiled as host C++ and checked element by element against the
oracle, bit for bit: every triangle and boundary edge of the wet/dry basin with two constituents
and of the all-terms basin (temporal alpha, EEV diffusion), at flow and concentration states
reached by the oracle's own steps, unperturbed and with the Jacobian's +-eps perturbation of each
vertex.  Runs on CPU; the GPU parity tests check the same code as compiled for sm_100a."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from adhv8_kraken_b200 import meshgen
from adhv8_kraken_b200.model import BCT_DIR
from oracle.oracle import Oracle

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
#include "trn_physics.cuh"
using namespace sw2;

// xy: x[3], y[3]; geo: djac, gx0, gy0, gx1, gy1, gx2, gy2; flow: h, ho, hoo, u, v (3 values each);
// con: c, co, coo (3 each); dac[3]; mat: ks, eev_coef, dm; phys: g, dll, alpha, tau_pg, dt.
// The element's constant parts are formed at the unperturbed concentration, as the kernels do.
extern "C" void host_trn_elem(const double* xy, const double* geo, const double* flow, const double* con,
                              const double* dac, const double* mat, int eev_mode, int wd, unsigned dir,
                              const double* phys, int pnode, double eps, int psign, double* out) {
    TrnElem E;
    for (int i = 0; i < 3; i++) {
        E.x[i] = xy[i]; E.y[i] = xy[3 + i];
        E.gx[i] = geo[1 + 2 * i]; E.gy[i] = geo[2 + 2 * i];
        E.h[i] = flow[i]; E.ho[i] = flow[3 + i]; E.hoo[i] = flow[6 + i];
        E.u[i] = flow[9 + i]; E.v[i] = flow[12 + i];
        E.co[i] = con[3 + i]; E.coo[i] = con[6 + i];
        E.dac[i] = dac[i];
    }
    E.djac = geo[0];
    E.ks = mat[0]; E.eev_coef = mat[1]; E.dm = mat[2];
    E.eev_mode = eev_mode; E.wd = wd; E.dir = dir;
    TrnParams P{phys[0], phys[1], phys[2], phys[3], phys[4]};
    TrnPre pre;
    trn_prepare(E, P, pre);
    double c[3] = {con[0], con[1], con[2]};
    if (pnode >= 0) c[pnode] += psign * eps;
    trn_elem_resid(E, pre, c, P, out);
}

// geo: djac, nx, ny; flow: h0, h1, u0, u1, v0, v1
extern "C" void host_trn_edge(const double* geo, const double* flow, int kind, int cflag, double flux_in,
                              double c_user, unsigned dir, const double* con, double dt, int pnode, double eps,
                              int psign, double* out) {
    TrnEdge B;
    B.djac = geo[0]; B.nx = geo[1]; B.ny = geo[2];
    for (int i = 0; i < 2; i++) { B.h[i] = flow[i]; B.u[i] = flow[2 + i]; B.v[i] = flow[4 + i]; }
    B.kind = kind; B.cflag = cflag; B.flux_in = flux_in; B.c_user = c_user; B.dir = dir;
    double c[2] = {con[0], con[1]};
    if (pnode >= 0) c[pnode] += psign * eps;
    trn_edge_resid(B, c, dt, out);
}

extern "C" double host_trn_eps(double cn, double refc) { return trn_eps(cn, refc); }
"""

EDGE_KIND = {10: 1, 9: 2, 4: 3, 18: 4}     # BCT_VEL_NEU, BCT_PRS_NEU, BCT_OUTFLOW, BCT_OVH_NEU -> DevMesh::bkind


@pytest.fixture(scope="module")
def host_trn():
    if shutil.which("g++") is None or not os.path.isdir("/usr/local/cuda/include"):
        pytest.skip("no host C++ compiler or CUDA headers")
    work = os.path.join(ROOT, "_build", "host_transport")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    src, lib = os.path.join(work, "shim.cpp"), os.path.join(work, "libhosttrn.so")
    with open(src, "w") as fh:
        fh.write(SHIM)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", CSRC, "-I", "/usr/local/cuda/include",
                        "-o", lib, src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(lib)
    dp = C.POINTER(C.c_double)
    L.host_trn_elem.argtypes = [dp, dp, dp, dp, dp, dp, C.c_int, C.c_int, C.c_uint, dp, C.c_int, C.c_double, C.c_int,
                                dp]
    L.host_trn_edge.argtypes = [dp, dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_uint, dp, C.c_double, C.c_int,
                                C.c_double, C.c_int, dp]
    L.host_trn_eps.argtypes = [C.c_double, C.c_double]
    L.host_trn_eps.restype = C.c_double
    yield L
    shutil.rmtree(work, ignore_errors=True)
    try:
        os.rmdir(os.path.dirname(work))
    except OSError:
        pass


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _check_model(L, m, steps):
    o = Oracle(m)
    for _ in range(steps):
        assert o.step()["status"] == 0
        assert all(s["status"] == 0 for s in o.transport_step())
    # one more flow step: the constituents' levels are those the next transport step starts from
    t0 = o.t
    assert o.step()["status"] == 0
    dt = m.dt
    series = m.series_values(t0, t0 + dt)
    lv = [o.get_state(l) for l in range(3)]
    wd = o.get_wd()
    dac = o.dacont()
    p = m.params
    phys = np.array([p.gravity, p.drying_limit, p.tau_temporal, p.tau_pg, dt])
    ks = m.roughness_heights()
    refc, dm, bc, ser, _ = m.transport_tables()
    checked = 0
    for k in range(len(m.constituents)):
        c = [o.get_conc(k, l) for l in range(3)]
        held = np.array([s >= 0 and bc[k, s] == BCT_DIR for s in m.node_string])
        for e in range(m.nelems2d):
            n = m.tri[e]
            djac, g = o.geometry(e)
            xy = np.concatenate([m.x[n], m.y[n]])
            geo = np.concatenate([[djac], g])
            flow = np.concatenate([lv[0][0][n], lv[1][0][n], lv[2][0][n], lv[0][1][n], lv[0][2][n]])
            con = np.concatenate([c[0][n], c[1][n], c[2][n]])
            mat_id = int(m.tri_mat[e])
            mat = m.materials[mat_id]
            matv = np.array([ks[mat_id], mat.eev_coef, dm[k, mat_id]])
            dirb = sum(1 << i for i in range(3) if held[n[i]])
            cases = [(-1, 0.0, 1)]
            for i in range(3):
                eps = L.host_trn_eps(c[0][n[i]], refc[k])
                cases += [(i, eps, 1), (i, eps, -1)]
            for pnode, eps, psign in cases:
                got = np.zeros(3)
                L.host_trn_elem(_dp(xy), _dp(geo), _dp(flow), _dp(con), _dp(dac[:, e]), _dp(matv), mat.eev_mode,
                                int(wd[e]), dirb, _dp(phys), pnode, eps, psign, _dp(got))
                exp = o.trn_body_resid(k, e, eps, pnode, psign)
                assert np.array_equal(got, exp), (k, e, pnode, psign, got, exp)
                checked += 1
        geom = _edge_geometry(m)
        for j in range(m.nelems1d):
            n = m.edges[j]
            s = int(m.edge_string[j])
            flow = np.concatenate([lv[0][0][n], lv[0][1][n], lv[0][2][n]])
            st = m.strings[s]
            flux = series[st.isigma] if st.isigma >= 0 else 0.0
            c_user = series[ser[k, s]] * (1.0 / refc[k]) if bc[k, s] else 0.0
            dirb = sum(1 << i for i in range(2) if held[n[i]])
            cases = [(-1, 0.0, 1)]
            for i in range(2):
                eps = L.host_trn_eps(c[0][n[i]], refc[k])
                cases += [(i, eps, 1), (i, eps, -1)]
            for pnode, eps, psign in cases:
                got = np.zeros(2)
                L.host_trn_edge(_dp(geom[j]), _dp(flow), EDGE_KIND[st.bc_flag], int(bc[k, s]), flux, c_user, dirb,
                                _dp(c[0][n]), dt, pnode, eps, psign, _dp(got))
                exp = o.trn_edge_resid(k, j, eps, pnode, psign)
                assert np.array_equal(got, exp), (k, j, pnode, psign, got, exp)
                checked += 1
    return checked


def _edge_geometry(m):
    """Edge length and outward normal as the library forms them (the oracle's restatement of
    elem1d_outward_nrml)."""
    out = np.zeros((m.nelems1d, 3))
    par = m.edge_parent()
    for j, (a, b) in enumerate(m.edges):
        dx, dy = m.x[b] - m.x[a], m.y[b] - m.y[a]
        L = np.sqrt(dx * dx + dy * dy)
        nx, ny = dy / L, -dx / L
        t = m.tri[par[j]]
        cx = (1 / 3) * (m.x[t[0]] + m.x[t[1]] + m.x[t[2]])
        cy = (1 / 3) * (m.y[t[0]] + m.y[t[1]] + m.y[t[2]])
        if (cx - m.x[a]) * nx + (cy - m.y[a]) * ny > 0:
            nx, ny = -nx, -ny
        out[j] = (np.sqrt((m.x[a] - m.x[b]) ** 2 + (m.y[a] - m.y[b]) ** 2), nx, ny)
    return out


def test_device_transport_physics_matches_oracle_bitwise_on_wet_dry_basin(host_trn):
    m = meshgen.basin_transport(nsteps=6)
    assert _check_model(host_trn, m, 3) > 15000


def test_device_transport_physics_matches_oracle_bitwise_with_eev_and_alpha(host_trn):
    m = meshgen.terms_transport(nsteps=5)
    assert _check_model(host_trn, m, 2) > 9000


def test_device_transport_physics_matches_oracle_bitwise_with_held_nodes(host_trn):
    m = meshgen.channel_transport(nsteps=4, nx=30, ny=6)
    assert _check_model(host_trn, m, 2) > 1000

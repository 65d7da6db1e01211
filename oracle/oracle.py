"""ctypes front end of the CPU oracle (``oracle/sw2_oracle.c``).  TEST INFRASTRUCTURE ONLY.

Used by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` as the checker of the B200 library; never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from adhv8_kraken_b200.capi import MeshArrays, Stats, make_params, c_double_p, c_int32_p

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "sw2_oracle.c")
LIB = os.path.join(HERE, "libsw2oracle.so")

_lib = None


def build(force: bool = False) -> str:
    hdr = os.path.join(HERE, "..", "include", "sw2gpu.h")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(hdr)):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=c99", "-o", LIB, SRC, "-lm"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        for name in ("orc_destroy", "orc_resid", "orc_load", "orc_wdflag"):
            getattr(L, name).argtypes = [C.c_void_p] + ([c_double_p] if name == "orc_resid" else [])
        L.orc_nnzb.restype = C.c_int
        L.orc_bandwidth.restype = C.c_int
        L.orc_step.restype = C.c_int
        L.orc_step.argtypes = [C.c_void_p, C.c_double, c_double_p, C.c_void_p]
        L.orc_linear_solve.restype = C.c_int
        L.orc_linear_solve.argtypes = [C.c_void_p, c_double_p, c_double_p]
        L.orc_set_dt.argtypes = [C.c_void_p, C.c_double, c_double_p]
        L.orc_body_resid.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, c_double_p]
        L.orc_nnzb.argtypes = [C.c_void_p]
        L.orc_bandwidth.argtypes = [C.c_void_p]
        L.orc_set_state.argtypes = [C.c_void_p, C.c_int, c_double_p, c_double_p, c_double_p]
        L.orc_get_state.argtypes = [C.c_void_p, C.c_int, c_double_p, c_double_p, c_double_p]
        L.orc_get_wd.argtypes = [C.c_void_p, c_int32_p]
        L.orc_set_wd.argtypes = [C.c_void_p, c_int32_p]
        L.orc_pattern.argtypes = [C.c_void_p, c_int32_p, c_int32_p]
        L.orc_get_matrix.argtypes = [C.c_void_p, c_double_p, c_double_p]
        L.orc_set_matrix.argtypes = [C.c_void_p, c_double_p, c_double_p]
        L.orc_geometry.argtypes = [C.c_void_p, C.c_int, c_double_p]
        L.orc_get_dacont.argtypes = [C.c_void_p, c_double_p]
        L.orc_edge_resid.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, c_double_p, c_double_p]
        L.orc_elem_error.argtypes = [C.c_void_p, c_double_p, c_double_p, c_double_p]
        L.orc_set_wind.argtypes = [C.c_void_p, c_int32_p, c_double_p, c_double_p, c_double_p]
        L.orc_set_wind.restype = C.c_int
        L.orc_set_waves.argtypes = [C.c_void_p, c_double_p, c_double_p, c_double_p]
        L.orc_set_waves.restype = None
        L.orc_grid_mass.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_grid_mass.restype = C.c_double
        L.orc_mass_flux.argtypes = [C.c_void_p, C.c_double, C.c_double, c_double_p]
        L.orc_mass_flux.restype = C.c_double
        L.orc_trn_setup.argtypes = [C.c_void_p, C.c_int, c_double_p, c_double_p, c_int32_p, c_int32_p]
        L.orc_trn_setup.restype = C.c_int
        L.orc_trn_set_conc.argtypes = [C.c_void_p, C.c_int, C.c_int, c_double_p]
        L.orc_trn_get_conc.argtypes = [C.c_void_p, C.c_int, C.c_int, c_double_p]
        L.orc_set_dacont.argtypes = [C.c_void_p, c_double_p]
        L.orc_trn_get_bcmask.argtypes = [C.c_void_p, c_int32_p]
        L.orc_trn_init.argtypes = [C.c_void_p, C.c_int]
        L.orc_trn_resid.argtypes = [C.c_void_p, C.c_int, c_double_p]
        L.orc_trn_load.argtypes = [C.c_void_p, C.c_int]
        L.orc_trn_get_matrix.argtypes = [C.c_void_p, c_double_p, c_double_p]
        L.orc_trn_step.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_trn_step.restype = C.c_int
        L.orc_trn_elem_error.argtypes = [C.c_void_p, c_double_p, c_double_p, c_double_p]
        for name in ("orc_trn_body_resid", "orc_trn_edge_resid"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, c_double_p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(c_double_p)


def _ip(a):
    return a.ctypes.data_as(c_int32_p)


class Oracle:
    """One SW2 model on the CPU, restating the reference step by step."""

    def __init__(self, model, nblock: int = 1, lin_rtol: float = 1e-5, lin_atol: float = 1e-10):
        self.model = model
        self.arrays = MeshArrays(model)
        self.params = make_params(model, lin_rtol=lin_rtol, lin_atol=lin_atol)
        L = lib()
        self.h = L.orc_create(C.byref(self.arrays.mesh), C.byref(self.params), nblock)
        if not self.h:
            raise ValueError("oracle rejected the model")
        self.V, self.T = model.nnodes, model.nelems2d
        self.nnzb = L.orc_nnzb(self.h)
        self.t = model.t0
        h0, u0, v0 = model.initial_state()
        for level in range(3):
            self.set_state(level, h0, u0, v0)
        self.ntrn = len(model.constituents)
        if self.ntrn:
            refc, dm, bc, ser, c0 = model.transport_tables()
            self._trn = (refc, dm, bc, ser)     # kept alive: the C side copies them anyway
            if L.orc_trn_setup(self.h, self.ntrn, _dp(refc), _dp(np.ascontiguousarray(dm)),
                               _ip(np.ascontiguousarray(bc)), _ip(np.ascontiguousarray(ser))):
                raise ValueError("oracle rejected the constituents")
            for k in range(self.ntrn):          # the hot start's old and older levels (ssw.c)
                for level in range(3):
                    self.set_conc(k, level, c0[k])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_state(self, level, h, u, v):
        h, u, v = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, u, v))
        lib().orc_set_state(C.c_void_p(self.h), level, _dp(h), _dp(u), _dp(v))

    def get_state(self, level=0):
        h, u, v = (np.zeros(self.V) for _ in range(3))
        lib().orc_get_state(C.c_void_p(self.h), level, _dp(h), _dp(u), _dp(v))
        return h, u, v

    def set_dt(self, dt, series):
        s = np.ascontiguousarray(series, dtype=np.float64)
        lib().orc_set_dt(C.c_void_p(self.h), dt, _dp(s) if s.size else None)

    def wdflag(self):
        lib().orc_wdflag(self.h)
        return self.get_wd()

    def get_wd(self):
        wd = np.zeros(self.T, np.int32)
        lib().orc_get_wd(C.c_void_p(self.h), _ip(wd))
        return wd

    def set_wd(self, wd):
        wd = np.ascontiguousarray(wd, dtype=np.int32)
        lib().orc_set_wd(C.c_void_p(self.h), _ip(wd))

    def pattern(self):
        rp = np.zeros(self.V + 1, np.int32)
        col = np.zeros(self.nnzb, np.int32)
        lib().orc_pattern(C.c_void_p(self.h), _ip(rp), _ip(col))
        return rp, col

    def resid(self):
        r = np.zeros(3 * self.V)
        lib().orc_resid(self.h, _dp(r))
        return r

    def load(self):
        """FD Jacobian (sorted BCSR values) and the residual after the tiny-diagonal fix."""
        lib().orc_load(self.h)
        val = np.zeros(9 * self.nnzb)
        r = np.zeros(3 * self.V)
        lib().orc_get_matrix(C.c_void_p(self.h), _dp(val), _dp(r))
        return val.reshape(-1, 3, 3), r

    def set_matrix(self, val, resid):
        val = np.ascontiguousarray(val, dtype=np.float64).reshape(-1)
        resid = np.ascontiguousarray(resid, dtype=np.float64)
        lib().orc_set_matrix(C.c_void_p(self.h), _dp(val), _dp(resid))

    def linear_solve(self, rhs):
        b = np.array(rhs, dtype=np.float64)
        x = np.zeros(3 * self.V)
        its = lib().orc_linear_solve(self.h, _dp(b), _dp(x))
        return x, its

    def body_resid(self, ie, eps=0.0, pnode=0, pvar=-1, psign=0):
        out = np.zeros(9)
        lib().orc_body_resid(self.h, ie, eps, pnode, pvar, psign, _dp(out))
        return out.reshape(3, 3)

    def dacont(self):
        """elem_rhs_dacont_extra_terms as [3, T] (continuity parts of shock capturing and SUPG of
        each element's last residual evaluation, the reference's side output for transport)."""
        out = np.zeros(3 * self.T)
        lib().orc_get_dacont(self.h, _dp(out))
        return out.reshape(3, self.T)

    def geometry(self, ie):
        """(djac, [gx0, gy0, gx1, gy1, gx2, gy2]) of element ie."""
        out = np.zeros(7)
        lib().orc_geometry(self.h, ie, _dp(out))
        return out[0], out[1:]

    def set_wind(self, mat_flag=None, mat_windatt=None, stress_x=None, stress_y=None):
        """Wind surface stress from nodal wind values (None: off)."""
        if stress_x is None:
            lib().orc_set_wind(self.h, None, None, None, None)
            return
        f = np.ascontiguousarray(mat_flag, dtype=np.int32)
        a = np.ascontiguousarray(mat_windatt, dtype=np.float64)
        sx = np.ascontiguousarray(stress_x, dtype=np.float64)
        sy = np.ascontiguousarray(stress_y, dtype=np.float64)
        if lib().orc_set_wind(self.h, f.ctypes.data_as(c_int32_p), _dp(a), _dp(sx), _dp(sy)):
            raise ValueError("wind stress flag not supported")

    def set_waves(self, rads_xx=None, rads_xy=None, rads_yy=None):
        """Wave radiation stress from nodal radiation stresses Sxx, Sxy, Syy (None: off)."""
        if rads_xx is None:
            lib().orc_set_waves(self.h, None, None, None)
            return
        a, b, c = (np.ascontiguousarray(r, dtype=np.float64) for r in (rads_xx, rads_xy, rads_yy))
        lib().orc_set_waves(self.h, _dp(a), _dp(b), _dp(c))

    def elem_error(self, refine_tol):
        """Adaption error indicator (ssw_2d_calculate_elem_error) of the current and old levels
        and the last dt: (elem_error [T], node_error [V]); refine_tol per material."""
        tol = np.ascontiguousarray(refine_tol, dtype=np.float64)
        ee, ne = np.zeros(self.T), np.zeros(self.V)
        lib().orc_elem_error(self.h, _dp(tol), _dp(ee), _dp(ne))
        return ee, ne

    def grid_mass(self, level=0, density=None):
        """Water mass of a time level (tl_find_grid_mass_elem2d)."""
        rho = self.model.params.density if density is None else density
        return lib().orc_grid_mass(self.h, level, rho)

    def mass_flux(self, dt, series_now=None, density=None):
        """Mass entering through sources and boundary edges over a step of dt at the current
        level (the per-step term tl_find_grid_mass_error_elem2d accumulates); series_now: value
        of every series at the evaluation time (water sources only)."""
        rho = self.model.params.density if density is None else density
        s = np.zeros(max(len(self.model.series), 1)) if series_now is None else np.ascontiguousarray(series_now, float)
        return lib().orc_mass_flux(self.h, rho, dt, _dp(s))

    def step(self, dt=None, t=None):
        """One time step with the series averaged over [t, t + dt]; returns the stats dict."""
        dt = self.model.dt if dt is None else dt
        t = self.t if t is None else t
        s = self.model.series_values(t, t + dt)
        st = Stats()
        rc = lib().orc_step(self.h, dt, _dp(s) if s.size else None, C.byref(st))
        if rc == 0:
            self.t = t + dt
        return st.as_dict()

    # ------------------------------------------------------------------ transport
    def set_conc(self, itrn, level, c):
        c = np.ascontiguousarray(c, dtype=np.float64)
        lib().orc_trn_set_conc(C.c_void_p(self.h), itrn, level, _dp(c))

    def get_conc(self, itrn, level=0):
        c = np.zeros(self.V)
        lib().orc_trn_get_conc(C.c_void_p(self.h), itrn, level, _dp(c))
        return c

    def set_dacont(self, dac):
        """elem_rhs_dacont_extra_terms as [3, T] (vertex-major, as dacont() returns it)."""
        d = np.ascontiguousarray(dac, dtype=np.float64).reshape(-1)
        lib().orc_set_dacont(C.c_void_p(self.h), _dp(d))

    def trn_init(self, itrn):
        """fe_transport_init: the current concentration from the old one, dry nodes 0, Dirichlet
        values; returns bc_mask."""
        lib().orc_trn_init(C.c_void_p(self.h), itrn)
        m = np.zeros(self.V, np.int32)
        lib().orc_trn_get_bcmask(C.c_void_p(self.h), _ip(m))
        return m

    def trn_resid(self, itrn):
        r = np.zeros(self.V)
        lib().orc_trn_resid(C.c_void_p(self.h), itrn, _dp(r))
        return r

    def trn_load(self, itrn):
        """Scalar FD Jacobian over the pattern (sorted columns) and the residual it goes with."""
        lib().orc_trn_load(C.c_void_p(self.h), itrn)
        val, r = np.zeros(self.nnzb), np.zeros(self.V)
        lib().orc_trn_get_matrix(C.c_void_p(self.h), _dp(val), _dp(r))
        return val, r

    def transport_step(self):
        """fe_transport after an accepted flow step: every constituent in order; returns the
        stats dicts (stops at the first failure, as the reference does)."""
        out = []
        for k in range(self.ntrn):
            st = Stats()
            rc = lib().orc_trn_step(C.c_void_p(self.h), k, C.byref(st))
            out.append(st.as_dict())
            if rc:
                break
        return out

    def trn_body_resid(self, itrn, ie, eps=0.0, pnode=-1, psign=1):
        out = np.zeros(3)
        lib().orc_trn_body_resid(C.c_void_p(self.h), itrn, ie, eps, pnode, psign, _dp(out))
        return out

    def trn_edge_resid(self, itrn, ie, eps=0.0, pnode=-1, psign=1):
        out = np.zeros(2)
        lib().orc_trn_edge_resid(C.c_void_p(self.h), itrn, ie, eps, pnode, psign, _dp(out))
        return out

    def trn_elem_error(self, refine_tol, elem_error):
        """The constituents' adaption error indicator (scon_calculate_elem2d_error) folded into
        elem_error (the flow's, as fe_main calls them): (elem_error [T], node_error [ntrn, V]);
        refine_tol [ntrn, nmats] (MP TRT)."""
        tol = np.ascontiguousarray(refine_tol, dtype=np.float64)
        ee = np.array(elem_error, dtype=np.float64)
        ne = np.zeros(self.ntrn * self.V)
        lib().orc_trn_elem_error(self.h, _dp(tol), _dp(ee), _dp(ne))
        return ee, ne.reshape(self.ntrn, self.V)

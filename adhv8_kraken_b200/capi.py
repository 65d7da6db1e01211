"""ctypes mirror of ``include/sw2gpu.h`` and marshalling of :class:`SW2Model`.

The same ``sw2gpu_mesh`` / ``sw2gpu_params`` structs feed the B200 library and
the CPU oracle, so both are driven from identical inputs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .model import SW2Model, UNSET_FLT

c_int32_p = C.POINTER(C.c_int32)
c_double_p = C.POINTER(C.c_double)

SW2GPU_OK = 0
SW2GPU_E_ARG = 1
SW2GPU_E_CUDA = 2
SW2GPU_E_NOMEM = 3
SW2GPU_E_NEWTON = 4
SW2GPU_E_LINEAR = 5
SW2GPU_E_NAN = 6
SW2GPU_E_TIMEOUT = 7
SW2GPU_FP64 = 0
SW2GPU_MIXED = 1
SW2GPU_PREC_BJACOBI = 0
SW2GPU_PREC_ILU0 = 1
SW2GPU_PREC_BAND = 2
SW2GPU_PREC_DILU = 3
SW2GPU_BCT_DIR = 1    # DB TRN
SW2GPU_BCT_NEU = 3    # NB TRN
SW2GPU_BCT_LID_DFT = 20         # lids on node strings: refused by sw2gpu_create (not built)
SW2GPU_BCT_LID_ELV = 21
SW2GPU_BCT_LID_DEP = 22


class Mesh(C.Structure):
    _fields_ = [
        ("nnodes", C.c_int32), ("nelems2d", C.c_int32), ("nelems1d", C.c_int32),
        ("nstrings", C.c_int32), ("nmats", C.c_int32), ("nseries", C.c_int32),
        ("x", c_double_p), ("y", c_double_p), ("z", c_double_p),
        ("node_string", c_int32_p), ("elem2d_nodes", c_int32_p), ("elem2d_mat", c_int32_p),
        ("elem1d_nodes", c_int32_p), ("elem1d_string", c_int32_p), ("elem1d_parent", c_int32_p),
        ("str_bc_flag", c_int32_p), ("str_isigma", c_int32_p), ("str_ivx", c_int32_p),
        ("str_ivy", c_int32_p), ("str_iu0", c_int32_p), ("str_rough_height", c_double_p),
        ("mat_eev_mode", c_int32_p), ("mat_ev", c_double_p), ("mat_eev_coef", c_double_p),
        ("mat_coriolis", c_double_p),
    ]


class Params(C.Structure):
    _fields_ = [
        ("gravity", C.c_double), ("density", C.c_double), ("viscosity", C.c_double),
        ("drying_lower_limit", C.c_double), ("drying_upper_limit", C.c_double),
        ("tau_temporal", C.c_double), ("tau_pg", C.c_double),
        ("tol_nonlin", C.c_double), ("inc_nonlin", C.c_double),
        ("max_nonlin_it", C.c_int32), ("max_lin_it", C.c_int32), ("max_linesearch_cuts", C.c_int32),
        ("precision", C.c_int32), ("precond", C.c_int32), ("reserved", C.c_int32),
        ("lin_rtol", C.c_double), ("lin_atol", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("newton_its", C.c_int32), ("linear_its", C.c_int32),
        ("linesearch_cuts", C.c_int32), ("resid_max", C.c_double), ("resid_l2", C.c_double),
        ("inc_max", C.c_double), ("device_ms", C.c_double), ("kernel_launches", C.c_int32),
        ("wd_elems", C.c_int32), ("jac_ms", C.c_double), ("krylov_ms", C.c_double),
        ("resid_ms", C.c_double), ("other_ms", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Transport(C.Structure):
    """sw2gpu_transport: the constituents (include/sw2gpu.h)."""
    _fields_ = [
        ("ntransport", C.c_int32), ("ref_conc", C.POINTER(C.c_double)), ("diffusion", C.POINTER(C.c_double)),
        ("str_bc_flag", C.POINTER(C.c_int32)), ("str_series", C.POINTER(C.c_int32)),
    ]


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


class RunStats(C.Structure):
    """sw2gpu_run_stats: one instance that left a continuous-batching engine."""
    _fields_ = [
        ("id", C.c_int64), ("status", C.c_int32), ("steps", C.c_int32), ("failures", C.c_int32),
        ("newton_its", C.c_int32), ("linear_its", C.c_int32), ("ticks", C.c_int32), ("t", C.c_double),
        ("dt", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RequestStats(C.Structure):
    """sw2gpu_request_stats: one finished request of a sw2gpu_server."""
    _fields_ = [
        ("id", C.c_int64), ("status", C.c_int32), ("steps", C.c_int32), ("failures", C.c_int32),
        ("newton_its", C.c_int32), ("linear_its", C.c_int32), ("reserved", C.c_int32), ("t", C.c_double),
        ("queue_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double), ("device_bytes", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


SW2GPU_PENDING = 100


class MeshArrays:
    """Owns the numpy buffers behind a :class:`Mesh` struct."""

    def __init__(self, m: SW2Model):
        self.keep = []
        S = len(m.strings)
        M = len(m.materials)

        def p(a, kind):
            arr = _i32(a) if kind == "i" else _f64(a)
            if arr.size == 0:
                arr = np.zeros(1, arr.dtype)
            self.keep.append(arr)
            return arr.ctypes.data_as(c_int32_p if kind == "i" else c_double_p)

        self.mesh = Mesh()
        me = self.mesh
        me.nnodes, me.nelems2d, me.nelems1d = m.nnodes, m.nelems2d, m.nelems1d
        me.nstrings, me.nmats, me.nseries = S, M, len(m.series)
        me.x, me.y, me.z = p(m.x, "f"), p(m.y, "f"), p(m.z, "f")
        me.node_string = p(m.node_string, "i")
        me.elem2d_nodes = p(m.tri.reshape(-1), "i")
        me.elem2d_mat = p(m.tri_mat, "i")
        me.elem1d_nodes = p(m.edges.reshape(-1), "i")
        me.elem1d_string = p(m.edge_string, "i")
        me.elem1d_parent = p(m.edge_parent() if m.nelems1d else np.zeros(0), "i")
        me.str_bc_flag = p([s.bc_flag for s in m.strings], "i")
        me.str_isigma = p([s.isigma for s in m.strings], "i")
        me.str_ivx = p([s.ivx for s in m.strings], "i")
        me.str_ivy = p([s.ivy for s in m.strings], "i")
        me.str_iu0 = p([s.iu0 for s in m.strings], "i")
        me.str_rough_height = p(m.roughness_heights(), "f")
        me.mat_eev_mode = p([mt.eev_mode for mt in m.materials], "i")
        me.mat_ev = p(np.array([mt.evs if mt.evs is not None else (0, 0, 0) for mt in m.materials],
                               dtype=np.float64).reshape(-1), "f")
        me.mat_eev_coef = p([mt.eev_coef for mt in m.materials], "f")
        me.mat_coriolis = p([mt.coriolis for mt in m.materials], "f")


def make_params(m: SW2Model, precision: int = SW2GPU_FP64, precond: int = SW2GPU_PREC_BJACOBI,
                lin_rtol: float = 1e-5, lin_atol: float = 1e-10) -> Params:
    p = m.params
    out = Params()
    out.gravity, out.density, out.viscosity = p.gravity, p.density, p.viscosity
    out.drying_lower_limit = out.drying_upper_limit = p.drying_limit
    out.tau_temporal, out.tau_pg = p.tau_temporal, p.tau_pg
    out.tol_nonlin = p.tol_nonlin
    out.inc_nonlin = p.inc_nonlin if p.inc_nonlin is not None else UNSET_FLT
    out.max_nonlin_it, out.max_lin_it = p.max_nonlin_it, p.max_lin_it
    out.max_linesearch_cuts = p.max_linesearch_cuts
    out.precision, out.precond = precision, precond
    out.lin_rtol, out.lin_atol = lin_rtol, lin_atol
    return out

"""Shared test helpers: the golden models and state loaders."""
import numpy as np

from adhv8_kraken_b200 import meshgen


def channel_model():
    return meshgen.channel()


def basin_model():
    return meshgen.bumpy_basin(700, seed=11, size=2000.0, nsteps=8, dt=5.0, nbins=3, name="basin")


def scale_model(nsteps=10):
    """The 1M-triangle benchmark basin's generator at 10k points (~20k triangles, the domain
    scaled like bench.py does, so the element size is the benchmark's)."""
    import math
    points = 10000
    return meshgen.bumpy_basin(points, seed=2024, size=20000.0 * math.sqrt(points / 5e5), nsteps=nsteps, dt=5.0,
                               name="scale")


def set_load_state(solver, model, ref, prefix="load0"):
    """Puts a solver (oracle or GPU) in the state the reference built its Jacobian at."""
    solver.set_state(0, ref[f"{prefix}_h"], ref[f"{prefix}_u"], ref[f"{prefix}_v"])
    solver.set_state(1, ref[f"{prefix}_h1"], ref[f"{prefix}_u1"], ref[f"{prefix}_v1"])
    solver.set_state(2, ref[f"{prefix}_h2"], ref[f"{prefix}_u2"], ref[f"{prefix}_v2"])
    t, dt = ref[f"{prefix}_t"]
    solver.set_dt(dt, model.series_values(t, t + dt))
    solver.set_wd(ref[f"{prefix}_wd"])


def fields(h, u, v):
    """Depth and unit discharge q = (uh, vh); used with field_errors()."""
    return {"h": h, "uh": h * u, "vh": h * v}


def field_errors(got, exp):
    """Relative errors per field: depth against max|h|; the unit-discharge field as a vector,
    max |q_got - q_exp| / max |q_exp| (its components alone can be round-off noise, e.g. vh
    in a straight channel)."""
    import numpy as np
    eh = float(np.abs(got["h"] - exp["h"]).max() / np.abs(exp["h"]).max())
    dq = np.hypot(got["uh"] - exp["uh"], got["vh"] - exp["vh"])
    qm = float(np.hypot(exp["uh"], exp["vh"]).max())
    return {"h": eh, "q": float(dq.max() / max(qm, 1e-300))}


def centroid_refine(m, elems):
    """The model `m` with each triangle of `elems` split at its centroid, as a refinement step of
    an adaption would: the triangle keeps its number as (a, b, new node), the two other parts and
    the new nodes are appended (node and triangle numbers kept).  The new node takes the mean
    bed, coordinates and hot-start state of the triangle's vertices."""
    import dataclasses
    import numpy as np
    x, y, z = list(m.x), list(m.y), list(m.z)
    h0, u0, v0 = list(m.h0), list(m.u0), list(m.v0)
    ns = list(m.node_string)
    tri = m.tri.copy()
    extra, extra_mat = [], []
    for e in elems:
        a, b, c = (int(q) for q in tri[e])
        k = len(x)
        for arr, src in ((x, m.x), (y, m.y), (z, m.z), (h0, m.h0), (u0, m.u0), (v0, m.v0)):
            arr.append((src[a] + src[b] + src[c]) / 3.0)
        ns.append(-1)
        tri[e] = (a, b, k)
        extra += [(b, c, k), (c, a, k)]
        extra_mat += [m.tri_mat[e]] * 2
    f = lambda a: np.asarray(a, dtype=np.float64)
    return dataclasses.replace(
        m, x=f(x), y=f(y), z=f(z), h0=f(h0), u0=f(u0), v0=f(v0),
        node_string=np.asarray(ns, dtype=np.int32),
        tri=np.concatenate([tri, np.asarray(extra, dtype=np.int32).reshape(-1, 3)]).astype(np.int32),
        tri_mat=np.concatenate([m.tri_mat, np.asarray(extra_mat, dtype=np.int32)]).astype(np.int32),
        name=m.name + "_refined")

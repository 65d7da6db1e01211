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

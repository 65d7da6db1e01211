"""Run the reference AdH executable (``oracle/_ref/adh_dump``) on an SW2 model.

Test infrastructure only (parity pin and CPU baseline).  The model is written as
AdH ``.2dm/.bc/.hot`` files, the executable runs its own time loop unmodified,
and the records appended by the observation harness (``oracle/ref/adh_dump.c``)
are parsed back into numpy arrays.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time
from typing import Dict, List

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "adh_dump")


def read_dump(path: str) -> List[tuple]:
    recs = []
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        tag = data[off:off + 8].rstrip(b"\0").decode()
        kind = int(np.frombuffer(data, np.int32, 1, off + 8)[0])
        cnt = int(np.frombuffer(data, np.int64, 1, off + 12)[0])
        off += 20
        dt = np.float64 if kind == 0 else np.int32
        arr = np.frombuffer(data, dt, cnt, off).copy()
        off += cnt * np.dtype(dt).itemsize
        recs.append((tag, arr))
    return recs


def parse(recs) -> Dict[str, list]:
    steps, loads, tloads = [], [], []
    i = 0
    while i < len(recs):
        tag, arr = recs[i]
        if tag == "step":
            hi = recs[i + 1][1]
            steps.append(dict(t=arr[0], dt=arr[1], seconds=float(arr[2]) if arr.size > 2 else 0.0,
                              newton_its=int(hi[0]), attempts=int(hi[1]),
                              h=recs[i + 2][1], u=recs[i + 3][1], v=recs[i + 4][1], wd=recs[i + 5][1]))
            i += 6
            if i < len(recs) and recs[i][0] == "mass":   # initial, current, error, accumulated flux
                m = recs[i][1]
                steps[-1].update(mass0=float(m[0]), mass=float(m[1]), mass_error=float(m[2]),
                                 mass_flux_total=float(m[3]))
                i += 1
            if i < len(recs) and recs[i][0] == "dacont":   # elem_rhs_dacont_extra_terms [3][T]
                steps[-1]["dacont"] = recs[i][1].reshape(3, -1)
                i += 1
            if i + 1 < len(recs) and recs[i][0] == "elemerr":   # adaption error indicator
                steps[-1]["elem_error"] = recs[i][1]
                steps[-1]["node_error"] = recs[i + 1][1]
                i += 2
                cerr = []
                while i < len(recs) and recs[i][0] == "conerr":   # the constituents' nodal indicator
                    cerr.append(recs[i][1])
                    i += 1
                if cerr:
                    steps[-1]["con_error"] = cerr
            cons = []
            while i < len(recs) and recs[i][0] == "con":        # constituent concentrations
                cons.append(recs[i][1])
                i += 1
            if cons:
                steps[-1]["con"] = cons
        elif tag == "tload":                                     # transport Jacobian build
            d = dict(itrn=int(arr[0]), t=arr[1], dt=arr[2])
            j = i + 1
            while j < len(recs) and recs[j][0] not in ("step", "load", "tload"):
                d[recs[j][0]] = recs[j][1]
                j += 1
            tloads.append(d)
            i = j
        elif tag == "load":
            d = dict(t=arr[0], dt=arr[1])
            j = i + 1
            while j < len(recs) and recs[j][0] not in ("step", "load", "tload"):
                d[recs[j][0]] = recs[j][1]
                j += 1
            loads.append(d)
            i = j
        else:
            i += 1
    return dict(steps=steps, loads=loads, tloads=tloads)


def run_reference(model, nsteps=None, loads: int = 0, workdir: str = None, timeout: float = 3600.0,
                  mass: bool = False, dacont: bool = False, error: bool = False, tloads: int = 0):
    """Run the reference on ``model``; returns parsed records and the wall time (s).  mass: also
    record the reference's grid mass diagnostics after every step; dacont: its transport side
    output elem_rhs_dacont_extra_terms; error: its adaption error indicator (elem_error per
    element and its nodal average); tloads: the inputs and results of the first `tloads`
    transport Jacobian builds.  A model with constituents records their concentrations after
    every step."""
    if not os.path.exists(EXE):
        raise FileNotFoundError("oracle/_ref/adh_dump is not built (python oracle/ref/build_ref.py)")
    tmp = workdir or tempfile.mkdtemp(prefix="adhref_")
    try:
        model.write_adh(tmp, "m", nsteps=nsteps)
        env = dict(os.environ, ADH_DUMP=os.path.join(tmp, "dump.bin"), ADH_DUMP_LOADS=str(loads),
                   ADH_DUMP_TLOADS=str(tloads))
        if mass:
            env["ADH_DUMP_MASS"] = "1"
        if dacont:
            env["ADH_DUMP_DACONT"] = "1"
        if error:
            env["ADH_DUMP_ERROR"] = "1"
        t0 = time.perf_counter()
        r = subprocess.run([EXE, "m"], cwd=tmp, env=env, capture_output=True, text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stdout[-3000:]}\n{r.stderr[-2000:]}")
        out = parse(read_dump(os.path.join(tmp, "dump.bin")))
    finally:
        if workdir is None:   # a scratch directory of our own
            shutil.rmtree(tmp, ignore_errors=True)
    out["wall"] = wall
    out["stdout"] = r.stdout
    return out

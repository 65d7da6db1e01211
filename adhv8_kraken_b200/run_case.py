"""Runs the seeded basin workload for a few time steps and prints per-step statistics.

    python -m adhv8_kraken_b200.run_case --points 500000 --steps 2 [--precision fp64|mixed]
                                         [--variant JAC_MINB,STAGES] [--precond bjacobi|dilu] [--dt S]
                                         [--constituents N]

    python -m adhv8_kraken_b200.run_case --ensemble 16 --steps 5 [--precision fp64|mixed]
                                         [--rebalance ROUNDS,FRACTION]

One JSON line per step (Newton and Krylov iterations, device time per phase; with constituents,
the transport step's too).  ``--ensemble N`` instead runs the first N members of the batched
ensemble (the bench's seeds 7000, 7001, ...) in one continuous-batching engine, one JSON line
per tick (phase times, launches, instances iterating).  This is the command the kernel profiles are taken on: it runs the
same code path as ``bench.py`` without the timing legs around it, so a profiler sees only the
steps asked for.  ``--constituents N`` gives the basin N general constituents as ``bench.py``'s
transport leg does (0.3 initially, entering at 1.0 with the inflow, MP DF 0.5) and runs the
transport after every flow step.
"""
from __future__ import annotations

import argparse
import json
import math


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=500000)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--precond", choices=["bjacobi", "dilu"], default="bjacobi")
    ap.add_argument("--dt", type=float, default=5.0)
    ap.add_argument("--variant", default=None,
                    help="launch variant 'jac_minb,stages' (e.g. 1,3); default: the library's own")
    ap.add_argument("--constituents", type=int, default=0)
    ap.add_argument("--ensemble", type=int, default=0, help="run N ensemble members in one engine")
    ap.add_argument("--rebalance", default=None, help="engine Krylov rebalancing 'rounds,fraction'")
    a = ap.parse_args(argv)
    if a.ensemble:
        return run_ensemble(a)
    import numpy as np
    from . import capi, meshgen
    from .model import Constituent
    from .sw2 import SW2GPU

    size = 20000.0 * math.sqrt(a.points / 5e5)
    model = meshgen.bumpy_basin(a.points, seed=a.seed, size=size, nsteps=a.steps, dt=a.dt, name="basin")
    if a.constituents:
        ser = meshgen.const_series(model, 1.0)
        nmat = len(model.materials)
        model.constituents = [Constituent(ref_conc=1.0, diffusion=[0.5] * nmat, edge_bc={nmat: ser},
                                          c0=np.full(model.nnodes, 0.3)) for _ in range(a.constituents)]
    prec = capi.SW2GPU_FP64 if a.precision == "fp64" else capi.SW2GPU_MIXED
    pc = capi.SW2GPU_PREC_BJACOBI if a.precond == "bjacobi" else capi.SW2GPU_PREC_DILU
    g = SW2GPU(model, precision=prec, precond=pc)
    if a.variant:
        g.set_variant(*(int(x) for x in a.variant.split(",")))
    print(json.dumps({"triangles": model.nelems2d, "nodes": model.nnodes, "nnzb": g.nnzb}))
    for _ in range(a.steps):
        st = g.step()
        print(json.dumps({k: st[k] for k in ("status", "newton_its", "linear_its", "device_ms", "jac_ms",
                                             "krylov_ms", "resid_ms", "other_ms")}))
        if st["status"] != 0:
            raise SystemExit(f"step failed with status {st['status']}")
        if a.constituents:
            for k, t in enumerate(g.transport_step()):
                print(json.dumps({"constituent": k, **{q: t[q] for q in ("status", "newton_its", "linear_its",
                                                                        "device_ms", "jac_ms", "krylov_ms",
                                                                        "resid_ms", "other_ms")}}))
                if t["status"] != 0:
                    raise SystemExit(f"transport of constituent {k} failed with status {t['status']}")
    g.close()


def run_ensemble(a):
    from . import capi, meshgen
    from .sw2 import SW2Engine, SW2GPU
    prec = capi.SW2GPU_FP64 if a.precision == "fp64" else capi.SW2GPU_MIXED
    models = [meshgen.ensemble_member(7000 + i, nsteps=a.steps) for i in range(a.ensemble)]
    gs = [SW2GPU(m, precision=prec) for m in models]
    eng = SW2Engine(prec)
    if a.rebalance:
        r, f = a.rebalance.split(",")
        eng.set_rebalance(int(r), float(f))
    for g in gs:
        eng.add(g, a.steps)
    print(json.dumps({"instances": len(gs), "triangles": sum(m.nelems2d for m in models)}))
    done = []
    while eng.active:
        done += eng.tick()
        print(json.dumps(eng.last_tick()))
    eng.close()
    bad = [d for d in done if d["status"] != 0]
    print(json.dumps({"finished": len(done), "gave_up": len(bad), "failures": sum(d["failures"] for d in done)}))
    for g in gs:
        g.close()


if __name__ == "__main__":
    main()

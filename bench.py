"""Benchmark of the B200 SW2 Newton step (triangle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--points P]

Workload (one "step" = one implicit time step: FD Jacobian + block-Jacobi BiCGSTAB +
damped Newton, to the reference's convergence test): the plain FP64 drop-in at scale --
a seeded Delaunay basin of 500k points (~1M triangles) over 20 km x 20 km with 40
Gaussian bumps (dry tops, wet/dry fronts), log-normal Manning n, an inflow hydrograph
ramping 1 -> 5 m^2/s over 30 steps, dt = 5 s.  Data are synthetic (no dataset exists).

* ``value``  -- triangle-steps/s with the state resident in HBM, timed with CUDA events on
  the library's stream (max over ranks for N > 1; every rank runs its own replica).
* ``e2e``    -- the same through the C ABI with host buffers: every step uploads the two
  time levels a step reads (current and old) from pinned host memory and reads the new state
  back into pinned memory, as a drop-in for the reference's ``fe_sw2_solve`` would (the caller
  advances its levels by rotating its buffers).
* ``mixed``  -- the mixed-precision path on the same workload (FP32 Jacobian storage,
  SpMV and preconditioner inside the FP64 Newton loop) with its error against the FP64 run.
* ``transport`` -- the same basin carrying one general constituent: the flow step then the
  transport step (fe_transport) every step, the transport's phases and the roofline of its
  Krylov kernel.
* ``roofline`` -- the dominant kernel (largest device time in the timed region).
* ``cpu_baseline`` -- the reference AdH executable built from its own sources
  (``oracle/_ref``), timed on this host's cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SW2 triangle-steps/s at <=1e-8 rel err vs FP64, plain vs batched; p50/p99 latency"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons sampled during the timed region:
    NVML every 20 ms (read-only queries), else nvidia-smi every 200 ms."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []          # (sm_mhz, max_mhz, set of active reasons)
        self._stop = threading.Event()
        self._t = None

    def _run_nvml(self, nv):
        h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            try:
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.rows.append((float(sm), float(mx), {k for k, b in self.REASONS.items() if bits & b}))
            self._stop.wait(0.02)

    def _run_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                r = [c.strip() for c in out.split(",")]
                if len(r) >= 9 and r[1].replace(".", "").isdigit():
                    self.rows.append((float(r[1]), float(r[2]), {names[i] for i in range(4) if r[5 + i] == "Active"}))
            except Exception:
                pass
            self._stop.wait(0.2)

    def _run(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
        except Exception:
            nv = None
        if nv is None:
            self._run_smi()
            return
        try:
            self._run_nvml(nv)
        except Exception:
            self._run_smi()

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        time.sleep(0.05)
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(set().union(*[r[2] for r in self.rows])), "samples": len(self.rows)}


def basin_model(points: int, nsteps: int):
    from adhv8_kraken_b200 import meshgen
    size = 20000.0 * math.sqrt(points / 5e5)
    return meshgen.bumpy_basin(points, seed=2024, size=size, nsteps=nsteps, dt=5.0, name="basin")


def max_over_ranks(x: float, world: int, device="cpu") -> float:
    """Largest value of x over the ranks (the timed region of the slowest replica)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world: int, triangles: int, steps: int, ms_max: float) -> float:
    """Whole-job triangle-steps/s of `world` replicas, each `steps` steps of `triangles`,
    timed by the slowest rank."""
    return world * triangles * steps / (ms_max * 1e-3)


def _ensemble_member(args):
    seed, nsteps = args
    from adhv8_kraken_b200 import meshgen
    return meshgen.ensemble_member(seed, nsteps=nsteps)


def ensemble_models(n: int, nsteps: int, seed0: int = 7000, procs: int = 0):
    """The batched-ensemble instances (triangle count log-uniform 5k-200k, own bathymetry
    seed, Manning median U[0.015, 0.05], inflow peak U[1, 8], dt U[2, 10]), generated in a
    spawn-started process pool (before any CUDA work in this process)."""
    from multiprocessing import get_context
    procs = procs or max(1, min(32, (os.cpu_count() or 2) - 1))
    with get_context("spawn").Pool(procs) as pool:
        return pool.map(_ensemble_member, [(seed0 + i, nsteps) for i in range(n)])


def run_small(stream, steps: int = 20, warmup: int = 3):
    """Config-1 channel (4,000 triangles), where launches and host round trips are a large
    part of a step: direct launches, the step's Newton iterations replayed from CUDA graphs, and
    the whole step as one graph with the Newton loop's decisions on the device."""
    import torch
    from adhv8_kraken_b200 import meshgen
    from adhv8_kraken_b200.sw2 import SW2GPU
    m = meshgen.channel(nsteps=warmup + steps)
    out = {"workload": f"channel: {m.nelems2d} triangles, dt {m.dt} s, {steps} steps after {warmup}"}
    for name, graphs in (("direct", False), ("graphs", True), ("step_graph", 2)):
        g = SW2GPU(m, stream=stream.cuda_stream)
        g.set_graphs(graphs)
        for _ in range(warmup):
            g.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            st = g.step()
            assert st["status"] == 0
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        g.close()
        out[name] = {"value": m.nelems2d / (ms * 1e-3), "ms_per_step": ms}
    return out


def _serve_member(args):
    seed, nsteps = args
    from adhv8_kraken_b200 import meshgen
    return meshgen.ensemble_member(seed, tri_lo=1e4, tri_hi=2e6, nsteps=nsteps, name="req")


def serve_requests(n: int, horizon_scale: float, seed0: int = 9000, procs: int = 0):
    """Serving-loop requests: meshes with triangle count log-uniform 10k-2M and their own
    bathymetry / roughness / inflow / dt draws, horizons uniform 10..500 steps times
    `horizon_scale` (at least one step); generated in a spawn-started process pool."""
    from multiprocessing import get_context
    rng = np.random.Generator(np.random.PCG64(seed0))
    horizons = [max(1, int(round(int(rng.integers(10, 501)) * horizon_scale))) for _ in range(n)]
    procs = procs or max(1, min(32, (os.cpu_count() or 2) - 1))
    with get_context("spawn").Pool(procs) as pool:
        models = pool.map(_serve_member, [(seed0 + 1 + i, h) for i, h in enumerate(horizons)])
    return models, horizons


def run_serving(models, horizons, lam: float, seed: int = 1):
    """Config-5 legs: Poisson arrivals at rate lam (req/s) into the library's request server,
    FP64 and mixed on the same requests; per request the latency from submission to result,
    and the aggregate triangle-steps/s from the first submission to the last result."""
    from adhv8_kraken_b200 import capi
    from adhv8_kraken_b200.sw2 import SW2Server
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / lam, len(models))
    out = {}
    for name, prec in (("fp64", capi.SW2GPU_FP64), ("mixed", capi.SW2GPU_MIXED)):
        srv = SW2Server(prec, hbm_fraction=0.8)
        t0 = time.perf_counter()
        due = t0
        ids = []
        for m, h, gap in zip(models, horizons, gaps):
            due += gap
            time.sleep(max(0.0, due - time.perf_counter()))
            ids.append(srv.submit(m, h))
        res = [srv.wait(i) for i in ids]
        wall = time.perf_counter() - t0
        srv.close()
        st = [r[0] for r in res]
        lat = np.array([x["latency_ms"] for x in st])
        work = sum(m.nelems2d * x["steps"] for m, x in zip(models, st))
        out[name] = {"value": work / wall, "p50_ms": float(np.percentile(lat, 50)),
                     "p99_ms": float(np.percentile(lat, 99)), "mean_queue_ms": float(np.mean([x["queue_ms"] for x in st])),
                     "failed": int(sum(1 for x in st if x["status"] != 0)), "wall_s": wall}
    out["workload"] = (f"serving loop: {len(models)} requests, Poisson arrivals at {lam} req/s, triangles "
                       f"log-uniform 10k-2M (total {sum(m.nelems2d for m in models)}), horizons "
                       f"{min(horizons)}-{max(horizons)} steps (sum {sum(horizons)})")
    out["requests"] = len(models)
    out["rate_per_s"] = lam
    return out


# Krylov rebalancing of the engine legs (sw2gpu_engine_set_rebalance): up to 4 launches per
# batched solve, the instances still iterating paused once half a launch's CTAs are done
ENGINE_REBALANCE = (4, 0.5)


def run_ensemble(models, stream, steps: int):
    """Config-4 legs on the same instances, every instance running `steps` time steps (a failed
    step is retried with dt / 4 and counts as wasted time; dt doubles back toward the nominal
    one after every accepted step, the reference's tc_end; an instance still failing after 8
    reductions gives up):

    * plain FP64 -- each instance stepped alone, one after the other (the drop-in path);
    * batched FP64 and batched mixed -- all instances in one continuous-batching engine
      (sw2gpu_engine_*): each tick is one launch per Newton phase over every instance, an
      instance that finished a step starts its next one in the following tick.

    Throughput = sum over instances of triangles x completed steps / device time."""
    import torch
    from adhv8_kraken_b200 import capi
    from adhv8_kraken_b200.sw2 import SW2Engine, SW2Error, SW2GPU, run

    tri = np.array([m.nelems2d for m in models], dtype=np.float64)

    def reset(gs):
        for g in gs:
            h0, u0, v0 = g.model.initial_state()
            for lvl in range(3):
                g.set_state(lvl, h0, u0, v0)
            g.t = g.model.t0

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    gave_up = {"plain_fp64": 0}
    ends = {}   # instance -> (status, steps, model time) at the end of the last engine leg

    def alone(gs):
        # the reference's time loop per instance: a failed step is retried with dt / 4, and an
        # instance that still fails after 8 reductions gives up (as the engine's instances do)
        done = 0.0
        for k, g in enumerate(gs):
            ok = [0]
            try:
                run(g, steps, callback=lambda i, st, ok=ok: ok.__setitem__(0, ok[0] + 1))
            except SW2Error:
                gave_up["plain_fp64"] += 1
            done += tri[k] * ok[0]
        return done

    def engine(gs, precision):
        eng = SW2Engine(precision, stream=stream.cuda_stream)
        eng.set_rebalance(*ENGINE_REBALANCE)
        for g in gs:
            eng.add(g, steps)
        res, ph = [], {"jac_ms": 0.0, "krylov_ms": 0.0, "resid_ms": 0.0, "other_ms": 0.0}
        ends.clear()
        ticks = 0
        while eng.active:
            res += eng.tick()
            lt = eng.last_tick()
            for key in ph:
                ph[key] += lt[key]
            ticks += 1
        eng.close()
        by_id = {id(g): k for k, g in enumerate(gs)}
        done = sum(tri[by_id[d["id"]]] * d["steps"] for d in res)
        for d in res:
            ends[by_id[d["id"]]] = (d["status"], d["steps"], d["t"])
        ph["gave_up"] = sum(1 for d in res if d["status"] != 0)
        return done, sum(d["failures"] for d in res), ticks, ph

    def warm(gs, precision):
        eng = SW2Engine(precision, stream=stream.cuda_stream)
        for g in gs:
            eng.add(g, 1)
        eng.run()
        eng.close()
        reset(gs)

    out = {"krylov_rebalance": {"rounds": ENGINE_REBALANCE[0], "fraction": ENGINE_REBALANCE[1]}}
    g64 = [SW2GPU(m, precision=capi.SW2GPU_FP64, stream=stream.cuda_stream) for m in models]
    warm(g64, capi.SW2GPU_FP64)
    ms, done = timed(lambda: alone(g64))
    out["plain_fp64"] = {"value": float(done / (ms * 1e-3)), "ms": ms, "gave_up": gave_up["plain_fp64"]}
    plain_state = [g.get_state(0) for g in g64]
    reset(g64)
    ms, (done, fails, ticks, ph) = timed(lambda: engine(g64, capi.SW2GPU_FP64))
    out["batched_fp64"] = {"value": float(done / (ms * 1e-3)), "ms": ms, "failed_steps": int(fails), "ticks": ticks,
                           "phase_ms": ph}
    b64_state = [g.get_state(0) for g in g64]
    ends64 = dict(ends)
    out["batched_fp64"]["bitwise_equal_to_plain"] = bool(all(
        all(np.array_equal(x, y) for x, y in zip(a, c)) for a, c in zip(plain_state, b64_state)))
    for g in g64:
        g.close()
    gm = [SW2GPU(m, precision=capi.SW2GPU_MIXED, stream=stream.cuda_stream) for m in models]
    warm(gm, capi.SW2GPU_MIXED)
    ms, (done, fails, ticks, ph) = timed(lambda: engine(gm, capi.SW2GPU_MIXED))
    # error of every instance's final state against its batched FP64 run (h, uh, vh), over the
    # instances that completed their steps in both runs and reached the same model time (an
    # instance whose dt path differs, a retry in one precision only, ends elsewhere in time)
    per_inst, compared = [], []
    for k, (g, ref) in enumerate(zip(gm, b64_state)):
        e = _rel_errs(*g.get_state(0), *ref)
        per_inst.append(e)
        a, b = ends.get(k), ends64.get(k)
        if a and b and a[0] == 0 and b[0] == 0 and a[2] == b[2]:
            compared.append(k)
    worst = max(compared, key=lambda k: max(per_inst[k].values())) if compared else 0
    out["batched_mixed"] = {"value": float(done / (ms * 1e-3)), "ms": ms, "failed_steps": int(fails), "ticks": ticks,
                            "phase_ms": ph, "instances_compared": len(compared),
                            "max_rel_err_vs_fp64": {f: max((per_inst[k][f] for k in compared), default=None)
                                                    for f in ("h", "uh", "vh")},
                            "rel_err_vs_fp64_per_instance": {f: [float("%.2e" % per_inst[k][f]) if k in compared
                                                                 else None for k in range(len(per_inst))]
                                                             for f in ("h", "uh", "vh")}}
    for g in gm:
        g.close()
    # the worst instance traced step by step: it runs alone (an instance computes in the engine
    # exactly what it computes alone) in FP64 and mixed, and its error after every step
    m = models[worst]
    trace = {}
    for name, prec in (("fp64", capi.SW2GPU_FP64), ("mixed", capi.SW2GPU_MIXED)):
        g = SW2GPU(m, precision=prec, stream=stream.cuda_stream)
        states = []
        try:
            run(g, steps, callback=lambda k, st, g=g, states=states: states.append(g.get_state(0)))
        except SW2Error:
            pass
        g.close()
        trace[name] = states
    out["batched_mixed"]["worst_instance"] = {
        "index": worst, "triangles": int(m.nelems2d), "dt": float(m.dt),
        "rel_err_vs_fp64_per_step": [{f: float("%.3e" % v) for f, v in _rel_errs(*a, *b).items()}
                                     for a, b in zip(trace["mixed"], trace["fp64"])]}
    out["workload"] = (f"batched ensemble: {len(models)} seeded basins, triangles log-uniform 5k-200k "
                       f"(total {int(tri.sum())}), own bathymetry, Manning median U[0.015,0.05], inflow peak "
                       f"U[1,8] m^2/s, dt U[2,10] s; {steps} steps per instance")
    out["instances"] = len(models)
    out["triangles"] = int(tri.sum())
    out["steps"] = steps
    return out


def _rel_errs(hm, um, vm, h64, u64, v64):
    """max |x - x_fp64| / max |x_fp64| for h, uh and vh (numpy or torch arrays)."""
    out = {}
    for name, a, b in (("h", hm, h64), ("uh", hm * um, h64 * u64), ("vh", hm * vm, h64 * v64)):
        d = abs(a - b).max()
        r = abs(b).max()
        out[name] = float(d) / max(float(r), 1e-300)
    return out


def run_config3(stream, points: int, steps: int):
    """Config 3: the mixed path at ~4M triangles (the 1M basin's generator at 2M points, the
    domain scaled to keep the element size), `steps` steps of 5 s, against the plain FP64 path on
    the same mesh step by step: the max relative h / uh / vh error per step.  The CPU reference
    cannot run this size (about a day for 50 steps on one core), so the FP64 GPU path -- pinned
    to the reference within 1e-10 per step on the same generator at 20k triangles -- is the FP64
    reference here.  Each leg snapshots its state into device memory after every step
    (sw2gpu_snapshot, 48 MB per step at 2M nodes, inside the timed region)."""
    import torch
    from adhv8_kraken_b200 import capi
    from adhv8_kraken_b200.sw2 import SW2GPU, run
    m = basin_model(points, steps + 8)
    T, V = m.nelems2d, m.nnodes
    dev = torch.device("cuda", torch.cuda.current_device())
    snaps, out = {}, {}
    for name, prec in (("fp64", capi.SW2GPU_FP64), ("mixed", capi.SW2GPU_MIXED)):
        g = SW2GPU(m, precision=prec, stream=stream.cuda_stream)
        variant = g.autotune()
        buf = torch.empty((steps, 3, V), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []

        def keep(k, st, g=g, buf=buf, stats=stats):
            stats.append(st)
            g.snapshot(0, buf[k, 0].data_ptr(), buf[k, 1].data_ptr(), buf[k, 2].data_ptr())
        e0.record(stream)
        run(g, steps, callback=keep)   # the reference's retry rule, should a step fail
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        g.close()
        snaps[name] = buf
        out[name] = {"value": T * steps / (ms * 1e-3), "ms_per_step": ms / steps,
                     "newton_its_per_step": sum(st["newton_its"] for st in stats) / steps,
                     "krylov_its_per_step": sum(st["linear_its"] for st in stats) / steps,
                     "dt_per_step": sorted(set(float(st["dt"]) for st in stats)),
                     "_dts": [float(st["dt"]) for st in stats],
                     "variant": {"jac_minb": variant[0], "krylov_stages": variant[1]}}
    a, b = snaps["mixed"], snaps["fp64"]
    out["same_dt_path"] = bool(out["mixed"].pop("_dts") == out["fp64"].pop("_dts"))
    per = {"h": [], "uh": [], "vh": []}
    for k in range(steps):
        e = _rel_errs(a[k, 0], a[k, 1], a[k, 2], b[k, 0], b[k, 1], b[k, 2])
        for f in per:
            per[f].append(float("%.3e" % e[f]))
    del snaps, a, b
    torch.cuda.empty_cache()
    out["max_rel_err_vs_fp64_per_step"] = per
    out["max_rel_err_vs_fp64"] = {f: max(v) for f, v in per.items()}
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["workload"] = (f"mixed precision at scale: the 1M basin's generator at {points} points, {T} triangles, "
                       f"{V} nodes, {steps} steps of 5 s from the hot start, FP64 and mixed on the same mesh")
    out["triangles"], out["nodes"], out["steps"] = T, V, steps
    return out


def cpu_reference_sample(points: int = 10000, steps: int = 4, procs: int = 1, timeout: float = 600.0):
    """Runs the reference executable on `procs` seeded instances concurrently (one per
    core); returns aggregate triangle-steps/s over the time-loop seconds of each run."""
    from adhv8_kraken_b200 import meshgen
    from oracle.ref_run import EXE, parse, read_dump
    if not os.path.exists(EXE):
        return None
    runs = []
    for r in range(procs):
        m = meshgen.bumpy_basin(points, seed=7000 + r, size=20000.0 * math.sqrt(points / 5e5), nsteps=steps,
                                dt=5.0, name="refsample")
        d = tempfile.mkdtemp(prefix="adhref_")
        m.write_adh(d, "m", nsteps=steps)
        env = dict(os.environ, ADH_DUMP=os.path.join(d, "dump.bin"), ADH_DUMP_LOADS="0")
        runs.append((m, d, subprocess.Popen([EXE, "m"], cwd=d, env=env, stdout=subprocess.DEVNULL,
                                            stderr=subprocess.DEVNULL)))
    tri_steps, secs = 0.0, []
    try:
        for m, d, p in runs:
            p.wait(timeout=timeout)
            out = parse(read_dump(os.path.join(d, "dump.bin")))
            s = sum(st["seconds"] for st in out["steps"])
            tri_steps += m.nelems2d * len(out["steps"])
            secs.append(s)
    finally:
        for _, d, p in runs:   # the runs' input decks and dumps are scratch
            if p.poll() is None:
                p.kill()
                p.wait()
            shutil.rmtree(d, ignore_errors=True)
    elapsed = max(secs)
    return {"value": tri_steps / elapsed, "tri_steps": tri_steps, "seconds": elapsed,
            "triangles": runs[0][0].nelems2d, "steps": steps, "procs": procs, "op_blk": runs[0][0].params.nblock}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    procs = os.cpu_count() or 1
    res = cpu_reference_sample(points=args.ref_points, steps=max(1, args.steps), procs=procs)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/adh_dump is not built"}))
        return
    line = {
        "metric": METRIC, "value": res["value"], "unit": "triangle-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / res["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"reference AdH executable (serial C, profile-LU block-Jacobi BiCGSTAB) on "
                               f"{procs} concurrent seeded basins of {res['triangles']} triangles, "
                               f"{res['steps']} steps each (bounded sample of the 1M-triangle workload)",
                   "op_blk": res["op_blk"]},
        "cpu_baseline": {"value": res["value"], "unit": "triangle-steps/s", "cores": procs, "kind": "reference",
                         "sample": f"{procs} x {res['triangles']} triangles x {res['steps']} steps, OP BLK {res['op_blk']}",
                         "op_blk": res["op_blk"]},
        "e2e": {"value": res["value"], "unit": "triangle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def transport_model(points: int, nsteps: int):
    """The benchmark basin carrying one general constituent: 0.3 everywhere at the start, entering
    at 1.0 with the inflow (NB TRN), diffusion 0.5 m^2/s on every material (MP DF)."""
    from adhv8_kraken_b200 import meshgen
    from adhv8_kraken_b200.model import Constituent
    m = basin_model(points, nsteps)
    ser = meshgen.const_series(m, 1.0)
    nmat = len(m.materials)
    m.constituents = [Constituent(ref_conc=1.0, diffusion=[0.5] * nmat, edge_bc={nmat: ser},
                                  c0=np.full(m.nnodes, 0.3))]
    return m


def run_transport(args, stream, variant, hbm, src):
    """Flow and transport steps on the benchmark basin with one constituent: triangle-steps/s of
    both, the transport's share and phases, and the roofline of the transport Krylov kernel
    (k_trn_bicgstab).  Its algorithmic bytes per iteration: two sweeps over the off-diagonal
    pattern (8 B value + 4 B column per entry, 4 B row pointer per row) and 20 vector streams of one
    double per node (sweep 1: r, q, rhat in, p, Ar, v out; sweep 2: r, v, Ar, rhat in, s, t out;
    update: x, p, s, t, v in, x, r, q out)."""
    import torch
    from adhv8_kraken_b200 import capi
    from adhv8_kraken_b200.sw2 import SW2GPU
    m = transport_model(args.points, args.warmup + args.steps + 8)
    T, V = m.nelems2d, m.nnodes
    g = SW2GPU(m, precision=capi.SW2GPU_FP64, stream=stream.cuda_stream)
    g.set_variant(*variant)
    for _ in range(args.warmup):
        assert g.step()["status"] == 0
        assert g.transport_step()[0]["status"] == 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fl, tr = [], []
    e0.record(stream)
    for _ in range(args.steps):
        fl.append(g.step())
        tr.append(g.transport_step()[0])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    assert all(s["status"] == 0 for s in fl + tr)
    c = g.get_conc(0)
    nnzb = g.nnzb
    g.close()
    k = args.steps
    kry = sum(t["krylov_ms"] for t in tr)
    lin = sum(t["linear_its"] for t in tr)
    iter_bytes = 2 * ((nnzb - V) * 12 + (V + 1) * 4) + 20 * 8 * V
    achieved = iter_bytes * lin / (kry * 1e-3) / 1e9 if kry > 0 else None
    return {"workload": f"the benchmark basin ({T} triangles) with one constituent (NB TRN inflow 1.0, "
                        f"MP DF 0.5, 0.3 initially), flow then transport every step, dt 5 s",
            "value": T * k / (ms * 1e-3), "unit": "triangle-steps/s", "ms_per_step": ms / k,
            "flow_ms_per_step": sum(f["device_ms"] for f in fl) / k,
            "transport_ms_per_step": sum(t["device_ms"] for t in tr) / k,
            "transport_newton_its_per_step": sum(t["newton_its"] for t in tr) / k,
            "transport_krylov_its_per_step": lin / k,
            "transport_phase_ms_per_step": {"jacobian": sum(t["jac_ms"] for t in tr) / k, "krylov": kry / k,
                                            "residual": sum(t["resid_ms"] for t in tr) / k,
                                            "other": sum(t["other_ms"] for t in tr) / k},
            "transport_launches_per_step": sum(t["kernel_launches"] for t in tr) / k,
            "krylov_roofline": {"kernel": "k_trn_bicgstab", "bound": "hbm", "achieved": achieved, "peak": hbm,
                                "unit": "GB/s", "frac": achieved / hbm if achieved else None, "peak_source": src,
                                "algorithmic_bytes_per_iteration": iter_bytes,
                                "us_per_iteration": 1e3 * kry / max(lin, 1)},
            "conc_range": [float(c.min()), float(c.max())]}


def run_ours(args, rank, world, local_rank, ens_models=None, serve=None):
    import torch
    import torch.distributed as dist
    from adhv8_kraken_b200 import capi
    from adhv8_kraken_b200.sw2 import SW2GPU

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(device=dev)
    model = basin_model(args.points, args.warmup + args.steps + 8)
    T, V = model.nelems2d, model.nnodes

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- plain FP64, state resident in HBM
    g = SW2GPU(model, precision=capi.SW2GPU_FP64, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        st = g.step()
        assert st["status"] == 0, st
    variant64 = g.autotune()   # launch variants change speed only, never results
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            stats.append(g.step())
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    assert all(s["status"] == 0 for s in stats), [s["status"] for s in stats]
    ms = max_over_ranks(ms, world, dev)
    value = replica_throughput(world, T, args.steps, ms)
    h64 = g.get_state(0)

    # ---- dominant kernel and its roofline
    jac = sum(s["jac_ms"] for s in stats)
    kry = sum(s["krylov_ms"] for s in stats)
    res = sum(s["resid_ms"] for s in stats)
    newton = sum(s["newton_its"] for s in stats)
    lin = sum(s["linear_its"] for s in stats)
    nnzb = g.nnzb
    hbm, src = peaks()
    # algorithmic bytes per launch.  FD Jacobian: element inputs + node state + 81 outputs per
    # triangle.  BiCGSTAB on the folded operator (block-Jacobi inverse multiplied into the
    # off-diagonal blocks, identity diagonal): per iteration two sweeps over the nnzb - V
    # off-diagonal blocks (72 B values + 4 B column) and the row pointers, plus 16 vector
    # streams of 3 doubles per node (sweep 1: q, p in, Ap out; sweep 2: r, Ap, q in, As out;
    # update: r, Ap, u, p, As in, u, r, p, best-u out).  Per launch once: b' and the inverses
    # in, b and u out (prologue), one more sweep with b, u in and r, q, p, Ap out, and the
    # exit pass (u and S in, state in and out, solution out).
    jac_bytes = T * (3 * 4 + 7 * 8 + 4 + 4 + 1) + V * 12 * 8 + T * 81 * 8
    sweep_bytes = (nnzb - V) * (9 * 8 + 4) + (V + 1) * 4
    kry_iter_bytes = 2 * sweep_bytes + V * 24 * 16
    kry_launch_bytes = V * (24 + 72 + 48) + sweep_bytes + V * 24 * 6 + V * (48 + 48 + 24)
    kernels = {
        "k_jac_elem": (jac, newton, jac_bytes),
        "k_bicgstab": (kry, newton, kry_iter_bytes * (lin / max(newton, 1)) + kry_launch_bytes),
    }
    name = max(kernels, key=lambda k: kernels[k][0])
    tot_ms, launches, bytes_per_launch = kernels[name]
    per_launch_ms = tot_ms / max(launches, 1)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    # measured DRAM traffic of the Krylov kernel: bytes per BiCGSTAB iteration and node from one
    # ncu capture of a smaller basin of the same generator (profiles/traffic_k_bicgstab_basin_
    # 600k_tri.md), times this run's nodes and mean iterations per launch (the sweeps' and the
    # vectors' bytes grow in proportion to both)
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic_k_bicgstab_basin_600k_tri.md")
    if name == "k_bicgstab" and os.path.exists(tf):
        with open(tf) as f:
            for ln in f:
                if ln.startswith("k_bicgstab_bytes_per_iteration_per_node:"):
                    traffic = float(ln.split(":")[1]) * V * (lin / max(newton, 1))
    roofline = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": src, "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch, "ms_per_launch": per_launch_ms,
                "share_of_step": tot_ms / ms}

    # ---- e2e through the C ABI with host buffers (drop-in semantics)
    g.close()
    g = SW2GPU(model, precision=capi.SW2GPU_FP64, stream=stream.cuda_stream)
    g.set_variant(*variant64)
    for _ in range(args.warmup):
        g.step()
    # the caller's host state: three pinned (h, u, v) sets, two holding the current and old
    # levels and one receiving the new state; advancing the levels rotates the roles.  A step
    # reads only these two: it shifts current -> old -> older and overwrites the third level.
    pinned = [torch.empty(V, dtype=torch.float64, pin_memory=True) for _ in range(9)]
    bufs = [tuple(p.numpy() for p in pinned[3 * k:3 * k + 3]) for k in range(3)]
    for lvl in range(2):
        g.get_state(lvl, out=bufs[lvl])
    levels, spare = [0, 1], 2
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for lvl in range(2):
            g.set_state(lvl, *bufs[levels[lvl]])
        st = g.step()
        assert st["status"] == 0
        g.get_state(0, out=bufs[spare])
        # the caller's state advances: old <- current <- new
        levels, spare = [spare, levels[0]], levels[1]
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, world, dev)
    e2e = {"value": replica_throughput(world, T, args.steps, e2e_s * 1e3), "unit": "triangle-steps/s",
           "h2d_bytes_per_step": 6 * 8 * V, "d2h_bytes_per_step": 3 * 8 * V}
    g.close()

    # ---- mixed precision on the same workload and its error vs the FP64 run
    gm = SW2GPU(model, precision=capi.SW2GPU_MIXED, stream=stream.cuda_stream)
    for _ in range(args.warmup):
        gm.step()
    variant_mixed = gm.autotune()
    torch.cuda.synchronize()
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m0.record(stream)
    mstats = [gm.step() for _ in range(args.steps)]
    m1.record(stream)
    torch.cuda.synchronize()
    mms = m0.elapsed_time(m1)
    hm = gm.get_state(0)
    gm.close()
    # depth error relative to max|h|; unit discharge q = (uh, vh) as a vector field
    err = {"h": float(np.abs(hm[0] - h64[0]).max() / np.abs(h64[0]).max())}
    dq = np.hypot(hm[0] * hm[1] - h64[0] * h64[1], hm[0] * hm[2] - h64[0] * h64[2])
    err["q"] = float(dq.max() / max(np.hypot(h64[0] * h64[1], h64[0] * h64[2]).max(), 1e-300))
    mixed = {"value": world * T * args.steps / (mms * 1e-3), "ms_per_step": mms / args.steps,
             "variant": {"jac_minb": variant_mixed[0], "krylov_stages": variant_mixed[1]},
             "max_rel_err_vs_fp64": err, "newton_its": sum(s["newton_its"] for s in mstats),
             "linear_its": sum(s["linear_its"] for s in mstats)}

    # ---- constituent transport on the same workload (fe_transport after every flow step)
    transport = run_transport(args, stream, variant64, hbm, src) if world == 1 else None

    # ---- batched ensemble (plain FP64 alone vs batched FP64 vs batched mixed)
    batched = None
    if ens_models:
        batched = run_ensemble(ens_models, stream, args.ens_steps)
    small = run_small(stream) if world == 1 else None
    config3 = run_config3(stream, args.c3_points, args.c3_steps) if (world == 1 and args.c3_points > 0) else None
    serving = None
    if serve:
        serving = run_serving(serve[0], serve[1], args.serve_rate)
        if args.serve_rates:   # the same requests at each arrival rate of the sweep
            serving["sweep"] = [run_serving(serve[0], serve[1], float(r)) for r in args.serve_rates.split(",")]
            for leg in serving["sweep"]:
                leg.pop("workload", None)

    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu:
        cpu_res = cpu_reference_sample(points=args.ref_points, steps=3, procs=1)
        if cpu_res:
            cpu = {"value": cpu_res["value"], "unit": "triangle-steps/s", "cores": 1, "kind": "reference",
                   "sample": f"reference AdH executable, one seeded basin of {cpu_res['triangles']} triangles "
                             f"from the same generator, 3 steps, OP BLK {cpu_res['op_blk']}, time loop only "
                             f"({cpu_res['seconds']:.1f} s)", "op_blk": cpu_res["op_blk"]}
    line = {
        "metric": METRIC, "value": value, "unit": "triangle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"plain FP64 SW2 drop-in at scale: seeded Delaunay basin, {T} triangles, "
                               f"{V} nodes, 40 bumps with dry tops, inflow ramp 1->5 m^2/s, dt 5 s",
                   "triangles": T, "nodes": V, "nnzb": nnzb, "precision": "fp64",
                   "l2": "inputs larger than L2 (BCSR alone is %.0f MB)" % (nnzb * 72 / 1e6),
                   "parallelism": f"replicas{world}",
                   "variant": {"jac_minb": variant64[0], "krylov_stages": variant64[1]}},
        "newton_its_per_step": newton / args.steps, "krylov_its_per_step": lin / args.steps,
        "phase_ms_per_step": {"jacobian": jac / args.steps, "krylov": kry / args.steps,
                              "residual": res / args.steps,
                              "other": (ms - jac - kry - res) / args.steps},
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "clocks": clk.summary(),
        "roofline": roofline,
        "e2e": e2e,
        "mixed": mixed,
        "transport": transport,
        "small": small,
        "config3": config3,
        "batched": batched,
        "serving": serving,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=500000)
    ap.add_argument("--ref-points", type=int, default=10000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ens", type=int, default=256, help="batched-ensemble instances (0: skip the leg)")
    ap.add_argument("--ens-steps", type=int, default=50, help="time steps per ensemble instance")
    ap.add_argument("--c3-points", type=int, default=2000000,
                    help="config-3 mixed-precision leg: basin points (~2x triangles; 0: skip the leg)")
    ap.add_argument("--c3-steps", type=int, default=50, help="config-3 time steps")
    ap.add_argument("--serve", type=int, default=24, help="serving-loop requests (0: skip the leg)")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--serve-rates", default="",
                    help="comma-separated arrival rates (req/s) of an extra serving sweep, e.g. 5,10,20,50,100,200")
    ap.add_argument("--serve-horizon-scale", type=float, default=0.1,
                    help="horizons U{10..500} steps times this factor (1.0: the full horizons)")
    args = ap.parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: launch the ranks (torchrun on this node, rendezvous on 127.0.0.1)
        # and let their rank 0 print the line
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        sys.stderr.write(f"bench.py: --gpus {args.gpus} but WORLD_SIZE is {world}: run one rank per GPU "
                         f"(torchrun --nproc-per-node {args.gpus}) or drop --gpus\n")
        sys.exit(2)
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if world > 1:
        args.ens = 0   # the ensemble legs are a single-GPU measurement
    ens = ensemble_models(args.ens, nsteps=args.ens_steps,
                          procs=max(1, ((os.cpu_count() or 2) - 1) // world)) if args.ens > 0 else None
    serve = None
    if world == 1 and args.serve > 0:
        serve = serve_requests(args.serve, args.serve_horizon_scale)
    try:
        run_ours(args, rank, world, local_rank, ens, serve)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

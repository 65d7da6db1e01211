"""The drop-in, end to end: the reference's own executable and time loop with its SW2 solve bound
to the B200 library.

``oracle/_ref/adh_gpu`` is the reference AdH built from its own sources with
``adhv8_kraken_b200/adapter/fe_sw2_solve_gpu.c`` linked in place of ``fe_sw2_solve``
(``--wrap=fe_sw2_solve``; ``oracle/ref/build_ref.py``).  Each of the reference's SW2 QA decks on
triangles (staged by the build into ``oracle/_ref/qa``) runs through it and through the unmodified
reference executable ``oracle/_ref/adh_dump``, both recording the state after every accepted
step.  The GPU run must follow the reference step for step -- the same number of accepted
steps and dt retries, Newton iterations within +-1, the state within the deck's tolerance
below -- and its own error report (error.out, written by the reference's TEST module against
the analytic solution) must read like the reference run's and like the stored error.out.last.

Tolerances.  The state is compared per step (depth against max |h|, unit discharge as a vector
field against the largest discharge of the reference run).  The plain FP64 GPU path matches the reference to
1e-10 per step where Newton converges tightly; the QA decks set their own Newton tolerance
(IP NTL up to 1e-4), and two solves that both stop below a loose tolerance can differ by what
that tolerance allows (the reference's last Newton increment comes from an exact block LU, the
GPU's from an inexact Krylov solve).  So each deck's state bound follows its IP NTL:
1e-10 for NTL <= 1e-8, otherwise 100 x NTL (relative).  The error-report numbers are error
measures against analytic solutions; a state difference of e (relative to the field) moves them
by at most about e times the field's magnitude, so they are compared to an absolute 1e-6 plus
1e-4 relative.  Words (PASS / FAIL, labels) must be identical."""
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import field_errors, fields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
GPU_EXE = os.path.join(REF, "adh_gpu")
CPU_EXE = os.path.join(REF, "adh_dump")
QA = os.path.join(REF, "qa")
# the reference's SW2 QA decks on triangles (wet_dry and angle_wind run with a wind series,
# MP WND STR 0; angle_wave with the radiation stresses of its hot file)
CASES = ["wet_dry", "angle_nb", "angle_source", "angle_dam", "angle_coriolis", "angle_wind", "angle_wave"]
NUM = re.compile(r"[-+]?\d+\.\d*(?:[eE][-+]?\d+)?|[-+]?\d+[eE][-+]?\d+")


def _ntl(bc_path):
    with open(bc_path) as f:
        for ln in f:
            w = ln.split()
            if len(w) >= 3 and w[0] == "IP" and w[1] == "NTL":
                return float(w[2])
    return 1e-8


def _run(exe, case, model=None):
    """Runs exe on a scratch copy of a staged QA deck (or on `model` written as a deck); returns
    (per-step records, error.out lines or None, error.out.last lines or None, IP NTL)."""
    from oracle.ref_run import parse, read_dump
    work = tempfile.mkdtemp(prefix=f"dropin_{case}_")
    try:
        run = os.path.join(work, case)
        if model is None:
            shutil.copytree(os.path.join(QA, case), run)
            (deck,) = [f[:-3] for f in os.listdir(run) if f.endswith(".bc")]
        else:
            deck = "m"
            model.write_adh(run, deck)
        env = dict(os.environ, ADH_DUMP=os.path.join(run, "dump.bin"), ADH_DUMP_LOADS="0")
        r = subprocess.run([exe, deck], cwd=run, env=env, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, (exe, r.stdout[-3000:], r.stderr[-2000:])
        steps = parse(read_dump(os.path.join(run, "dump.bin")))["steps"]
        report = stored = None
        if model is None:
            with open(os.path.join(run, "error.out")) as fh:
                report = [ln for ln in fh.read().splitlines() if ln.strip()]
            with open(os.path.join(run, "error.out.last")) as fh:
                stored = [ln for ln in fh.read().splitlines() if ln.strip()]
        return steps, report, stored, _ntl(os.path.join(run, deck + ".bc"))
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _compare_trajectories(case, gpu_steps, ref_steps, tol):
    """Accepted steps one for one: the same model times, dt and attempts (dt retries), Newton
    iterations within +-1 per attempt, the state within tol.  Depth is measured against the
    step's max |h|; unit discharge against the largest discharge of the reference run (a deck
    that settles to rest, like angle_wave, ends with a vanishing discharge field whose own
    maximum would turn round-off into a large relative number)."""
    assert len(gpu_steps) == len(ref_steps), (len(gpu_steps), len(ref_steps))
    qpeak = max(float(np.hypot(r["h"] * r["u"], r["h"] * r["v"]).max()) for r in ref_steps)
    worst = {"h": 0.0, "q": 0.0}
    for k, (g, r) in enumerate(zip(gpu_steps, ref_steps)):
        assert g["t"] == r["t"] and g["dt"] == r["dt"], (k, g["t"], r["t"], g["dt"], r["dt"])
        assert g["attempts"] == r["attempts"], k
        assert abs(g["newton_its"] - r["newton_its"]) <= max(1, r["attempts"]), (k, g["newton_its"], r["newton_its"])
        fg, fr = fields(g["h"], g["u"], g["v"]), fields(r["h"], r["u"], r["v"])
        errs = {"h": field_errors(fg, fr)["h"],
                "q": float(np.hypot(fg["uh"] - fr["uh"], fg["vh"] - fr["vh"]).max()) / max(qpeak, 1e-300)}
        for f, e in errs.items():
            worst[f] = max(worst[f], e)
            assert e <= tol, (case, k, f, e, tol)
    return worst


def _split(line):
    return NUM.sub("#", line).split(), [float(x) for x in NUM.findall(line)]


def test_dropin_binary_binds_the_library():
    """The drop-in executable exists wherever the reference was built here, defines the
    --wrap binding of fe_sw2_solve and loads libsw2gpu.so (no GPU needed)."""
    if not os.path.exists(CPU_EXE):
        pytest.skip("reference executable not built")
    assert os.path.exists(GPU_EXE)
    syms = subprocess.run(["nm", GPU_EXE], capture_output=True, text=True).stdout
    assert re.search(r"\bT __wrap_fe_sw2_solve\b", syms)
    assert re.search(r"\bT fe_sw2_solve_gpu\b", syms)
    assert re.search(r"\bU sw2gpu_step\b", syms)
    deps = subprocess.run(["ldd", GPU_EXE], capture_output=True, text=True).stdout
    assert "libsw2gpu.so" in deps and "not found" not in deps


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_reference_time_loop_with_the_gpu_step_matches_the_reference(case):
    if not (os.path.exists(GPU_EXE) and os.path.isdir(os.path.join(QA, case))):
        pytest.fail("oracle/_ref/adh_gpu or the staged QA decks are missing (python oracle/ref/build_ref.py)")
    ref_steps, ref_report, stored, ntl = _run(CPU_EXE, case)
    gpu_steps, gpu_report, _, _ = _run(GPU_EXE, case)
    tol = 1e-10 if ntl <= 1e-8 else 100.0 * ntl
    worst = _compare_trajectories(case, gpu_steps, ref_steps, tol)
    print(f"{case}: {len(gpu_steps)} steps, worst per-step error h {worst['h']:.2e} q {worst['q']:.2e} (bound {tol:g})")
    _compare_reports(gpu_report, ref_report)
    # the stored report too, wherever the reference built here reproduces it (all but angle_wind,
    # whose stored transect error the reference's own run misses: 7.2e-6 FAIL against 3.5e-8 PASS)
    if _reports_agree(ref_report, stored):
        _compare_reports(gpu_report, stored)


def _reports_agree(a, b):
    return len(a) == len(b) and all(_split(x)[0] == _split(y)[0] and np.allclose(_split(x)[1], _split(y)[1],
                                                                                rtol=1e-4, atol=1e-6)
                                    for x, y in zip(a, b))


def _compare_reports(got, exp):
    assert len(got) == len(exp)
    for g, e in zip(got, exp):
        gw, gn = _split(g)
        ew, en = _split(e)
        assert gw == ew, (g, e)
        assert np.allclose(gn, en, rtol=1e-4, atol=1e-6), (g, e)


@pytest.mark.gpu
def test_retry_path_through_the_reference_time_loop_matches_the_reference():
    """Retry-path parity: the channel with a one-step inflow spike and at most 5 Newton iterations
    (meshgen.channel_spike).  In the reference the step that meets the spike fails twice and is
    retried with dt / 4 each time (tc_scale, src/fe/fe_newton.c:854-892), a later step fails once,
    and after every accepted step the time loop doubles dt back toward the nominal 10 s
    (tc_end, src/tools/tc_end.c:55-66), re-shifting the time levels on every attempt
    (src/fe/fe_main.c:353).  Through the drop-in the GPU step must take the same path: the
    same accepted steps, dt and attempts, and the state within 1e-10 every step."""
    if not os.path.exists(GPU_EXE):
        pytest.fail("oracle/_ref/adh_gpu is missing (python oracle/ref/build_ref.py)")
    from adhv8_kraken_b200 import meshgen
    m = meshgen.channel_spike()
    ref_steps, _, _, _ = _run(CPU_EXE, "spike", m)
    gpu_steps, _, _, _ = _run(GPU_EXE, "spike", m)
    assert sum(s["attempts"] for s in ref_steps) > len(ref_steps)   # the case does fail and retry
    worst = _compare_trajectories("spike", gpu_steps, ref_steps, 1e-10)
    print(f"spike: {len(gpu_steps)} steps, {sum(s['attempts'] for s in gpu_steps)} attempts, worst per-step "
          f"error h {worst['h']:.2e} q {worst['q']:.2e}")



@pytest.mark.gpu
@pytest.mark.parametrize("case", ["channel_transport", "basin_transport", "terms_transport"])
def test_transport_dropin_follows_the_reference(case):
    """The reference's time loop with its flow and its constituent transport on the device
    (fe_transport bound by --wrap=fe_transport to the library's transport step): the same accepted
    steps as the unmodified reference and every constituent's concentration within 1e-9 of the
    field's maximum after every step (the flow's own per-step differences, carried)."""
    from adhv8_kraken_b200 import meshgen
    from conftest import relerr
    m = getattr(meshgen, case)()
    ref_steps, _, _, _ = _run(CPU_EXE, case, model=m)
    gpu_steps, _, _, _ = _run(GPU_EXE, case, model=m)
    assert len(gpu_steps) == len(ref_steps) == m.nsteps
    for k, (a, b) in enumerate(zip(gpu_steps, ref_steps)):
        assert a["attempts"] == b["attempts"] == 1
        assert len(a["con"]) == len(b["con"]) == len(m.constituents)
        for j in range(len(m.constituents)):
            assert relerr(a["con"][j], b["con"][j]) <= 1e-9, (case, k, j)

"""Build the reference AdH executable from its own sources into ``oracle/_ref/``.

Test infrastructure only: the binary is the parity pin for the C restatement in
``oracle/sw2_oracle.c`` and the "reference" CPU baseline.  Nothing is copied out
of the reference tree and its build system is not used; the recipe is:

1. Three shim headers are derived with ``sed``-style substitutions into
   ``oracle/_ref/shim`` (the shipped headers have their struct includes, their
   globals and every prototype commented out):

   * ``type.h``   -- the ``//#include "s*.h"`` struct includes re-enabled, plus
     ``<stdbool.h>`` and ``ssuperModel.h``;
   * ``global_header.h`` -- the commented globals (``debug``, ``DEBUG_TIME``,
     ``screen_output``, ``test_case_flag``, ...) re-enabled;
   * ``fnctn.h``  -- every commented prototype re-enabled, plus ``fe_prototypes.h``.

   ``gcc -iquote``-style priority is obtained with ``-I<shim> -I-``, so the
   reference ``.c`` files compile in place with these headers in front.
2. The translation units listed by the CMake files of the serial SW2 build
   (``fe``, ``fe/sw2``, ``solver``, ``friction``, ``structs``, ``initio``, ...)
   are compiled with ``gcc -O2 -fcommon``; units that only serve MPI, PETSc,
   groundwater, sediment coupling or ADCIRC winds are left out.
3. The objects are linked with the observation harness ``adh_dump.c`` and
   ``--wrap=fe_main --wrap=fe_sw2_load --wrap=fe_transport_load`` into ``oracle/_ref/adh_dump``.
4. The same objects, the same harness and the drop-in binding of the B200 library
   (``adhv8_kraken_b200/adapter/fe_sw2_solve_gpu.c``, compiled against the reference's own
   headers) are linked with ``--wrap=fe_sw2_solve --wrap=ssw_2d_calculate_elem_error
   --wrap=fe_transport`` against ``libsw2gpu.so`` into ``oracle/_ref/adh_gpu``: the reference's
   own executable and time loop with its SW2 solve and its constituent transport replaced by the
   GPU's.  Only where the library is built.
5. The reference's SW2 QA decks that run on triangles (``qa/sw2/<case>/tri``: mesh, boundary
   cards, hot start and the stored ``error.out.last``) are staged into ``oracle/_ref/qa`` so
   that the drop-in can run them where the reference tree is absent.

Usage: ``python oracle/ref/build_ref.py [REFERENCE_SRC]``.  The reference's ``src`` directory
is the argument, else the environment variable ``ADH_REFERENCE_SRC``, else a checkout of the
reference beside this repository (``../reference/src`` from the repository root).  Re-running
only rebuilds missing objects.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.normpath(os.path.join(HERE, "..", "_ref"))
SUBDIRS = ["fe", "fe/sw2", "fe/sw3", "fe/ns3", "fe/sw_hybrid", "fe/diffusive_wave", "fe/transport",
           "fe/sediment", "debug", "elem", "turbulence", "initio", "solver", "tools", "messg", "friction",
           "grid", "columns", "structs", "meteor", "node", "main"]
EXCLUDE = ["petsc_test", "messg_arecv", "messg_barrier", "messg_pack", "messg_unpack", "messg_wait",
           "partition_", "elem/elem_hash_add_entry.c", "solv_coarse_solve", "fe_bedload", "adh_cpl_func",
           "pack_icnt", "pack_dcnt", "swindlib"]
STUBS = "void *mod_cstorm = 0;\n"


def _shims(src: str) -> str:
    shim = os.path.join(OUT, "shim")
    os.makedirs(shim, exist_ok=True)
    with open(os.path.join(src, "include", "type.h")) as f:
        t = f.read()
    t = "#include <stdbool.h>\n" + re.sub(r"^//#include", "#include", t, flags=re.M) + '\n#include "ssuperModel.h"\n'
    with open(os.path.join(shim, "type.h"), "w") as f:
        f.write(t)
    with open(os.path.join(src, "include", "global_header.h")) as f:
        g = f.read()
    g = re.sub(r"^//(int ROTATE|SDEBUG debug|double DEBUG_TIME|SSCREEN_OUTPUT|STESTCASE|double \*\*\*coupled"
               r"|int \*\*root_ids|double total_mass)", r"\1", g, flags=re.M)
    with open(os.path.join(shim, "global_header.h"), "w") as f:
        f.write(g)
    with open(os.path.join(src, "include", "fnctn.h")) as f:
        h = f.read()
    h = re.sub(r"^//", "", h, flags=re.M) + '\n#include "fe_prototypes.h"\n'
    with open(os.path.join(shim, "fnctn.h"), "w") as f:
        f.write(h)
    return shim


def _include_dirs(src: str):
    dirs = [os.path.join(src, d) for d in ("include", "structs", "debug/include")]
    for root, subdirs, _ in os.walk(src):
        rel = os.path.relpath(root, src)
        if any(rel.startswith(p) for p in ("NEW_ADH", "fe_new", "structs_new", "STAND_ALONE", "pt")):
            continue
        if "UMFPACK" in rel or "Cmake" in rel or "/." in root:
            continue
        dirs.append(root)
    return dirs


def _sources(src: str):
    srcs = []
    for d in SUBDIRS:
        with open(os.path.join(src, d, "CMakeLists.txt")) as f:
            lines = [ln for ln in f if not ln.lstrip().startswith("#")]
        for m in re.findall(r"[A-Za-z0-9_./]+\.c\b", "".join(lines)):
            rel = f"{d}/{m}"
            if any(x in rel for x in EXCLUDE):
                continue
            if os.path.exists(os.path.join(src, rel)):
                srcs.append(rel)
    return sorted(set(srcs))


REFERENCE_SRC = os.environ.get("ADH_REFERENCE_SRC") or os.path.normpath(
    os.path.join(HERE, "..", "..", "..", "reference", "src"))


def sources_present(src: str = REFERENCE_SRC) -> bool:
    return os.path.isdir(src)


def build(src: str = REFERENCE_SRC, jobs: int = os.cpu_count() or 4) -> str:
    exe = os.path.join(OUT, "adh_dump")
    if not os.path.isdir(src):
        if os.path.exists(exe):
            return exe
        raise FileNotFoundError(f"reference sources not found at {src}")
    shim = _shims(src)
    objdir = os.path.join(OUT, "obj")
    os.makedirs(objdir, exist_ok=True)
    flags = ["-O2", "-w", "-fcommon", f"-I{shim}", "-I-"] + [f"-I{d}" for d in _include_dirs(src)]

    def cc(rel):
        obj = os.path.join(objdir, rel.replace("/", "_")[:-2] + ".o")
        if not os.path.exists(obj):
            r = subprocess.run(["gcc", "-c"] + flags + [os.path.join(src, rel), "-o", obj],
                               capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"compile failed: {rel}\n{r.stderr[-2000:]}")
        return obj

    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(cc, _sources(src)))
    stub = os.path.join(OUT, "stubs.c")
    with open(stub, "w") as f:
        f.write(STUBS)
    harness = os.path.join(HERE, "adh_dump.c")
    hobj = os.path.join(objdir, "adh_dump.o")
    subprocess.run(["gcc", "-c"] + flags + [harness, "-o", hobj], check=True, capture_output=True)
    subprocess.run(["gcc", "-fcommon", "-o", exe] + objs + [hobj, stub, "-lm",
                    "-Wl,--wrap=fe_main", "-Wl,--wrap=fe_sw2_load", "-Wl,--wrap=fe_transport_load"], check=True)
    stage_qa(src)
    lib = os.path.join(REPO, "adhv8_kraken_b200", "libsw2gpu.so")
    if os.path.exists(lib):
        build_gpu_harness(flags, objs, hobj, stub, lib)
    return exe


REPO = os.path.normpath(os.path.join(HERE, "..", ".."))
GPU_EXE = os.path.join(OUT, "adh_gpu")
QA_CASES = ["wet_dry", "angle_nb", "angle_source", "angle_dam", "angle_coriolis", "angle_wind", "angle_wave"]


def build_gpu_harness(flags, objs, hobj, stub, lib) -> str:
    """The reference executable with fe_sw2_solve bound to the B200 library (step 4)."""
    adapter = os.path.join(REPO, "adhv8_kraken_b200", "adapter", "fe_sw2_solve_gpu.c")
    aobj = os.path.join(OUT, "obj", "fe_sw2_solve_gpu.o")
    subprocess.run(["gcc", "-c"] + flags + [f"-I{os.path.join(REPO, 'include')}", adapter, "-o", aobj], check=True)
    libdir = os.path.dirname(lib)
    rpath = "$ORIGIN/" + os.path.relpath(libdir, OUT)
    subprocess.run(["gcc", "-fcommon", "-o", GPU_EXE] + objs + [hobj, aobj, stub, f"-L{libdir}", "-lsw2gpu", "-lm",
                    f"-Wl,-rpath,{rpath}", "-Wl,--wrap=fe_main", "-Wl,--wrap=fe_sw2_load",
                    "-Wl,--wrap=fe_transport_load",
                    "-Wl,--wrap=fe_sw2_solve", "-Wl,--wrap=ssw_2d_calculate_elem_error", "-Wl,--wrap=fe_transport"],
                   check=True)
    return GPU_EXE


def stage_qa(src: str) -> str:
    """Copies the SW2 QA decks on triangles into oracle/_ref/qa/<case> (step 5)."""
    import shutil
    qa = os.path.normpath(os.path.join(src, "..", "qa", "sw2"))
    dst = os.path.join(OUT, "qa")
    for case in QA_CASES:
        d = os.path.join(dst, case)
        if os.path.isdir(os.path.join(qa, case, "tri")) and not os.path.isdir(d):
            shutil.copytree(os.path.join(qa, case, "tri"), d)
            os.chmod(d, 0o755)
            for f in os.listdir(d):
                os.chmod(os.path.join(d, f), 0o644)
    return dst


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else REFERENCE_SRC))

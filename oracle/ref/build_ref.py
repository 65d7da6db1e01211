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
   ``--wrap=fe_main --wrap=fe_sw2_load`` into ``oracle/_ref/adh_dump``.

Usage: ``python oracle/ref/build_ref.py [REFERENCE_SRC]`` (default
``/root/reference/src``).  Re-running only rebuilds missing objects.
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


REFERENCE_SRC = "/root/reference/src"


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
                    "-Wl,--wrap=fe_main", "-Wl,--wrap=fe_sw2_load"], check=True)
    return exe


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else REFERENCE_SRC))

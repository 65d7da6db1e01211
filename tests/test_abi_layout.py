"""The ctypes mirrors of the C ABI structs (adhv8_kraken_b200/capi.py) have the size and field
offsets of include/sw2gpu.h, as the C compiler lays them out: a host program compiled against
the header prints them and the test compares field by field (a mismatch would pass garbage
through every call without an error)."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from adhv8_kraken_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = [("sw2gpu_mesh", capi.Mesh), ("sw2gpu_params", capi.Params), ("sw2gpu_stats", capi.Stats),
           ("sw2gpu_run_stats", capi.RunStats), ("sw2gpu_request_stats", capi.RequestStats),
           ("sw2gpu_transport", capi.Transport)]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_structs_match_the_header():
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "sw2gpu.h"', "int main(void) {"]
    for cname, py in STRUCTS:
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'    printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["    return 0;", "}"]
    work = os.path.join(ROOT, "_build", "abi_layout")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    try:
        src, exe = os.path.join(work, "layout.c"), os.path.join(work, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        r = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe, src],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-2000:]
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    finally:
        shutil.rmtree(work, ignore_errors=True)
        try:
            os.rmdir(os.path.dirname(work))   # only if nothing else lives there
        except OSError:
            pass
    got = {}
    for ln in out:
        if ln:
            name, field, val = ln.split()
            got[(name, field)] = int(val)
    for cname, py in STRUCTS:
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)

"""The C ABI: the library builds for sm_100a, loads without a GPU and exports every
entry point that include/sw2gpu.h declares."""
import ctypes
import os
import re

from adhv8_kraken_b200 import build
from adhv8_kraken_b200.sw2 import LIB_PATH, SYMBOLS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "sw2gpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(sw2gpu_[a-z_0-9]+)\s*\(", text)))


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.samefile(path, LIB_PATH)
    ctypes.CDLL(path)


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(build.build())
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(SYMBOLS) == names


def test_abi_version_and_error_string():
    lib = ctypes.CDLL(build.build())
    assert lib.sw2gpu_abi_version() == 1
    lib.sw2gpu_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.sw2gpu_last_error(), bytes)


def test_create_rejects_null_arguments():
    lib = ctypes.CDLL(build.build())
    out = ctypes.c_void_p()
    assert lib.sw2gpu_create(None, None, None, ctypes.byref(out)) == 1

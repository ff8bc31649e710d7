"""The C ABI: header <-> ctypes layout, and every declared symbol exported by the library."""
import ctypes
import os
import re

import pytest

from pathtracerglsl_b200 import abi, _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ptx_rt.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(ptr_\w+)\s*\(", text, re.M)))


def test_struct_sizes_match_header():
    for name, size in abi.EXPECTED_SIZES.items():
        assert ctypes.sizeof(getattr(abi, name)) == size, name


def test_header_and_binding_declare_the_same_entry_points():
    assert declared_functions() == sorted(_native.SIGNATURES)


def test_library_exports_every_declared_symbol():
    from pathtracerglsl_b200 import build
    build.build()
    lib = ctypes.CDLL(build.LIB)   # loads without a GPU (the CUDA runtime is linked statically)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing
    assert lib.ptr_abi_version() == abi.ABI_VERSION

"""The C-ABI library: builds for sm_100a, loads, exports every entry point
declared in include/nicam_cuda.h (no compute call without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "nicam_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nc_[a-z_]+)\s*\(", src)))


def test_header_and_binding_agree(pkg):
    assert declared_functions() == sorted(pkg.EXPORTS)


def test_library_exports_all_symbols(pkg):
    from importlib import import_module
    build = import_module("pynicam-dc_b200.build")
    path = build.build()
    lib = ctypes.CDLL(path)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_create_without_gpu_fails_loudly(pkg, golden):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    geo, _ = golden
    with pytest.raises(pkg.NicamError):
        pkg.NicamCuda(geo)

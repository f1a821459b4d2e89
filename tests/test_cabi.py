"""The C-ABI library: builds for sm_100a, loads, exports every entry point
declared in include/*.h (the drop-in surface nicam_cuda.h and the test hooks
of nicam_cuda_debug.h; no compute call without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    import glob
    src = "".join(open(f).read() for f in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nc_[a-z0-9_]+)\s*\(", src)))


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


def test_history_item_ids_match_header(pkg):
    """the binding's history item order is the id list nc_history_vars documents"""
    import re
    hdr = open(os.path.join(ROOT, "include", "nicam_cuda.h")).read()
    doc = hdr[hdr.index("int nc_history_vars") - 2500:hdr.index("int nc_history_vars")]
    ids = {int(n): name for n, name in re.findall(r"\b(\d+) ((?:ml|sl)_\w+)", doc)}
    items = pkg.runtime.HIST_ITEMS
    for n, name in ids.items():
        assert items[n] == name, (n, name)
    assert len(items) == 45 and items[26:30] == ("sl_u850", "sl_v850", "sl_w850", "sl_t850")
    assert items[38:42] == ("sl_u100", "sl_v100", "sl_w100", "sl_t100")
    assert items[42:] == pkg.runtime.HIST_CHEM == ("sl_cl", "sl_cl2", "sl_cly")


def test_status_codes_map_to_exceptions(pkg):
    """a non-zero status becomes NicamError with the library's message;
    NC_ERR_NONFINITE (a NaN-seeded state found by nc_check_finite or a
    download) becomes NonFiniteStateError (no GPU: a stand-in library)"""
    class FakeLib:
        def __init__(self, msg):
            self.msg = msg

        def nc_last_error(self):
            return self.msg

    rt = pkg.runtime
    rt._check(0, FakeLib(b""))
    with pytest.raises(pkg.NonFiniteStateError, match="variable 5") as ei:
        rt._check(rt.NC_ERR_NONFINITE, FakeLib(b"nc_check_finite: non-finite value in prognostic variable 5"))
    assert ei.value.status == rt.NC_ERR_NONFINITE
    with pytest.raises(pkg.NicamError) as ei:
        rt._check(rt.NC_ERR_STATE, FakeLib(b"nc_step: no state uploaded"))
    assert not isinstance(ei.value, pkg.NonFiniteStateError) and ei.value.status == rt.NC_ERR_STATE

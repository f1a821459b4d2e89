import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    """the product package (its directory name is not a Python identifier)"""
    return importlib.import_module("pynicam-dc_b200")


@pytest.fixture(scope="session")
def golden():
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_trc.npz"))


@pytest.fixture(scope="session")
def golden_hs():
    """gl03 z10 with the reference's Held-Suarez forcing (make_hs.py): setup
    arrays (plus GRD_LAT at K0), the column latitudes and three states"""
    from make_golden import load
    geo, st = load(os.path.join(GOLDEN, "gl03_z10_hs.npz"))
    lat = geo.pop("GRD_LAT")
    return geo, lat, st


TRC_COORDS = ("GRD_LON", "GRD_LAT", "GRD_Z", "GRD_ZH", "GRD_LON_pl", "GRD_LAT_pl", "GRD_Z_pl", "GRD_ZH_pl")


@pytest.fixture(scope="session")
def golden_trcadv():
    """gl03 z10 DCMIP 1-1 offline tracer advection run by the reference
    (make_trcadv.py): setup arrays (including integ_type and the coordinates
    the prescribed winds read) and four states"""
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_trcadv.npz"))

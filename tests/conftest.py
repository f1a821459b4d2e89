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
def golden_warm():
    """gl03 z10 with RAIN_TYPE WARM (vapour, cloud and rain tracers in the
    thermodynamics), two steps of the reference (make_golden.py --case
    gl03_z10_warm)"""
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_warm.npz"))


@pytest.fixture(scope="session")
def golden_nlhdiff():
    """gl03 z10 with the NONLINEAR1 hyperdiffusion (Kh from the temperature
    Laplacian, clipped per level), two steps of the reference (make_golden.py
    --case gl03_z10_nlhdiff); the set-up carries hdiff_nl_kh_max,
    hdiff_nl_minlim and hdiff_nl_area"""
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_nlhdiff.npz"))


@pytest.fixture(scope="session")
def golden_rayleigh():
    """gl03 z10 with the Rayleigh sponge above 15 km, two steps of the
    reference (make_golden.py --case gl03_z10_rayleigh); the set-up carries
    rayleigh_coef, rayleigh_coef_h and rayleigh_only_w"""
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_rayleigh.npz"))


@pytest.fixture(scope="session")
def golden_kessler():
    """gl03 z10 RAIN_TYPE WARM with the reference's DCMIP forcing, Kessler
    microphysics only (make_kessler.py): setup arrays (GRD_Z the full-level
    heights), three states and the precipitation rate after each step"""
    import numpy as np
    from make_golden import load
    path = os.path.join(GOLDEN, "gl03_z10_kessler.npz")
    geo, st = load(path)
    d = np.load(path)
    return geo, st, {k: d[k] for k in d.files if k.startswith("precip")}


@pytest.fixture(scope="session")
def golden_kessler_chem():
    """the Kessler case with the reference's terminator toy chemistry as well
    (make_kessler.py --chem): Cl and Cl2 in tracers 3 and 4 (NCHEM_STR,
    NCHEM_END) away from their equilibrium, the column latitudes and
    longitudes (GRD_LAT, GRD_LON at K0, radians), three states and the
    precipitation after each step"""
    import numpy as np
    from make_golden import load
    path = os.path.join(GOLDEN, "gl03_z10_kessler_chem.npz")
    geo, st = load(path)
    d = np.load(path)
    return geo, st, {k: d[k] for k in d.files if k.startswith("precip")}


def _dcmip_fixture(name, vl=10):
    import numpy as np
    from make_golden import load
    path = os.path.join(GOLDEN, f"gl03_z{vl}_{name}.npz")
    geo, st = load(path)
    d = np.load(path)
    return geo, st, {k: d[k] for k in d.files if k.startswith("precip")}


@pytest.fixture(scope="session")
def golden_dcmip11():
    """the DCMIP2016 case 1-1 scheme set run by the reference
    (make_kessler.py --case dcmip11): Kessler, the simple physics with the
    latitude-dependent sea-surface temperature and no large-scale
    condensation, the terminator chemistry; set-up arrays with the
    half-level heights, surface height, column lat / lon and unit vectors"""
    return _dcmip_fixture("dcmip11")


@pytest.fixture(scope="session")
def golden_dcmip21():
    """the DCMIP2016 case 2-1 scheme set (moist Held-Suarez: Kessler, the
    simple physics with the Held-Suarez SST and exchange coefficient, the
    Held-Suarez relaxation on top) run by the reference
    (make_kessler.py --case dcmip21)"""
    return _dcmip_fixture("dcmip21")


@pytest.fixture(scope="session")
def golden_dcmip12bryan():
    """the DCMIP2016 case 1-2 (tropical cyclone) scheme set with the Bryan
    boundary layer run by the reference (make_kessler.py --case dcmip12bryan)"""
    return _dcmip_fixture("dcmip12bryan", 30)


@pytest.fixture(scope="session")
def golden_smdry():
    """the simple physics with RAIN_TYPE DRY (vapour the only water tracer) run
    by the reference (make_kessler.py --case smdry)"""
    return _dcmip_fixture("smdry")


@pytest.fixture(scope="session")
def golden_smlsc():
    """the simple physics alone with its large-scale condensation and the
    constant sea-surface temperature, run by the reference
    (make_kessler.py --case smlsc)"""
    return _dcmip_fixture("smlsc")


def dcmip_oracle_args(geo):
    """the oracle's forcing_step_kessler keywords for a DCMIP fixture"""
    fl = [int(x) for x in geo["dcmip_flags"]]
    chem = (geo["GRD_LAT"], geo["GRD_LON"], int(geo["NCHEM_STR"]), int(geo["NCHEM_END"])) \
        if "NCHEM_STR" in geo else None
    sm = dict(zh=geo["GRD_ZH"], zsfc=geo["GRD_zsfc"], lat=geo["GRD_LAT"], ij=geo["GMTR_p_IJ"],
              latdepend=bool(fl[2]), lsc=bool(fl[3]), held_suarez=bool(fl[4]), mitc=fl[5],
              bryan=bool(fl[6])) if fl[1] else None
    return dict(chem=chem, kessler_on=bool(fl[0]), sm=sm)


def dcmip_device_setup(geo):
    """the fixture's set-up with the DCMIP entries the device reads (GRD_LAT
    itself would be taken for the Held-Suarez latitudes)"""
    import numpy as np
    g = {k: v for k, v in geo.items() if k not in ("GRD_LAT", "GRD_LON", "GRD_ZH", "GRD_zsfc", "GMTR_p_IJ")}
    g["AF_dcmip_kessler"] = 1
    g["AF_dcmip_schemes"] = np.asarray(geo["dcmip_flags"], np.int64)
    if "NCHEM_STR" in geo:
        g["AF_dcmip_chem"] = np.asarray([int(geo["NCHEM_STR"]), int(geo["NCHEM_END"])], np.int64)
        g["AF_dcmip_lon"] = geo["GRD_LON"]
    if "GRD_LAT" in geo:
        g["AF_dcmip_lat"] = geo["GRD_LAT"]
    if "GRD_ZH" in geo:
        g["AF_dcmip_zh"], g["AF_dcmip_zsfc"], g["AF_dcmip_ij"] = geo["GRD_ZH"], geo["GRD_zsfc"], geo["GMTR_p_IJ"]
    return g


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


@pytest.fixture(scope="session")
def golden_trcadv12():
    """the same for DCMIP 1-2 (Hadley-like circulation; make_trcadv.py --case
    1-2): the setup also carries the key trcadv_case"""
    from make_golden import load
    return load(os.path.join(GOLDEN, "gl03_z10_trcadv12.npz"))


@pytest.fixture(scope="session")
def golden_hist():
    """the reference's own history diagnostics of the gl03_z10_trc run
    (make_hist.py): the extra setup they read (keys without the geo. prefix:
    GRD_Z, GRD_LAT, GRD_zsfc, GRD_dgz, GMTR_p_IJ, GMTR_area, constants, tracer
    indices), the outputs after step 2 (seeded after step 1) and the step
    counts and dt of the two calls"""
    import numpy as np
    z = np.load(os.path.join(GOLDEN, "gl03_z10_hist.npz"))
    hg = {k[4:]: z[k] for k in z.files if k.startswith("geo.")}
    out = {k[5:]: z[k] for k in z.files if k.startswith("hist.")}
    return hg, out


def hist_geo(geo: dict, hg: dict) -> dict:
    """the setup dict of a handle with history diagnostics: the fixture's
    arrays under the keys the backend's setup collects (``hist_*``)"""
    g = dict(geo)
    g.update(hist_hgt=hg["GRD_Z"], hist_lat=hg["GRD_LAT"], hist_zsfc=hg["GRD_zsfc"], hist_dgz=hg["GRD_dgz"],
             hist_area=hg["GMTR_area"], hist_IJ=hg["GMTR_p_IJ"])
    for k in ("LHV", "UNDEF", "PSAT0", "RTEM00", "CPovR_liq", "CPovR_ice", "LovR_liq", "LovR_ice",
              "I_QV", "I_QC", "I_QR", "I_QI", "I_QS", "I_QG"):
        g["hist_" + k] = hg[k]
    g["hist_SAT_LLIMIT"], g["hist_SAT_ULIMIT"] = hg["SAT_LLIMIT"], hg["SAT_ULIMIT"]
    return g

"""The reference-facing step API (backend.CudaDyn, the object the reference's
driver would construct in place of Dyn) driven through a stand-in of the
reference's model services built from the golden fixtures (fake_msc.py)."""
import numpy as np
import pytest

from fake_msc import fake_msc


def test_geo_from_msc_reproduces_the_fixture_setup(pkg, golden):
    """backend.geo_from_msc reads the services under the reference's attribute
    names and yields the setup the fixture generator wrote"""
    backend = __import__(pkg.__name__ + ".backend", fromlist=["geo_from_msc"])
    geo, st = golden
    msc = fake_msc(geo, st["state0"], st["state0_pl"])
    got = backend.geo_from_msc(msc)
    # the fixture also carries the level heights the oracle reads; the device path does not
    assert set(geo) - set(got) == {"GRD_gz", "GRD_gzh"} and set(got) <= set(geo)
    for k in got:
        assert np.array_equal(np.asarray(got[k]), np.asarray(geo[k])), k


def test_unsupported_configurations_raise(pkg, golden):
    backend = __import__(pkg.__name__ + ".backend", fromlist=["CudaDyn"])
    geo, st = golden
    for attr, val in (("AF_TYPE", "DCMIP"), ("THUBURN_LIM", False), ("DYN_DIV_NUM", 2)):
        msc = fake_msc(geo, st["state0"], st["state0_pl"])
        setattr(msc.rcnf, attr, val)
        with pytest.raises(NotImplementedError):
            backend.CudaDyn._check_config(msc)
    msc = fake_msc(geo, st["state0"], st["state0_pl"])
    msc.tim.TIME_integ_type = "RK4"
    with pytest.raises(NotImplementedError):
        backend.CudaDyn._check_config(msc)


_DCMIP_KEYS = ("GRD_Z", "GRD_ZH", "GRD_zsfc", "GMTR_p_IJ", "GRD_LAT", "GRD_LON", "NCHEM_STR", "NCHEM_END",
               "dcmip_flags")


def _dcmip_msc(geo, st, chem=True):
    g = {k: v for k, v in geo.items() if k not in _DCMIP_KEYS}
    extra = {k: geo[k] for k in _DCMIP_KEYS if k in geo}
    return fake_msc(g, st["state0"], st["state0_pl"], af_type="DCMIP", dcmip=extra)


@pytest.mark.parametrize("case", ["golden_dcmip11", "golden_smlsc", "golden_dcmip21", "golden_dcmip12bryan",
                                  "golden_smdry"])
def test_dcmip_simple_physics_setup_from_services(pkg, case, request):
    """the simple physics passes the configuration check (with or without
    Kessler, with moist Held-Suarez, with the Bryan boundary layer) and
    geo_from_msc hands the device its switches, half-level heights, surface
    height, latitude and unit vectors; RAIN_TYPE other than WARM is refused"""
    backend = __import__(pkg.__name__ + ".backend", fromlist=["geo_from_msc"])
    geo, st, _ = request.getfixturevalue(case)
    msc = _dcmip_msc(geo, st)
    backend.CudaDyn._check_config(msc)
    got = backend.geo_from_msc(msc)
    assert list(got["AF_dcmip_schemes"]) == [int(x) for x in geo["dcmip_flags"]]
    for k, w in (("AF_dcmip_zh", "GRD_ZH"), ("AF_dcmip_zsfc", "GRD_zsfc"), ("AF_dcmip_ij", "GMTR_p_IJ"),
                 ("AF_dcmip_lat", "GRD_LAT")):
        assert np.array_equal(got[k], geo[w]), k
    msc = _dcmip_msc(geo, st)
    msc.rcnf.RAIN_TYPE = "COLD"
    with pytest.raises(NotImplementedError):
        backend.CudaDyn._check_config(msc)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["golden_dcmip11", "golden_dcmip21", "golden_dcmip12bryan",
                                  "golden_smdry"])
def test_cudadyn_dcmip_simple_physics(pkg, case, request):
    """the reference-facing step API with the DCMIP2016 case 1-1 (Kessler,
    simple physics, chemistry) and case 2-1 (moist Held-Suarez) scheme sets:
    1e-12 relative L2 over the state and the precipitation"""
    geo, st, pr = request.getfixturevalue(case)
    msc = _dcmip_msc(geo, st)
    dyn = pkg.CudaDyn(msc=msc)
    try:
        for n in (1, 2):
            dyn.dynamics_step(msc)
            precip = dyn.forcing_step(msc)
            dyn.sync_prgvar_to_host(msc.prgv, msc)
            ref = st[f"state{n}"]
            err = np.sqrt(np.sum((msc.prgv.PRG_var - ref) ** 2)) / np.sqrt(np.sum(ref ** 2))
            assert err <= 1e-12, (n, err)
            want = pr[f"precip{n}"]
            assert np.sqrt(np.sum((np.asarray(precip) - want) ** 2)) <= 1e-12 * np.sqrt(np.sum(want ** 2)), n
    finally:
        dyn.core.close()


def test_dcmip_setup_from_services(pkg, golden_kessler_chem):
    """Kessler with the terminator chemistry passes the configuration check
    and yields the chemistry's set-up (tracer indices, column lat / lon); a
    third chemistry tracer does not"""
    backend = __import__(pkg.__name__ + ".backend", fromlist=["geo_from_msc"])
    geo, st, _ = golden_kessler_chem
    msc = _dcmip_msc(geo, st, True)
    backend.CudaDyn._check_config(msc)
    got = backend.geo_from_msc(msc)
    assert got["AF_dcmip_kessler"] == 1 and list(got["AF_dcmip_chem"]) == [3, 4]
    assert np.array_equal(got["AF_dcmip_lat"], geo["GRD_LAT"]) and np.array_equal(got["AF_dcmip_lon"], geo["GRD_LON"])
    assert np.array_equal(got["GRD_Z"], geo["GRD_Z"])

    msc = _dcmip_msc(geo, st, True)
    msc.rcnf.NCHEM_END = 5
    with pytest.raises(NotImplementedError):
        backend.CudaDyn._check_config(msc)


def _numf_msc(geo, st, case):
    """services for the NONLINEAR1 or Rayleigh fixture: the reference's numfilter
    attributes (make_golden.NUMF) and the arrays it set up"""
    from make_golden import NUMF
    skip = ("hdiff_nl_kh_max", "hdiff_nl_minlim", "hdiff_nl_area", "rayleigh_coef", "rayleigh_coef_h",
            "rayleigh_only_w")
    g = {k: v for k, v in geo.items() if k not in skip}
    if case == "nlhdiff":
        o = NUMF["gl03_z10_nlhdiff"]
        opts = dict(hdiff_nonlinear=True, Kh_coef=np.full(np.asarray(geo["VMTR_GSGAM2"]).shape, -999.0),
                    Kh_coef_maxlim=o["Kh_coef_maxlim"], Kh_coef_minlim=o["Kh_coef_minlim"],
                    ZD_hdiff_nl=o["ZD_hdiff_nl"], AREA_ave=float(geo["hdiff_nl_area"]))
    else:
        opts = dict(NUMFILTER_DOrayleigh=True, rayleigh_coef=geo["rayleigh_coef"],
                    rayleigh_coef_h=geo["rayleigh_coef_h"], rayleigh_damp_only_w=False)
    return fake_msc(g, st["state0"], st["state0_pl"], numf_opts=opts)


@pytest.mark.parametrize("case", ["nlhdiff", "rayleigh"])
def test_numfilter_setup_from_services(pkg, case, request):
    """backend.geo_from_msc hands the NONLINEAR1 bounds (the per-level upper
    bound restated from the reference's height_factor, equal to the one the
    reference computed) and the Rayleigh coefficients to the device set-up,
    and the configuration check accepts them"""
    backend = __import__(pkg.__name__ + ".backend", fromlist=["geo_from_msc"])
    geo, st = request.getfixturevalue("golden_" + case)
    msc = _numf_msc(geo, st, case)
    backend.CudaDyn._check_config(msc)
    got = backend.geo_from_msc(msc)
    keys = ("hdiff_nl_kh_max", "hdiff_nl_minlim", "hdiff_nl_area") if case == "nlhdiff" else \
        ("rayleigh_coef", "rayleigh_coef_h", "rayleigh_only_w")
    for k in keys:
        assert np.array_equal(np.asarray(got[k]), np.asarray(geo[k])), k
    msc.numf.NUMFILTER_DOdivdamp_2d = True
    with pytest.raises(NotImplementedError):
        backend.CudaDyn._check_config(msc)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["nlhdiff", "rayleigh"])
def test_cudadyn_numfilter_options(pkg, case, request):
    """the reference-facing step API with NONLINEAR1 or the Rayleigh sponge:
    two steps bit for bit with the reference's"""
    geo, st = request.getfixturevalue("golden_" + case)
    msc = _numf_msc(geo, st, case)
    dyn = pkg.CudaDyn(msc=msc)
    try:
        for n in (1, 2):
            dyn.dynamics_step(msc)
            dyn.sync_prgvar_to_host(msc.prgv, msc)
            assert np.array_equal(msc.prgv.PRG_var, st[f"state{n}"]), n
            assert np.array_equal(msc.prgv.PRG_var_pl, st[f"state{n}_pl"]), n
    finally:
        dyn.core.close()


@pytest.mark.gpu
def test_cudadyn_dcmip_kessler_with_chemistry(pkg, golden_kessler_chem):
    """the reference-facing step API with DCMIP forcing (Kessler + terminator
    chemistry): forcing_step returns the precipitation; states within the
    1e-12 relative L2 of the device forcing test"""
    geo, st, pr = golden_kessler_chem
    msc = _dcmip_msc(geo, st, True)
    dyn = pkg.CudaDyn(msc=msc)
    try:
        for n in (1, 2):
            dyn.dynamics_step(msc)
            precip = dyn.forcing_step(msc)
            dyn.sync_prgvar_to_host(msc.prgv, msc)
            ref = st[f"state{n}"]
            err = np.sqrt(np.sum((msc.prgv.PRG_var - ref) ** 2)) / np.sqrt(np.sum(ref ** 2))
            assert err <= 1e-12, (n, err)
            want = pr[f"precip{n}"]
            assert np.sqrt(np.sum((np.asarray(precip) - want) ** 2)) <= 1e-12 * np.sqrt(np.sum(want ** 2)), n
    finally:
        dyn.core.close()


@pytest.mark.gpu
def test_cudadyn_steps_through_the_reference_api(pkg, golden):
    geo, st = golden
    msc = fake_msc(geo, st["state0"], st["state0_pl"])
    dyn = pkg.CudaDyn(msc=msc)
    try:
        dyn.dynamics_step(msc)
        assert dyn.forcing_step(msc) is None            # AF_TYPE NONE: no-op
        with pytest.raises(AssertionError):
            dyn.assert_host_prgvar_synced("test")       # host PRG_var is stale now
        dyn.sync_prgvar_to_host(msc.prgv, msc)
        dyn.assert_host_prgvar_synced("test")
        assert np.array_equal(msc.prgv.PRG_var, st["state1"])
        assert np.array_equal(msc.prgv.PRG_var_pl, st["state1_pl"])
        dyn.run_timeloop_chunk(msc, 1)
        dyn.sync_prgvar_to_host(msc.prgv, msc)
        assert np.array_equal(msc.prgv.PRG_var, st["state2"])
    finally:
        dyn.core.close()


@pytest.mark.gpu
def test_cudadyn_held_suarez_forcing(pkg, golden_hs):
    geo, lat, st = golden_hs
    msc = fake_msc(geo, st["state0"], st["state0_pl"], af_type="HELD-SUAREZ", lat=lat)
    dyn = pkg.CudaDyn(msc=msc)
    try:
        for n in (1, 2):
            dyn.dynamics_step(msc)
            dyn.forcing_step(msc)
            dyn.sync_prgvar_to_host(msc.prgv, msc)
            ref = st[f"state{n}"]
            err = np.sqrt(np.sum((msc.prgv.PRG_var - ref) ** 2)) / np.sqrt(np.sum(ref ** 2))
            assert err <= 1e-12, (n, err)
    finally:
        dyn.core.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["golden_trcadv", "golden_trcadv12"])
def test_cudadyn_offline_tracer_advection(pkg, case, request):
    """three offline-advection steps through the step API, with the DCMIP 1-1
    and the 1-2 winds"""
    from conftest import TRC_COORDS
    geo, st = request.getfixturevalue(case)
    geo = dict(geo)
    coords = {k: geo.pop(k) for k in TRC_COORDS}
    geo.pop("integ_type")
    dcase = str(geo.pop("trcadv_case", "1-1"))
    msc = fake_msc(geo, st["state0"], st["state0_pl"], integ_type="TRCADV", coords=coords, dctest_case=dcase)
    dyn = pkg.CudaDyn(msc=msc)
    try:
        dyn.run_timeloop_chunk(msc, 3)
        dyn.sync_prgvar_to_host(msc.prgv, msc)
        ref = st["state3"]
        for v in range(ref.shape[-1]):
            den = np.sqrt(np.sum(ref[..., v] ** 2))
            err = np.sqrt(np.sum((msc.prgv.PRG_var[..., v] - ref[..., v]) ** 2))
            assert err <= 1e-12 * max(den, 1.0), (v, err, den)
    finally:
        dyn.core.close()

"""The CPU oracle against the golden states written by the reference itself
(tests/golden/make_golden.py): bit-for-bit on two consecutive large steps."""
import numpy as np
import pytest

from oracle import nicam_step as O


def test_oracle_matches_reference_two_steps(golden):
    geo, st = golden
    G = O.Geo(geo)
    for s in (0, 1):
        out, out_pl = O.dynamics_step(G, st[f"state{s}"], st[f"state{s}_pl"])
        assert np.array_equal(out, st[f"state{s + 1}"]), f"step {s + 1} regional"
        assert np.array_equal(out_pl, st[f"state{s + 1}_pl"]), f"step {s + 1} pole"


def test_oracle_matches_reference_warm_rain(golden_warm):
    """three water tracers (RAIN_TYPE WARM): cv and qd over the water range"""
    geo, st = golden_warm
    G = O.Geo(geo)
    assert G.nqw == 3
    for s in (0, 1):
        out, out_pl = O.dynamics_step(G, st[f"state{s}"], st[f"state{s}_pl"])
        assert np.array_equal(out, st[f"state{s + 1}"]), f"step {s + 1} regional"
        assert np.array_equal(out_pl, st[f"state{s + 1}_pl"]), f"step {s + 1} pole"


@pytest.mark.parametrize("case", ["golden_nlhdiff", "golden_rayleigh"])
def test_oracle_numfilter_options_match_reference(case, request):
    """the NONLINEAR1 hyperdiffusion and the Rayleigh sponge: two steps of
    the oracle equal the reference's bit for bit"""
    geo, st = request.getfixturevalue(case)
    G = O.Geo(geo)
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2):
        s, sp = O.dynamics_step(G, s, sp)
        assert np.array_equal(s, st[f"state{n}"]) and np.array_equal(sp, st[f"state{n}_pl"]), n


def test_nonlinear_kh_takes_every_branch(golden_nlhdiff, monkeypatch):
    """in the NONLINEAR1 fixture's first step Kh sits at its lower bound, at
    the per-level upper bound and strictly between them, each for a sizeable
    share of the cells, so the clip is tested both ways"""
    geo, st = golden_nlhdiff
    seen = []
    orig = O.hdiff_nonlinear_coef

    def spy(g, a, b):
        kh, kh_pl = orig(g, a, b)
        lo, hi = float(g.hdiff_nl_minlim), np.asarray(g.hdiff_nl_kh_max)[None, None, :, None]
        seen.append(((kh == lo).mean(), (kh == hi).mean(), ((kh > lo) & (kh < hi)).mean()))
        return kh, kh_pl
    monkeypatch.setattr(O, "hdiff_nonlinear_coef", spy)
    O.dynamics_step(O.Geo(geo), st["state0"], st["state0_pl"])
    assert len(seen) == 3 and all(min(f) > 0.05 for f in seen), seen


def test_rayleigh_fixture_is_active(golden, golden_rayleigh):
    """the sponge changed the momentum against the undamped run from the same
    state, and its coefficient is zero below 15 km"""
    _, st0 = golden
    geo, st = golden_rayleigh
    assert np.array_equal(st["state0"], st0["state0"])
    assert np.abs(st["state1"][..., 1] - st0["state1"][..., 1]).max() > 1e-3
    rc = np.asarray(geo["rayleigh_coef"])
    assert np.all(rc[np.asarray(geo["GRD_gz"]) < 15000.0] == 0.0) and rc.max() > 0.0


def test_oracle_kessler_forcing_matches_reference(golden_kessler):
    """dynamics step + DCMIP forcing with Kessler microphysics, against the
    reference run (tests/golden/make_kessler.py): states and precipitation"""
    geo, st, pr = golden_kessler
    G = O.Geo(geo)
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2):
        s, sp = O.dynamics_step(G, s, sp)
        s, sp, precip = O.forcing_step_kessler(G, s, sp, geo["GRD_Z"])
        assert np.array_equal(s, st[f"state{n}"]) and np.array_equal(sp, st[f"state{n}_pl"]), n
        assert np.array_equal(precip, pr[f"precip{n}"]), n


def test_oracle_terminator_chemistry_matches_reference(golden_kessler_chem):
    """dynamics step + DCMIP forcing with Kessler microphysics and the
    terminator toy chemistry on Cl / Cl2, against the reference run
    (tests/golden/make_kessler.py --chem): states and precipitation"""
    geo, st, pr = golden_kessler_chem
    G = O.Geo(geo)
    chem = (geo["GRD_LAT"], geo["GRD_LON"], int(geo["NCHEM_STR"]), int(geo["NCHEM_END"]))
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2):
        s, sp = O.dynamics_step(G, s, sp)
        s, sp, precip = O.forcing_step_kessler(G, s, sp, geo["GRD_Z"], chem=chem)
        assert np.array_equal(s, st[f"state{n}"]) and np.array_equal(sp, st[f"state{n}_pl"]), n
        assert np.array_equal(precip, pr[f"precip{n}"]), n


@pytest.mark.parametrize("case", ["golden_dcmip11", "golden_smlsc", "golden_dcmip21", "golden_dcmip12bryan",
                                  "golden_smdry"])
def test_oracle_simple_physics_matches_reference(case, request):
    """dynamics step + DCMIP forcing with the simple physics (with Kessler and
    the chemistry as in DCMIP2016 case 1-1; alone with the large-scale
    condensation and constant SST), against the reference run: states and
    precipitation bit for bit"""
    from conftest import dcmip_oracle_args
    geo, st, pr = request.getfixturevalue(case)
    G = O.Geo(geo)
    kw = dcmip_oracle_args(geo)
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2):
        s, sp = O.dynamics_step(G, s, sp)
        s, sp, precip = O.forcing_step_kessler(G, s, sp, geo["GRD_Z"], **kw)
        assert np.array_equal(s, st[f"state{n}"]) and np.array_equal(sp, st[f"state{n}_pl"]), n
        assert np.array_equal(precip, pr[f"precip{n}"]), n


def test_oracle_chemistry_history_columns_match_reference(golden_kessler_chem):
    """sl_cl, sl_cl2, sl_cly of the chemistry run's last state: the oracle's
    history equals the reference's Dyn.history_vars_step bit for bit"""
    import os
    from conftest import GOLDEN
    from oracle import nicam_history as OH
    geo, st, _ = golden_kessler_chem
    d = np.load(os.path.join(GOLDEN, "gl03_z10_kessler_chem.npz"))
    hg = {k[5:]: d[k] for k in d.files if k.startswith("hgeo.")}
    names = ("sl_cl", "sl_cl2", "sl_cly")
    got = OH.History()(O.Geo(geo), hg, st["state2"], items=names)
    for n in names:
        assert np.array_equal(got[n], d["hist." + n]), n
    assert 1e-6 < d["hist.sl_cly"].min() and d["hist.sl_cly"].max() < 1e-5   # mixing ratios of order 4e-6


def test_moist_held_suarez_fixture_is_active(golden_kessler, golden_dcmip21):
    """the Held-Suarez relaxation replaced the momentum tendency: the moist
    Held-Suarez run moved the momentum away from the Kessler-only run"""
    _, a, _ = golden_kessler
    _, b, _ = golden_dcmip21
    assert np.array_equal(a["state0"], b["state0"])
    assert np.abs(a["state1"][..., 1] - b["state1"][..., 1]).max() > 0.1


def test_simple_physics_fixtures_are_active(golden_kessler_chem, golden_dcmip11, golden_smlsc):
    """the simple physics moved momentum, energy and vapour against the same
    run without it, and its condensation rained in a fifth of the columns"""
    _, a, _ = golden_kessler_chem
    _, b, _ = golden_dcmip11
    assert np.array_equal(a["state0"], b["state0"])
    for v, lim in ((1, 0.1), (5, 10.0), (6, 1e-5)):
        assert np.abs(a["state1"][..., v] - b["state1"][..., v]).max() > lim, v
    _, _, pr = golden_smlsc
    assert (pr["precip1"] > 0).mean() > 0.2


def test_sst_of_the_device_setup_equals_the_oracle(pkg, golden_dcmip11):
    """the sea-surface temperature runtime.setup_table hands the device is the
    oracle's (pinned to the reference by the fixture), in both forms"""
    geo, _, _ = golden_dcmip11
    lat = geo["GRD_LAT"]
    for latdep in (True, False):
        assert np.array_equal(pkg.runtime.dcmip_sst(lat, latdep), O.dcmip_sst(lat, latdep))
    for mitc in (1, 2, 3):
        assert np.array_equal(pkg.runtime.dcmip_sst(lat, False, True, mitc), O.dcmip_sst(lat, False, True, mitc))


def test_terminator_fixture_is_active(golden_kessler_chem):
    """the chemistry changed Cl and Cl2 against the same step without it,
    and conserved the total chlorine Cl + 2 Cl2 of every cell"""
    geo, st, _ = golden_kessler_chem
    G = O.Geo(geo)
    s, sp = O.dynamics_step(G, st["state0"], st["state0_pl"])
    s, _, _ = O.forcing_step_kessler(G, s, sp, geo["GRD_Z"])
    d_cl = st["state1"][..., 9] - s[..., 9]
    assert np.abs(d_cl).max() > 1e-3 * np.abs(s[..., 9]).max()
    cly, cly0 = st["state1"][..., 9] + 2.0 * st["state1"][..., 10], s[..., 9] + 2.0 * s[..., 10]
    assert np.abs(cly - cly0).max() <= 1e-12 * np.abs(cly0).max()


def test_kessler_fixture_is_active(golden_warm, golden_kessler):
    """the microphysics changed the water and energy against the unforced
    WARM run of the same case, and it rained somewhere"""
    _, st0 = golden_warm
    _, st, pr = golden_kessler
    assert np.array_equal(st["state0"], st0["state0"])
    assert np.abs(st["state1"][..., 5] - st0["state1"][..., 5]).max() > 1.0
    assert np.abs(st["state1"][..., 8] - st0["state1"][..., 8]).max() > 1e-4
    assert pr["precip1"].max() > 0.0


def test_golden_tracer_is_nontrivial(golden):
    _, st = golden
    q = st["state0"][..., 6]
    assert q.max() > 1e-3 and (q > 0).mean() > 0.5


def test_oracle_held_suarez_matches_reference_two_steps(golden_hs):
    """dynamics step + Held-Suarez forcing step, against the reference run
    with AF_TYPE 'HELD-SUAREZ' (tests/golden/make_hs.py)"""
    geo, lat, st = golden_hs
    G = O.Geo(geo)
    for s in (0, 1):
        out, out_pl = O.dynamics_step(G, st[f"state{s}"], st[f"state{s}_pl"])
        out, out_pl = O.forcing_step_hs(G, out, out_pl, lat)
        assert np.array_equal(out, st[f"state{s + 1}"]), f"step {s + 1} regional"
        assert np.array_equal(out_pl, st[f"state{s + 1}_pl"]), f"step {s + 1} pole"


def test_held_suarez_fixture_is_forced(golden, golden_hs):
    """the forced states differ from the unforced reference run of the same case"""
    _, _, st = golden_hs
    _, st0 = golden
    assert np.array_equal(st["state0"], st0["state0"])
    d = np.abs(st["state1"][..., 1:4] - st0["state1"][..., 1:4]).max()
    assert d > 0.0


def test_oracle_trcadv12_matches_reference_three_steps(golden_trcadv12):
    """offline tracer advection with the DCMIP 1-2 winds (Hadley-like
    circulation, test12_velocity) against the reference's own run"""
    from conftest import TRC_COORDS
    geo, st = golden_trcadv12
    geo = dict(geo)
    co = [geo.pop(k) for k in TRC_COORDS]
    assert str(geo.pop("integ_type")) == "TRCADV" and str(geo.pop("trcadv_case")) == "1-2"
    G = O.Geo(geo)
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2, 3):
        s, sp = O.trcadv_step(G, s, sp, n * G.dtl, *co, case="1-2")
        assert np.array_equal(s, st[f"state{n}"]), f"step {n} regional"
        assert np.array_equal(sp, st[f"state{n}_pl"]), f"step {n} pole"
    assert np.abs(st["state3"][..., 7] - st["state0"][..., 7]).max() > 1e-3   # the tracer layer moved
    assert np.abs(st["state2"][..., 4] - st["state1"][..., 4]).max() > 0.0    # w is time-dependent


def test_oracle_trcadv_matches_reference_three_steps(golden_trcadv):
    """offline tracer advection (integ_type TRCADV, DCMIP 1-1 winds) against
    the reference's own run (tests/golden/make_trcadv.py)"""
    from conftest import TRC_COORDS
    geo, st = golden_trcadv
    geo = dict(geo)
    co = [geo.pop(k) for k in TRC_COORDS]
    assert str(geo.pop("integ_type")) == "TRCADV"
    G = O.Geo(geo)
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2, 3):
        s, sp = O.trcadv_step(G, s, sp, n * G.dtl, *co)
        assert np.array_equal(s, st[f"state{n}"]), f"step {n} regional"
        assert np.array_equal(sp, st[f"state{n}_pl"]), f"step {n} pole"
    # four passive tracers were advected and the winds were reset every step
    assert np.abs(st["state3"][..., 7:11] - st["state0"][..., 7:11]).max() > 0.0
    assert np.abs(st["state2"][..., 1:5] - st["state1"][..., 1:5]).max() > 0.0


def test_oracle_history_matches_reference(golden, golden_hist):
    """the derived history diagnostics (oracle/nicam_history.py) against the
    reference's own Dyn.history_vars_step after steps 1 and 2
    (tests/golden/make_hist.py): all 42 fields bit-for-bit, the tendencies
    over one step included"""
    from oracle import nicam_history as OH
    geo, st = golden
    hg, ref = golden_hist
    G = O.Geo(geo)
    H = OH.History()
    s, sp = st["state0"], st["state0_pl"]
    for n in (1, 2):
        keep = {}
        s, sp = O.dynamics_step(G, s, sp, keep=keep)
        out = H(G, hg, s, dt=float(ref["dtl"]), nstep=int(ref[f"nstep{n}"]), w_prev=keep["w"])
    assert sorted(out) == sorted(OH.ML + OH.SL)
    for k in OH.ML + OH.SL:
        assert np.array_equal(out[k], ref[k]), k
    for k in ("ml_du", "ml_dtem", "ml_dq", "sl_pw", "ml_th_prime", "sl_u850", "ml_rh"):
        assert np.abs(ref[k]).max() > 0.0, k

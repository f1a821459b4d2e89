"""Derived history diagnostics on the device (nc_history_vars) against the
reference's own Dyn.history_vars_step (tests/golden/make_hist.py) and the
oracle (oracle/nicam_history.py).

Fields formed with the step's own arithmetic (the diagnostic state, winds,
cell-centre w, omega, moist static energy, the interval tendencies, surface
pressure, the tracer column sums of an absent species) must match bit for
bit.  The potential temperatures, the saturation ratios and the pressure-level
slices go through pow, exp and log, which CUDA and numpy may round differently
in the last bit, and the per-layer mean of th_prime and the column water sum
add in another order: those are compared to a relative max-norm of 1e-12 (the
one-step parity tolerance of the step itself)."""
import os

import numpy as np
import pytest

from oracle import nicam_history as OH
from oracle import nicam_step as O

pytestmark = pytest.mark.gpu

EXACT = {"ml_u", "ml_v", "ml_w", "ml_omg", "ml_pres", "ml_tem", "ml_rho", "ml_hgt", "ml_mse", "ml_du", "ml_dv",
         "ml_dw", "ml_dtem", "ml_dq", "ml_ucos", "ml_vcos", "sl_ps", "sl_lwp", "sl_iwp"}
TOL = 1e-12


def _rel(a, b):
    den = np.abs(b).max()
    return float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a).max())


def _check(got, want, names):
    for k in names:
        assert got[k].shape == want[k].shape, k
        if k in EXACT:
            assert np.array_equal(got[k], want[k]), (k, _rel(got[k], want[k]))
        else:
            assert _rel(got[k], want[k]) <= TOL, (k, _rel(got[k], want[k]))


def _core(pkg, golden, golden_hist):
    from conftest import hist_geo
    geo, _ = golden
    hg, _ = golden_hist
    return pkg.NicamCuda(hist_geo(geo, hg))


def test_history_two_steps_vs_reference(pkg, golden, golden_hist):
    """seeded after step 1 (tendencies zero), then all 42 fields after step 2
    (the chemistry's columns have their own test)"""
    _, st = golden
    _, ref = golden_hist
    names = tuple(n for n in pkg.runtime.HIST_ITEMS if n not in pkg.runtime.HIST_CHEM)
    assert sorted(names) == sorted(OH.ML + OH.SL)
    c = _core(pkg, golden, golden_hist)
    c.upload(st["state0"], st["state0_pl"])
    c.step(1)
    h1 = c.history_vars(names, nstep=int(ref["nstep1"]), dt=float(ref["dtl"]))
    for k in OH.TEND:
        assert not np.any(h1[k]), k
    c.step(1)
    h2 = c.history_vars(names, nstep=int(ref["nstep2"]), dt=float(ref["dtl"]))
    _check(h2, ref, names)


def test_history_before_any_step_vs_oracle(pkg, golden, golden_hist):
    """a fresh handle: the boundary rows of w are zero, as the reference's
    UNDEF-filled buffer reads through its filter; a subset of names"""
    geo, st = golden
    hg, ref = golden_hist
    names = ("ml_w", "ml_omg", "ml_th", "sl_w500", "sl_pw", "ml_th_prime")
    c = _core(pkg, golden, golden_hist)
    c.upload(st["state1"], st["state1_pl"])
    got = c.history_vars(names, nstep=1, dt=float(ref["dtl"]))
    want = OH.History()(O.Geo(geo), hg, st["state1"], items=names, dt=float(ref["dtl"]), nstep=1)
    assert sorted(got) == sorted(names)
    _check(got, want, names)


def test_history_step_api_through_backend(pkg, golden, golden_hist):
    """CudaDyn.history_vars_step with the reference's I/O groups: only the
    groups being written are formed; the tendencies follow the step count"""
    from fake_msc import fake_msc
    geo, st = golden
    hg, ref = golden_hist
    io_names = ["ml_u", "ml_dtem", "ml_th", "sl_ps", "sl_t850"]
    msc = fake_msc(geo, st["state0"], st["state0_pl"], hist=hg, io_names=io_names)
    assert np.array_equal(np.stack([msc.gmtr.GMTR_p[:, :, 0, :, i] for i in range(2, 8)], axis=-1),
                          hg["GMTR_p_IJ"])
    dyn = pkg.backend.CudaDyn(msc)
    dt = float(ref["dtl"])
    assert dt == msc.tim.TIME_dtl
    dyn.dynamics_step(msc)
    msc.tim.TIME_cstep = 1
    h1 = dyn.history_vars_step(msc)
    assert sorted(h1) == sorted(io_names) and not np.any(h1["ml_dtem"])
    dyn.dynamics_step(msc)
    msc.tim.TIME_cstep = 2
    h3 = dyn.history_vars_step(msc, write_2d=False)
    assert sorted(h3) == ["ml_dtem", "ml_th", "ml_u"]
    _check(h3, ref, h3)
    msc.io._diag_names_2d = ["sl_cl"]
    with pytest.raises(NotImplementedError):   # no terminator chemistry on this handle
        dyn.history_vars_step(msc)


def test_history_needs_its_setup(pkg, golden):
    """a handle created without the HIST_* entries refuses, with a status"""
    geo, st = golden
    c = pkg.NicamCuda(geo)
    c.upload(st["state0"], st["state0_pl"])
    with pytest.raises(pkg.NicamError):
        c.history_vars(("ml_u",), nstep=0, dt=1200.0)
    with pytest.raises(NotImplementedError):
        c.history_vars(("sl_foo",), nstep=0, dt=1200.0)


def test_chemistry_columns_vs_reference(pkg, golden_kessler_chem):
    """sl_cl, sl_cl2 and sl_cly (the terminator chemistry's column means,
    mod_history_vars.py:149-156) of the DCMIP chemistry run's last state
    against the reference's: bit for bit (sums in the reference's order, no
    transcendental functions); a handle without HIST_chem refuses them"""
    import numpy as np
    from conftest import GOLDEN, hist_geo
    geo, st, _ = golden_kessler_chem
    d = np.load(os.path.join(GOLDEN, "gl03_z10_kessler_chem.npz"))
    hg = {k[5:]: d[k] for k in d.files if k.startswith("hgeo.")}
    g = hist_geo({k: v for k, v in geo.items() if k not in ("GRD_LAT", "GRD_LON")}, hg)
    names = ("sl_cl", "sl_cl2", "sl_cly")
    c = pkg.NicamCuda(g, graph=False)
    try:
        c.upload(st["state2"], st["state2_pl"])
        with pytest.raises(pkg.NicamError):
            c.history_vars(names, nstep=2, dt=float(geo["dtl"]))
    finally:
        c.close()
    g["hist_NCHEM"] = hg["NCHEM"]
    c = pkg.NicamCuda(g, graph=False)
    try:
        c.upload(st["state2"], st["state2_pl"])
        out = c.history_vars(names, nstep=2, dt=float(geo["dtl"]))
    finally:
        c.close()
    for n in names:
        print(n, "max relative difference", _rel(out[n], d["hist." + n]))
        assert np.array_equal(out[n], d["hist." + n]), n

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
def test_cudadyn_offline_tracer_advection(pkg, golden_trcadv):
    from conftest import TRC_COORDS
    geo, st = golden_trcadv
    geo = dict(geo)
    coords = {k: geo.pop(k) for k in TRC_COORDS}
    geo.pop("integ_type")
    msc = fake_msc(geo, st["state0"], st["state0_pl"], integ_type="TRCADV", coords=coords)
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

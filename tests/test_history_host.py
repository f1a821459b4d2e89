"""Host logic of CudaDyn.history_vars_step (mirror of the reference's
Dyn.history_vars_step, pynicamdc/nhm/dynamics/mod_dynamics.py:737-772): which
names are formed for the I/O groups being written, and what reaches the
device call; a recording stand-in replaces the device core."""
from types import SimpleNamespace as NS

import pytest


class _Core:
    def __init__(self):
        self.calls = []

    def history_vars(self, names, nstep, dt):
        self.calls.append((tuple(names), nstep, dt))
        return {n: None for n in names}


def _dyn(pkg, chem=False):
    d = object.__new__(pkg.backend.CudaDyn)
    d.core, d._device_valid, d._host_stale, d._forced = _Core(), True, True, False
    d._hist_chem = chem
    return d


def _msc(io=None):
    m = NS(tim=NS(TIME_cstep=7, TIME_dtl=150.0))
    if io is not None:
        m.io = io
    return m


def test_names_follow_the_io_groups(pkg):
    d = _dyn(pkg)
    io = NS(_diag_names=["ml_th", "ml_u"], _diag_names_2d=["sl_ps"])
    assert sorted(d.history_vars_step(_msc(io))) == ["ml_th", "ml_u", "sl_ps"]
    assert sorted(d.history_vars_step(_msc(io), write_2d=False)) == ["ml_th", "ml_u"]
    assert sorted(d.history_vars_step(_msc(io), write_3d=False)) == ["sl_ps"]
    names, nstep, dt = d.core.calls[0]
    assert names == ("ml_u", "ml_th", "sl_ps") and nstep == 7 and dt == 150.0   # the device's id order


def test_without_io_every_item(pkg):
    """every item, the chemistry's columns only with the chemistry configured
    (the reference forms them for AF_TYPE 'DCMIP' with NCHEM_STR >= 0)"""
    out = _dyn(pkg).history_vars_step(_msc())
    assert tuple(out) == tuple(n for n in pkg.runtime.HIST_ITEMS if n not in pkg.runtime.HIST_CHEM)
    out = _dyn(pkg, chem=True).history_vars_step(_msc())
    assert tuple(out) == pkg.runtime.HIST_ITEMS


def test_empty_groups_form_nothing(pkg):
    d = _dyn(pkg)
    assert d.history_vars_step(_msc(NS(_diag_names=[], _diag_names_2d=[]))) == {}


def test_unknown_names_raise(pkg):
    """names the device does not form, and the chemistry's columns without
    the chemistry, raise before any device call"""
    d = _dyn(pkg)
    for names in (["sl_foo"], ["sl_cly"]):
        with pytest.raises(NotImplementedError):
            d.history_vars_step(_msc(NS(_diag_names=["ml_u"], _diag_names_2d=names)))
    assert d.core.calls == []
    d = _dyn(pkg, chem=True)
    assert sorted(d.history_vars_step(_msc(NS(_diag_names=[], _diag_names_2d=["sl_cly"])))) == ["sl_cly"]


def test_setup_table_history_entries(pkg, golden, golden_hist):
    """the HIST_* entries nc_create reads: shapes, cos(lat) with numpy's cos,
    constants and tracer indices in the header's order, PRE00 alongside"""
    import numpy as np
    from conftest import hist_geo
    geo, _ = golden
    hg, _ = golden_hist
    t = pkg.runtime.setup_table(hist_geo(geo, hg))
    G, K, L = (int(np.asarray(geo[k])) for k in ("gall_1d", "kall", "lall"))
    assert t["HIST_hgt"].shape == (G, G, K, L)
    for k in ("HIST_coslat", "HIST_zsfc", "HIST_area"):
        assert t[k].shape == (G, G, 1, L), k
    assert t["HIST_IJ"].shape == (G, G, 1, L, 6)
    assert np.array_equal(t["HIST_coslat"][:, :, 0, :], np.cos(hg["GRD_LAT"]))
    assert t["HIST_consts"].tolist() == [float(hg[k]) for k in ("LHV", "UNDEF", "PSAT0", "RTEM00", "CPovR_liq",
                                                                 "CPovR_ice", "LovR_liq", "LovR_ice",
                                                                 "SAT_LLIMIT", "SAT_ULIMIT")]
    assert t["HIST_tracers"].dtype == np.int64 and t["HIST_tracers"].tolist()[0] == int(hg["I_QV"])
    assert float(t["PRE00"]) == float(np.asarray(geo["PRE00"]))
    assert "HIST_hgt" not in pkg.runtime.setup_table(geo)

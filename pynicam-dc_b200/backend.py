"""The ``cuda`` backend object that stands in for the reference's ``Dyn``.

pyNICAM-DC's driver calls, per step, ``dyn.dynamics_step(msc)`` and
``dyn.forcing_step(msc)`` (pynicamdc/api.py:724-730), or
``dyn.run_timeloop_chunk(msc, K)`` for fused chunks (api.py:697-699), and
drains the device state with ``dyn.sync_prgvar_to_host(prgv, msc)`` before
output and budgets (api.py:800, nhm/share/mod_embudget.py:68).  ``CudaDyn``
offers the same methods with the same meaning:

* ``dynamics_step(msc)`` -- one large step of ``Dyn.dynamics_step``
  (nhm/dynamics/mod_dynamics.py:1725-2741) on the device; the host
  ``prgv.PRG_var`` becomes stale (the reference's "drain only at output"
  invariant, mod_dynamics.py:2693-2697);
* ``run_timeloop_chunk(msc, K)`` -- K such steps (mod_dynamics.py:784);
* ``sync_prgvar_to_host(prgv, msc)`` -- copy the device state into
  ``prgv.PRG_var`` / ``prgv.PRG_var_pl`` in place (mod_dynamics.py:429-440);
* ``assert_host_prgvar_synced(who)`` -- ``AssertionError`` on a stale host read
  (mod_dynamics.py:460-468);
* ``forcing_step(msc)`` -- a no-op for ``AF_TYPE = NONE`` like the reference
  (mod_dynamics.py:597); the Held-Suarez forcing (``AF_TYPE = HELD-SUAREZ``)
  on the device through ``nc_forcing_step``; DCMIP forcing is not part of
  this backend and raises at set-up.

Geometry, metrics and operator coefficients are read once from the
reference's setup services on ``msc`` (grd, gmtr, oprt, vmtr, bsst, comm, ...)
and uploaded; the device keeps them for the run.
"""
from __future__ import annotations

import numpy as np

from . import restart
from .runtime import HIST_CHEM, HIST_ITEMS, NicamCuda


def _dcmip_flags(msc) -> dict:
    """the DCMIP scheme flags the reference resolved (mod_af_dcmip.py
    AF_dcmip_init): from ``msc.afdcmip`` when the services carry it, else the
    reference module's instance"""
    obj = getattr(msc, "afdcmip", None)
    if obj is None:
        import sys
        mod = sys.modules.get("pynicamdc.nhm.forcing.mod_af_dcmip")
        obj = getattr(mod, "afdcmip", None) if mod is not None else None
    keys = ("USE_Kessler", "USE_SimpleMicrophys", "USE_ToyChemistry", "USE_HeldSuarez", "SM_Latdepend_SST",
            "SM_LargeScaleCond", "SM_PBL_Bryan")
    out = {k: bool(getattr(obj, k, False)) for k in keys}
    out["SM_MITC_SST_TYPE"] = int(getattr(obj, "SM_MITC_SST_TYPE", 1))
    return out


def geo_from_msc(msc) -> dict:
    """Collect the setup arrays of the reference's services into the flat
    dict that ``NicamCuda`` uploads (attribute names kept)."""
    m = msc
    a = m.adm
    g = dict(kall=a.ADM_kall, kmin=a.ADM_kmin, kmax=a.ADM_kmax, gall_1d=a.ADM_gall_1d, gmin=a.ADM_gmin,
             gmax=a.ADM_gmax, lall=a.ADM_lall, have_sgp=np.asarray(a.ADM_have_sgp),
             nq=m.prgv.PRG_var.shape[-1] - 6)
    g["pntmask"] = np.asarray(m.ppm.pntmask)
    c = m.cnst
    g.update(GRAV=c.CONST_GRAV, Rdry=c.CONST_Rdry, CVdry=c.CONST_CVdry, CPdry=c.CONST_CPdry, Rvap=c.CONST_Rvap,
             OHM=c.CONST_OHM, RADIUS=c.CONST_RADIUS, EPS=c.CONST_EPS, HUGE=c.CONST_HUGE, PRE00=c.CONST_PRE00)
    g.update(rscale=m.grd.GRD_rscale, alpha=float(m.rcnf.NON_HYDRO_ALPHA), dtl=m.tim.TIME_dtl,
             dts=m.tim.TIME_dts, hdiff_fact_rho=m.numf.hdiff_fact_rho)
    nf = m.numf
    Kh, dd = np.asarray(nf.Kh_coef), np.asarray(nf.divdamp_coef)
    nonlinear = bool(getattr(nf, "hdiff_nonlinear", False))
    if not ((nonlinear or np.all(Kh == Kh.flat[0])) and np.all(dd == dd.flat[0])):
        raise NotImplementedError("cuda backend: only spatially uniform (DIRECT) diffusion coefficients "
                                  "or the NONLINEAR1 hyperdiffusion")
    g["Kh_coef"], g["divdamp_coef"] = (0.0 if nonlinear else float(Kh.flat[0])), float(dd.flat[0])
    if nonlinear:
        # NONLINEAR1: the device forms Kh every large step from the temperature
        # Laplacian; its per-level upper bound (height_factor, mod_numfilter.py:
        # 832-843, 920-922), lower bound and the mean cell area
        z, htop, zd = np.asarray(m.grd.GRD_gz), m.grd.GRD_htop, nf.ZD_hdiff_nl
        pi = getattr(m.cnst, "CONST_PI", np.pi)
        fact = np.zeros(len(z))
        for k in range(len(z)):
            sw = 0.5 + np.sign(z[k] - zd) * 0.5
            fact[k] = sw * 0.5 * (1.0 - np.cos(pi * (z[k] - zd) / (htop - zd)))
        g["hdiff_nl_kh_max"] = (1.0 - fact) * nf.Kh_coef_maxlim + fact * nf.Kh_coef_minlim
        g["hdiff_nl_minlim"] = float(nf.Kh_coef_minlim)
        g["hdiff_nl_area"] = float(nf.AREA_ave)
    if getattr(nf, "NUMFILTER_DOrayleigh", False):   # the sponge coefficients (mod_numfilter.py:225-233)
        g["rayleigh_coef"] = np.asarray(nf.rayleigh_coef, np.float64)
        g["rayleigh_coef_h"] = np.asarray(nf.rayleigh_coef_h, np.float64)
        g["rayleigh_only_w"] = int(bool(getattr(nf, "rayleigh_damp_only_w", False)))
    g["sstep"] = np.asarray(m.dyn.num_of_iteration_sstep[:m.dyn.num_of_iteration_lstep])
    g["CVW"] = np.asarray(m.rcnf.CVW)
    g["NQW_END"] = int(m.rcnf.NQW_END)
    co = m.comm
    g["copy_r2r"] = co.Copy_list_r2r[:, :int(co.Copy_info_r2r[co.I_size])].astype(np.int64)
    g["copy_p2r"] = co.Copy_list_p2r[:, :int(co.Copy_info_p2r[co.I_size])].astype(np.int64)
    g["copy_r2p"] = co.Copy_list_r2p[:, :int(co.Copy_info_r2p[co.I_size])].astype(np.int64)
    g["copy_sgp"] = co.Singular_list[:, :int(co.Singular_info[co.I_size])].astype(np.int64)
    for k, v in vars(m.vmtr).items():
        if k.startswith("VMTR_") and isinstance(v, np.ndarray):
            g[k] = v
    for k in ("GRD_x", "GRD_x_pl", "GRD_xr", "GRD_xr_pl", "GRD_afact", "GRD_bfact", "GRD_cfact", "GRD_dfact",
              "GRD_rdgz", "GRD_rdgzh"):
        g[k] = getattr(m.grd, k)
    for k in ("OPRT_coef_div", "OPRT_coef_grad", "OPRT_coef_lap", "OPRT_coef_intp", "OPRT_coef_diff"):
        g[k] = getattr(m.oprt, k)
        g[k + "_pl"] = getattr(m.oprt, k + "_pl")
    for k in ("GMTR_t", "GMTR_a", "GMTR_p"):
        g[k] = getattr(m.gmtr, k)
        g[k + "_pl"] = getattr(m.gmtr, k + "_pl")
    for k in ("rho_bs", "pre_bs", "tem_bs"):
        g[k] = getattr(m.bsst, k)
        g[k + "_pl"] = getattr(m.bsst, k + "_pl")
    if m.tim.TIME_integ_type == "TRCADV":
        # the coordinates of the prescribed winds (mod_forcing.py forcing_update)
        K0 = m.adm.ADM_K0
        grd = m.grd
        g["integ_type"] = "TRCADV"
        if getattr(m.rcnf, "DCTEST_case", "1-1") == "1-2":   # the Hadley-like circulation's winds
            g["trcadv_case"] = "1-2"
        g["GRD_LON"] = np.ascontiguousarray(grd.GRD_LON[:, :, K0, :])
        g["GRD_LAT"] = np.ascontiguousarray(grd.GRD_LAT[:, :, K0, :])
        g["GRD_LON_pl"] = np.ascontiguousarray(grd.GRD_LON_pl[:, K0, :])
        g["GRD_LAT_pl"] = np.ascontiguousarray(grd.GRD_LAT_pl[:, K0, :])
        g["GRD_Z"] = np.ascontiguousarray(grd.GRD_vz[:, :, :, :, grd.GRD_Z])
        g["GRD_ZH"] = np.ascontiguousarray(grd.GRD_vz[:, :, :, :, grd.GRD_ZH])
        g["GRD_Z_pl"] = np.ascontiguousarray(grd.GRD_vz_pl[:, :, :, grd.GRD_Z])
        g["GRD_ZH_pl"] = np.ascontiguousarray(grd.GRD_vz_pl[:, :, :, grd.GRD_ZH])
    elif getattr(m.rcnf, "AF_TYPE", "NONE") == "DCMIP":
        # Kessler microphysics only (checked by CudaDyn._check_config): the
        # full-level heights it reads and the forcing's flags (mod_forcing.py:44-71)
        g["AF_dcmip_kessler"] = 1
        g["GRD_Z"] = np.ascontiguousarray(m.grd.GRD_vz[:, :, :, :, m.grd.GRD_Z])
        frc = getattr(m, "frc", None)
        g["AF_negative_fixer"] = int(bool(getattr(frc, "NEGATIVE_FIXER", False)))
        g["AF_update_tot_dens"] = int(bool(getattr(frc, "UPDATE_TOT_DENS", True)))
        fl = _dcmip_flags(msc)
        K0 = m.adm.ADM_K0
        g["AF_dcmip_schemes"] = np.asarray([fl["USE_Kessler"], fl["USE_SimpleMicrophys"], fl["SM_Latdepend_SST"],
                                            fl["SM_LargeScaleCond"], fl["USE_HeldSuarez"], fl["SM_MITC_SST_TYPE"],
                                            fl["SM_PBL_Bryan"]], np.int64)
        if fl["USE_ToyChemistry"] or fl["USE_SimpleMicrophys"] or fl["USE_HeldSuarez"]:
            g["AF_dcmip_lat"] = np.ascontiguousarray(m.grd.GRD_LAT[:, :, K0, :])
        if fl["USE_ToyChemistry"]:   # terminator chemistry on the Cl / Cl2 tracers
            g["AF_dcmip_chem"] = np.asarray([m.rcnf.NCHEM_STR, m.rcnf.NCHEM_END], np.int64)
            g["AF_dcmip_lon"] = np.ascontiguousarray(m.grd.GRD_LON[:, :, K0, :])
        if fl["USE_SimpleMicrophys"]:   # the simple physics' geometry (mod_forcing.py:236-247)
            gm = m.gmtr
            g["AF_dcmip_zh"] = np.ascontiguousarray(m.grd.GRD_vz[:, :, :, :, m.grd.GRD_ZH])
            g["AF_dcmip_zsfc"] = np.ascontiguousarray(m.grd.GRD_zs[:, :, K0, :, m.grd.GRD_ZSFC])
            g["AF_dcmip_ij"] = np.ascontiguousarray(np.stack(
                [gm.GMTR_p[:, :, K0, :, n] for n in (gm.GMTR_p_IX, gm.GMTR_p_IY, gm.GMTR_p_IZ, gm.GMTR_p_JX,
                                                     gm.GMTR_p_JY, gm.GMTR_p_JZ)], axis=-1))
    elif getattr(m.rcnf, "AF_TYPE", "NONE") == "HELD-SUAREZ":
        # the column latitudes the forcing reads (mod_dynamics.py: GRD_LAT[:, :, K0, :])
        g["GRD_LAT"] = np.ascontiguousarray(m.grd.GRD_LAT[:, :, m.adm.ADM_K0, :])
    g.update(_history_setup(m))
    return {k: np.asarray(v) for k, v in g.items()}


def pole_centre_sources(m):
    """the p2r copies COMM_var reverses to fill the pole centres
    (share/mod_comm.py:2249-2262): rows [pole g, pole l, i, j, l] of the copies
    whose regional side belongs to the region the pole is assigned to"""
    a, co = m.adm, m.comm
    cl = co.Copy_list_p2r
    rows = []
    for ipos in range(int(co.Copy_info_p2r[co.I_size])):
        l_reg = int(cl[co.I_l_to, ipos])
        r = a.RGNMNG_lp2r[l_reg, co.Copy_info_p2r[co.I_prc_to]]
        if r == a.RGNMNG_rgn4pl[a.I_NPL] or r == a.RGNMNG_rgn4pl[a.I_SPL]:
            rows.append([int(cl[co.I_gridi_from, ipos]), int(cl[co.I_l_from, ipos]), int(cl[co.I_gridi_to, ipos]),
                         int(cl[co.I_gridj_to, ipos]), l_reg])
    return np.asarray(rows, np.int64).reshape(-1, 5)


def _history_setup(m) -> dict:
    """what the derived history diagnostics read (mod_history_vars.py:30-186,
    nhm/share/mod_saturation.py): height, latitude, surface height, layer
    thicknesses, the GMTR_p east/north vectors and cell areas at K0, the
    saturation constants and the tracer indices; empty when the services do
    not carry them (the handle then has no history diagnostics)"""
    try:
        K0 = m.adm.ADM_K0
        grd, gm, cn, st, r = m.grd, m.gmtr, m.cnst, m.satr, m.rcnf
        h = {"hist_hgt": np.ascontiguousarray(grd.GRD_vz[:, :, :, :, grd.GRD_Z]),
             "hist_lat": np.ascontiguousarray(grd.GRD_LAT[:, :, K0, :]),
             "hist_zsfc": np.ascontiguousarray(grd.GRD_zs[:, :, K0, :, grd.GRD_ZSFC]),
             "hist_dgz": np.asarray(grd.GRD_dgz),
             "hist_area": np.ascontiguousarray(gm.GMTR_area),
             "hist_IJ": np.stack([gm.GMTR_p[:, :, K0, :, i] for i in (gm.GMTR_p_IX, gm.GMTR_p_IY, gm.GMTR_p_IZ,
                                                                       gm.GMTR_p_JX, gm.GMTR_p_JY, gm.GMTR_p_JZ)],
                                 axis=-1),
             "hist_LHV": cn.CONST_LHV, "hist_UNDEF": cn.CONST_UNDEF, "hist_PSAT0": cn.CONST_PSAT0,
             "hist_RTEM00": st.RTEM00, "hist_CPovR_liq": st.CPovR_liq, "hist_CPovR_ice": st.CPovR_ice,
             "hist_LovR_liq": st.LovR_liq, "hist_LovR_ice": st.LovR_ice,
             "hist_SAT_LLIMIT": st.SATURATION_LLIMIT_TEMP, "hist_SAT_ULIMIT": st.SATURATION_ULIMIT_TEMP,
             "hist_I_QV": r.I_QV}
        for k in ("I_QC", "I_QR", "I_QI", "I_QS", "I_QG"):
            h["hist_" + k] = getattr(r, k, -1)
        if getattr(r, "AF_TYPE", "") == "DCMIP" and getattr(r, "NCHEM_STR", -1) >= 0:   # mod_io.py:259-261
            h["hist_NCHEM"] = np.asarray([r.NCHEM_STR, r.NCHEM_END], np.int64)
    except AttributeError:
        return {}
    return h


class CudaDyn:
    """Device-resident replacement of the reference's ``Dyn`` step API."""

    def __init__(self, msc=None, geo: dict = None, graph: bool = True, precision: str = "float64"):
        """``precision``: "float64" or "mixed" (see ``NicamCuda``); the
        reference selects its working precision with
        ``Backend.configure(name, precision)`` (share/mod_backend.py:175)."""
        if geo is None:
            if msc is None:
                raise ValueError("CudaDyn needs the reference services (msc) or a setup dict (geo)")
            self._check_config(msc)
            geo = geo_from_msc(msc)
        self.core = NicamCuda(geo, graph=graph, precision=precision)
        self._forced = ("GRD_LAT" in geo and str(np.asarray(geo.get("integ_type", "RK3"))) != "TRCADV") or \
            bool(int(np.asarray(geo.get("AF_dcmip_kessler", 0))))
        self._kessler = bool(int(np.asarray(geo.get("AF_dcmip_kessler", 0))))
        self._hist_chem = "hist_NCHEM" in geo
        self._host_stale = False
        self._device_valid = False

    @staticmethod
    def _check_config(msc):
        r = msc.rcnf
        if msc.tim.TIME_integ_type == "TRCADV":
            if (getattr(r, "DCTEST_type", "") != "Traceradvection" or getattr(r, "DCTEST_case", "") not in ("1-1", "1-2")):
                raise NotImplementedError("cuda backend: offline tracer advection with the DCMIP 1-1 or 1-2 winds")
        elif msc.tim.TIME_integ_type != "RK3":
            raise NotImplementedError("cuda backend: RK3 time integration or TRCADV only")
        if r.TRC_ADV_TYPE != "MIURA2004" or not r.THUBURN_LIM:
            raise NotImplementedError("cuda backend: MIURA2004 tracer advection with Thuburn limiters only")
        nf = msc.numf
        if nf.lap_order_hdiff != 2 or nf.lap_order_divdamp != 2 or \
                nf.NUMFILTER_DOdivdamp_2d or nf.NUMFILTER_DOdivdamp_v or nf.NUMFILTER_DOhorizontaldiff_lap1:
            raise NotImplementedError("cuda backend: lap_order 2 hyperdiffusion (DIRECT or NONLINEAR1) and 3-D "
                                      "divdamp, optionally the Rayleigh sponge; no 2-D/vertical divdamp or lap1")
        if r.DYN_DIV_NUM != 1:
            raise NotImplementedError("cuda backend: DYN_DIV_NUM = 1 only")
        if int(getattr(r, "NQW_STR", 0)) != 0 or int(getattr(r, "I_QV", 0)) != 0 or \
                int(getattr(r, "NQW_END", 0)) >= 6:
            raise NotImplementedError("cuda backend: water tracers must come first (NQW_STR = I_QV = 0), at most six")
        if getattr(r, "AF_TYPE", "NONE") == "DCMIP":
            flags = _dcmip_flags(msc)
            rain = getattr(r, "RAIN_TYPE", "DRY")
            if not (flags.get("USE_Kessler") or flags.get("USE_SimpleMicrophys")) \
                    or rain not in ("WARM", "DRY") or (flags.get("USE_Kessler") and rain != "WARM") or \
                    (flags.get("USE_ToyChemistry") and int(getattr(r, "NCHEM_END", -1)) - int(getattr(r, "NCHEM_STR", -1)) != 1):
                raise NotImplementedError("cuda backend: DCMIP forcing with Kessler microphysics (RAIN_TYPE WARM) "
                                          "and / or the simple physics (WARM or DRY), optionally the terminator "
                                          "chemistry (two tracers) and moist Held-Suarez")
        elif getattr(r, "AF_TYPE", "NONE") not in ("NONE", "HELD-SUAREZ"):
            raise NotImplementedError("cuda backend: artificial forcing NONE or HELD-SUAREZ only")

    # -- the reference's step API -------------------------------------------
    def dynamics_step(self, msc):
        self._ensure_device(msc)
        self.core.step(1)
        self._host_stale = True

    def run_timeloop_chunk(self, msc, K: int):
        """K large steps; with the Held-Suarez forcing active each step is
        followed by the forcing step, as in the reference's per-step loop
        (pynicamdc/api.py:724-730)"""
        self._ensure_device(msc)
        if self._forced:
            for _ in range(int(K)):
                self.core.step(1)
                self.core.forcing_step()
        else:
            self.core.step(int(K))
        self._host_stale = True

    def forcing_step(self, msc):
        af = getattr(msc.rcnf, "AF_TYPE", "NONE")
        if af in ("NONE", None):
            return None
        if af not in ("HELD-SUAREZ", "DCMIP") or not self._forced or (af == "DCMIP") != self._kessler:
            raise NotImplementedError(f"cuda backend: artificial forcing {af!r} is not configured on the device")
        self._ensure_device(msc)
        self.core.forcing_step()
        self._host_stale = True
        if self._kessler:   # the reference's forcing_step returns the precipitation for DCMIP
            return self.core.forcing_precip()
        return None

    def history_vars_step(self, msc, write_3d=True, write_2d=True):
        """Dyn.history_vars_step (mod_dynamics.py:737-772): the derived history
        diagnostics of the current state, computed on the device
        (nc_history_vars) and returned as host arrays; the names are the I/O
        groups being written (``msc.io._diag_names`` / ``_diag_names_2d``), all
        of them without an I/O object.  The tendencies keep their previous
        output on the device, as the reference's ``Hvar`` keeps it."""
        io = getattr(msc, "io", None)
        active = None
        if io is not None:
            active = set()
            if write_3d:
                active |= set(getattr(io, "_diag_names", []))
            if write_2d:
                active |= set(getattr(io, "_diag_names_2d", []))
        every = HIST_ITEMS if self._hist_chem else tuple(n for n in HIST_ITEMS if n not in HIST_CHEM)
        names = every if active is None else tuple(n for n in every if n in active)
        if active is not None and active & set(HIST_CHEM) and not self._hist_chem:
            raise NotImplementedError("cuda backend: the chemistry's history columns need AF_TYPE 'DCMIP' "
                                      "with the terminator chemistry")
        if active is not None and active - set(HIST_ITEMS):
            raise NotImplementedError(f"cuda backend: history diagnostics {sorted(active - set(HIST_ITEMS))} "
                                      "are not built on the device")
        self._ensure_device(msc)
        return self.core.history_vars(names, nstep=msc.tim.TIME_cstep, dt=msc.tim.TIME_dtl)

    def restart_output(self, msc, basename: str, ctime: int = 0):
        """Prgvar.restart_output (nhm/share/mod_prgvar.py:182-216) for
        output_io_mode "ADVANCED" and the prognostic items, written from the
        device state without a host copy of PRG_var: <basename>000000 (one
        process holds every region)."""
        prgv = msc.prgv
        if prgv.output_io_mode != "ADVANCED" or getattr(prgv, "output_diagnostics", False):
            raise NotImplementedError("cuda backend: restart output in the ADVANCED (fio) format with the "
                                      "prognostic variables only")
        items = [(name, desc, unit, slot) for (name, desc, unit, _src, slot) in
                 prgv._restart_output_items(msc.rcnf)]
        self._ensure_device(msc)
        a = msc.adm
        rgnid = [int(a.RGNMNG_lp2r[l, a.ADM_prc_me]) for l in range(a.ADM_lall)]
        restart.write(self.core, basename + "0" * 6, items, prgv.layername, rgnid, a.ADM_glevel, a.ADM_rlevel,
                      ctime)

    def restart_input(self, msc):
        """Prgvar.restart_input's prognostic read (nhm/share/mod_prgvar.py:266-330)
        of <restart_input_basename>000000 in the ADVANCED (fio) format straight
        into the device state (COMM_var included); the host PRG_var is then
        stale."""
        prgv, r = msc.prgv, msc.rcnf
        if prgv.input_io_mode != "ADVANCED" or getattr(prgv, "input_diagnostics", False):
            raise NotImplementedError("cuda backend: restart input in the ADVANCED (fio) format, prognostic read")
        names = [r.PRG_name[v] for v in range(r.PRG_vmax0)] + ["rhog" + r.TRC_name[q] for q in range(r.TRC_vmax)]
        restart.read(self.core, prgv.restart_input_basename + "0" * 6, names, pole_centre_sources(msc),
                     allow_missingq=bool(getattr(prgv, "allow_missingq", False)))
        self._device_valid = True
        self._host_stale = True

    def sync_prgvar_to_host(self, prgv, msc=None):
        if not self._device_valid:
            return
        self.core.download(prgv.PRG_var, prgv.PRG_var_pl)
        self._host_stale = False

    def assert_host_prgvar_synced(self, who: str = ""):
        if self._host_stale:
            raise AssertionError(f"host PRG_var read while the device state is newer ({who}); "
                                 "call sync_prgvar_to_host first")

    def _ensure_device(self, msc):
        if not self._device_valid:
            pv, pvp = msc.prgv.PRG_var, msc.prgv.PRG_var_pl
            self.core.upload(np.ascontiguousarray(pv), np.ascontiguousarray(pvp))
            self._device_valid = True

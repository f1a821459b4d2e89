"""A stand-in for the reference's model services (``msc``) built from a golden
fixture, with the attribute names and shapes the reference's objects carry
(adm, cnst, grd, gmtr, oprt, vmtr, bsst, comm, rcnf, tim, numf, dyn, ppm,
prgv).  Lets the tests drive ``CudaDyn`` through the reference's step API
(``dynamics_step(msc)``, ``sync_prgvar_to_host(prgv, msc)``, ...) where the
reference package itself is not installed."""
from __future__ import annotations

from types import SimpleNamespace as NS

import numpy as np


def fake_msc(geo: dict, state, state_pl, af_type: str = "NONE", lat=None, integ_type: str = "RK3",
             coords: dict = None, hist: dict = None, io_names=None, dcmip: dict = None,
             numf_opts: dict = None, dctest_case: str = "1-1"):
    g = {k: np.asarray(v) for k, v in geo.items()}
    sc = lambda k: g[k].reshape(-1)[0].item()
    adm = NS(ADM_kall=int(sc("kall")), ADM_kmin=int(sc("kmin")), ADM_kmax=int(sc("kmax")),
             ADM_gall_1d=int(sc("gall_1d")), ADM_gmin=int(sc("gmin")), ADM_gmax=int(sc("gmax")),
             ADM_lall=int(sc("lall")), ADM_have_sgp=g["have_sgp"], ADM_K0=0)
    cnst = NS(CONST_GRAV=sc("GRAV"), CONST_Rdry=sc("Rdry"), CONST_CVdry=sc("CVdry"), CONST_CPdry=sc("CPdry"),
              CONST_Rvap=sc("Rvap"), CONST_OHM=sc("OHM"), CONST_RADIUS=sc("RADIUS"), CONST_EPS=sc("EPS"),
              CONST_HUGE=sc("HUGE"), CONST_PRE00=sc("PRE00"))
    if hist is not None:
        cnst.CONST_LHV, cnst.CONST_UNDEF, cnst.CONST_PSAT0 = (np.asarray(hist[k]).item()
                                                            for k in ("LHV", "UNDEF", "PSAT0"))
    grd = NS(GRD_rscale=sc("rscale"))
    for k in ("GRD_x", "GRD_x_pl", "GRD_xr", "GRD_xr_pl", "GRD_afact", "GRD_bfact", "GRD_cfact", "GRD_dfact",
              "GRD_rdgz", "GRD_rdgzh"):
        setattr(grd, k, g[k])
    if lat is not None:
        grd.GRD_LAT = np.asarray(lat)[:, :, None, :]
    if coords is not None:   # offline tracer advection: lon/lat at K0 and the heights
        grd.GRD_Z, grd.GRD_ZH = 0, 1
        grd.GRD_LON = coords["GRD_LON"][:, :, None, :]
        grd.GRD_LAT = coords["GRD_LAT"][:, :, None, :]
        grd.GRD_LON_pl = coords["GRD_LON_pl"][:, None, :]
        grd.GRD_LAT_pl = coords["GRD_LAT_pl"][:, None, :]
        grd.GRD_vz = np.stack([coords["GRD_Z"], coords["GRD_ZH"]], axis=-1)
        grd.GRD_vz_pl = np.stack([coords["GRD_Z_pl"], coords["GRD_ZH_pl"]], axis=-1)
    gmtr = NS(**{k: g[k] for k in ("GMTR_t", "GMTR_a", "GMTR_p", "GMTR_t_pl", "GMTR_a_pl", "GMTR_p_pl")})
    satr = None
    if hist is not None:   # what the history diagnostics read (make_hist.py's extra setup)
        grd.GRD_Z, grd.GRD_ZSFC = 0, 0
        grd.GRD_vz = np.asarray(hist["GRD_Z"])[..., None]
        grd.GRD_LAT = np.asarray(hist["GRD_LAT"])[:, :, None, :]
        grd.GRD_zs = np.asarray(hist["GRD_zsfc"])[:, :, None, :, None]
        grd.GRD_dgz = np.asarray(hist["GRD_dgz"])
        gmtr.GMTR_area = np.asarray(hist["GMTR_area"])
        gmtr.GMTR_p_IX, gmtr.GMTR_p_IY, gmtr.GMTR_p_IZ, gmtr.GMTR_p_JX, gmtr.GMTR_p_JY, gmtr.GMTR_p_JZ = range(2, 8)
        h = lambda k: np.asarray(hist[k]).item()
        satr = NS(RTEM00=h("RTEM00"), CPovR_liq=h("CPovR_liq"), CPovR_ice=h("CPovR_ice"), LovR_liq=h("LovR_liq"),
                  LovR_ice=h("LovR_ice"), SATURATION_LLIMIT_TEMP=h("SAT_LLIMIT"),
                  SATURATION_ULIMIT_TEMP=h("SAT_ULIMIT"))
    oprt = NS(**{k: g[k] for k in g if k.startswith("OPRT_")})
    vmtr = NS(**{k: g[k] for k in g if k.startswith("VMTR_")})
    bsst = NS(**{k: g[k] for k in ("rho_bs", "pre_bs", "tem_bs", "rho_bs_pl", "pre_bs_pl", "tem_bs_pl")})
    comm = NS(I_size=0)
    for name, key in (("r2r", "copy_r2r"), ("p2r", "copy_p2r"), ("r2p", "copy_r2p")):
        setattr(comm, "Copy_list_" + name, g[key])
        setattr(comm, "Copy_info_" + name, np.array([g[key].shape[1]]))
    comm.Singular_list = g["copy_sgp"]
    comm.Singular_info = np.array([g["copy_sgp"].shape[1]])
    rcnf = NS(NON_HYDRO_ALPHA=sc("alpha"), CVW=g["CVW"], NQW_STR=0, I_QV=0, NQW_END=int(np.asarray(g.get("NQW_END", 0))), AF_TYPE=af_type, TRC_ADV_TYPE="MIURA2004",
              THUBURN_LIM=True, DYN_DIV_NUM=1,
              DCTEST_type="Traceradvection" if integ_type == "TRCADV" else "",
              DCTEST_case=dctest_case if integ_type == "TRCADV" else "")
    tim = NS(TIME_dtl=sc("dtl"), TIME_dts=sc("dts"), TIME_integ_type=integ_type, TIME_cstep=0)
    if hist is not None:
        for k in ("I_QV", "I_QC", "I_QR", "I_QI", "I_QS", "I_QG"):
            setattr(rcnf, k, int(np.asarray(hist[k]).item()))
    n = int(sc("gall_1d")) ** 2 * int(sc("lall"))
    numf = NS(hdiff_fact_rho=sc("hdiff_fact_rho"), Kh_coef=np.full(n, sc("Kh_coef")),
              divdamp_coef=np.full(n, sc("divdamp_coef")), lap_order_hdiff=2, lap_order_divdamp=2,
              NUMFILTER_DOrayleigh=False, NUMFILTER_DOdivdamp_2d=False, NUMFILTER_DOdivdamp_v=False,
              NUMFILTER_DOhorizontaldiff_lap1=False, hdiff_nonlinear=False)
    if numf_opts:   # numfilter options (NONLINEAR1 bounds and mean cell area, Rayleigh coefficients)
        for k, v in numf_opts.items():
            setattr(numf, k, v)
    if "GRD_gz" in g:   # the level heights and model-top height the NONLINEAR1 bounds read
        grd.GRD_gz = g["GRD_gz"]
        grd.GRD_htop = g["GRD_gzh"][int(sc("kmax")) + 1] - g["GRD_gzh"][int(sc("kmin"))]
    sstep = g["sstep"].astype(np.int64)
    dyn = NS(num_of_iteration_lstep=len(sstep), num_of_iteration_sstep=np.concatenate([sstep, np.zeros(4, np.int64)]))
    ppm = NS(pntmask=g["pntmask"])
    prgv = NS(PRG_var=np.array(state, copy=True), PRG_var_pl=np.array(state_pl, copy=True))
    m = NS(adm=adm, cnst=cnst, grd=grd, gmtr=gmtr, oprt=oprt, vmtr=vmtr, bsst=bsst, comm=comm, rcnf=rcnf,
           tim=tim, numf=numf, dyn=dyn, ppm=ppm, prgv=prgv)
    if satr is not None:
        m.satr = satr
    if dcmip is not None:   # DCMIP forcing: the schemes of dcmip_flags (Kessler only when absent)
        chem = "NCHEM_STR" in dcmip
        fl = [int(x) for x in dcmip.get("dcmip_flags", (1, 0, 0, 0, 0, 1, 0))]
        grd.GRD_Z, grd.GRD_ZH, grd.GRD_ZSFC = 0, 1, 0
        zh = dcmip.get("GRD_ZH", dcmip["GRD_Z"])
        grd.GRD_vz = np.stack([np.asarray(dcmip["GRD_Z"]), np.asarray(zh)], axis=-1)
        if "GRD_LAT" in dcmip:
            grd.GRD_LAT = np.asarray(dcmip["GRD_LAT"])[:, :, None, :]
            grd.GRD_LON = np.asarray(dcmip["GRD_LON"])[:, :, None, :]
        if chem:
            rcnf.NCHEM_STR, rcnf.NCHEM_END = int(dcmip["NCHEM_STR"]), int(dcmip["NCHEM_END"])
        if fl[1]:   # the simple physics' surface height; its unit vectors are GMTR_p columns 2..7
            grd.GRD_zs = np.asarray(dcmip["GRD_zsfc"])[:, :, None, :, None]
            gmtr.GMTR_p_IX, gmtr.GMTR_p_IY, gmtr.GMTR_p_IZ, gmtr.GMTR_p_JX, gmtr.GMTR_p_JY, gmtr.GMTR_p_JZ = range(2, 8)
            assert np.array_equal(gmtr.GMTR_p[:, :, 0, :, 2:8], dcmip["GMTR_p_IJ"])
        rcnf.RAIN_TYPE = "WARM" if int(np.asarray(g.get("NQW_END", 0))) == 2 else "DRY"
        m.afdcmip = NS(USE_Kessler=bool(fl[0]), USE_SimpleMicrophys=bool(fl[1]), SM_Latdepend_SST=bool(fl[2]),
                       SM_LargeScaleCond=bool(fl[3]), SM_PBL_Bryan=bool(fl[6]), USE_ToyChemistry=chem,
                       USE_HeldSuarez=bool(fl[4]), SM_MITC_SST_TYPE=fl[5])
        m.frc = NS(NEGATIVE_FIXER=False, UPDATE_TOT_DENS=True)
    if io_names is not None:   # the I/O object's diagnostic groups (share/mod_io.py:248-265)
        m.io = NS(_diag_names=[n for n in io_names if n.startswith("ml_")],
                  _diag_names_2d=[n for n in io_names if n.startswith("sl_")])
    return m

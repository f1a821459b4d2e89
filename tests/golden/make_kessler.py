"""Generate the DCMIP forcing fixtures by running the reference itself.

The gl03 z10 RAIN_TYPE WARM case of make_golden.py (reference prep tools, JW
balanced jet, seeded vapour / cloud / rain fields) with the reference's DCMIP
artificial forcing switched on with Kessler warm-rain microphysics only
(runconfparam AF_TYPE = 'DCMIP', forcing_dcmip_param USE_Kessler = true; the
scheme set of DCMIP2016 case 1-3): every large step is Dyn.dynamics_step
followed by Dyn.forcing_step (pynicamdc/api.py:724-730).  Stores the setup
arrays, the full-level heights GRD_vz[..., GRD_Z] the microphysics reads, and
the states before and after two forced steps.  With --chem the run also
carries the two chemistry tracers Cl and Cl2 (CHEM_TYPE PASSIVE,
CHEM_TRC_vmax 2) with the DCMIP terminator toy chemistry on
(USE_ToyChemistry), started at half and one and a half times the reaction's
equilibrium so that it acts, and the column latitudes and longitudes the
chemistry reads are stored too, with the reference's history columns of the
chemistry (sl_cl, sl_cl2, sl_cly) of the last state and the set-up arrays the
history diagnostics read (hgeo.*).  --case dcmip11 adds the DCMIP simple physics
(USE_SimpleMicrophys with the latitude-dependent sea-surface temperature, no
large-scale condensation: the scheme set of DCMIP2016 case 1-1) to Kessler
and the chemistry; --case smlsc runs the simple physics alone with its
large-scale condensation and the constant sea-surface temperature; --case dcmip21 the moist
Held-Suarez scheme set of DCMIP2016 case 2-1; --case dcmip12bryan the
tropical-cyclone scheme set with the Bryan boundary layer; --case smdry the
simple physics with RAIN_TYPE DRY (vapour the only water tracer).  They
also store the half-level heights, the surface height and the column unit
vectors the simple physics reads.

    python tests/golden/make_kessler.py --ref <pyNICAM-DC checkout> --out tests/golden [--chem | --case NAME]
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402

GL, VL, ZTOP, DTL, GAMMA, NSTEPS = 3, 10, 30000.0, 1200.0, 7.68e17, 2


# case name: (forcing_dcmip_param, terminator chemistry)
CASES = {
    "kessler": ({"USE_Kessler": True}, False),
    "kessler_chem": ({"USE_Kessler": True}, True),
    "dcmip11": ({"USE_Kessler": True, "USE_SimpleMicrophys": True, "SM_Latdepend_SST": True,
                 "SM_LargeScaleCond": False}, True),
    "smlsc": ({"USE_Kessler": False, "USE_SimpleMicrophys": True, "SM_Latdepend_SST": False,
               "SM_LargeScaleCond": True}, False),
    # the DCMIP2016 case 1-2 (tropical cyclone) scheme set with the Bryan boundary layer
    "dcmip12bryan": ({"USE_Kessler": True, "USE_SimpleMicrophys": True, "SM_Latdepend_SST": False,
                      "SM_LargeScaleCond": False, "SM_PBL_Bryan": True}, False),
    # the simple physics with RAIN_TYPE DRY (vapour the only water tracer; the DCMIP2016 DRY presets)
    "smdry": ({"USE_Kessler": False, "USE_SimpleMicrophys": True, "SM_Latdepend_SST": True,
               "SM_LargeScaleCond": True}, False),
    # DCMIP2016 case 2-1, moist Held-Suarez (the SET_DCMIP2016_21 scheme set)
    "dcmip21": ({"USE_Kessler": True, "USE_SimpleMicrophys": True, "SM_Latdepend_SST": False,
                 "SM_LargeScaleCond": False, "USE_HeldSuarez": True}, False),
}


# RAIN_TYPE of a case (WARM where absent): the simple physics alone also runs dry
RAIN = {"smdry": "DRY"}
# the Bryan boundary layer mixes below 1 km: 30 layers put the lowest ones there
VLAYERS = {"dcmip12bryan": 30}


def run(ref: str, out_dir: str, case: str = "kessler"):
    import toml
    flags, chem = CASES[case]
    sm = bool(flags.get("USE_SimpleMicrophys", False))
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "kessler")
        vl = VLAYERS.get(case, VL)
        MG.prep(ref, case_dir, GL, vl, ZTOP)
        rain = RAIN.get(case, "WARM")
        c = toml.loads(MG.model_toml(ref, GL, vl, DTL, GAMMA, NSTEPS, rain))
        c["runconfparam"]["AF_TYPE"] = "DCMIP"
        c["forcing_dcmip_param"] = dict(flags)
        if chem:
            c["runconfparam"]["CHEM_TYPE"] = "PASSIVE"
            c["chemvarparam"] = {"CHEM_TRC_vmax": 2}
            c["forcing_dcmip_param"]["USE_ToyChemistry"] = True
        with open(os.path.join(case_dir, "case", "config", "nhm_jw.toml"), "w") as f:
            f.write(toml.dumps(c))
        with open(os.path.join(case_dir, "drv.toml"), "w") as f:
            f.write('[driver]\nbackend="numpy"\nprecision="float64"\ncomm="serial"\n'
                    'nhm_driver_cnf="./case/config/nhm_jw.toml"\n')
        os.chdir(case_dir)
        for n in ("dask", "dask.array", "zarr", "xarray"):
            sys.modules.setdefault(n, types.ModuleType(n))
        sys.modules["dask"].array = sys.modules["dask.array"]
        sys.path.insert(0, ref)
        from pynicamdc.api import pyNICAM
        nic = pyNICAM("drv.toml")
        import pynicamdc.share.mod_io as mio
        from pynicamdc.nhm.forcing.mod_af_dcmip import afdcmip

        class _NoIo:
            PRGout_interval = 10 ** 9
            PRGout_interval_2d = 10 ** 9
            PRGout_step0 = False
            PRGout_diagnostics = False

            def IO_setup(self, *a, **k):
                pass

            def IO_PRGstep(self, *a, **k):
                pass

            def IO_finalize(self):
                pass
        mio.Io = _NoIo
        nic.initialize()
        m = nic.msc
        assert m.rcnf.AF_TYPE == "DCMIP" and afdcmip.USE_SimpleMicrophys == sm
        for k, v in flags.items():
            assert getattr(afdcmip, k) == v, k
        assert afdcmip.USE_ToyChemistry == chem and afdcmip.SM_MITC_SST_TYPE == 1
        nw = 3 if rain == "WARM" else 1   # vapour, cloud, rain / vapour only
        assert m.rcnf.NQW_END == nw - 1 and m.rcnf.I_QV == 0
        assert not m.frc.NEGATIVE_FIXER and m.frc.UPDATE_TOT_DENS
        pv, pvp = m.prgv.PRG_var, m.prgv.PRG_var_pl
        kk = pv.shape[2]
        lat, lon = m.grd.GRD_LAT[:, :, 0, :], m.grd.GRD_LON[:, :, 0, :]
        latp, lonp = m.grd.GRD_LAT_pl[:, 0, :], m.grd.GRD_LON_pl[:, 0, :]
        for n in range(nw):
            sc = MG.WATER_SCALE[n]
            pv[..., 6 + n] = pv[..., 0] * sc * np.moveaxis(MG.tracer_field(lat, lon, kk), -1, 2)
            pvp[..., 6 + n] = pvp[..., 0] * sc * np.moveaxis(MG.tracer_field(latp, lonp, kk), -1, 1)
            pv[:, :, 0, :, 6 + n] = 0.0
            pv[:, :, -1, :, 6 + n] = 0.0
            pvp[:, 0, :, 6 + n] = 0.0
            pvp[:, -1, :, 6 + n] = 0.0
        if chem:
            from pynicamdc.nhm.forcing import terminator
            assert (m.rcnf.NCHEM_STR, m.rcnf.NCHEM_END) == (3, 4)
            r2d = 180.0 / np.pi
            for arr, la, lo in ((pv, lat, lon), (pvp, latp, lonp)):
                cl, cl2 = terminator.initial_value_terminator(la * r2d, lo * r2d, np.float64)
                kax = 2 if arr is pv else 1
                q0 = arr[..., 6] / arr[..., 0]
                arr[..., 9] = arr[..., 0] * 0.5 * np.expand_dims(cl, kax) * (1.0 - q0)
                arr[..., 10] = arr[..., 0] * 1.5 * np.expand_dims(cl2, kax) * (1.0 - q0)
        out = {"geo." + k: v for k, v in MG.geo_from_msc(m, pv.shape[-1] - 6).items()}
        K0 = m.adm.ADM_K0
        if chem or sm:
            out["geo.GRD_LAT"] = np.ascontiguousarray(m.grd.GRD_LAT[:, :, K0, :])
            out["geo.GRD_LON"] = np.ascontiguousarray(m.grd.GRD_LON[:, :, K0, :])
        if chem:
            out["geo.NCHEM_STR"], out["geo.NCHEM_END"] = np.asarray(3), np.asarray(4)
        if sm:   # what the simple physics reads besides the state (mod_forcing.py:236-247)
            gm = m.gmtr
            idx = [gm.GMTR_p_IX, gm.GMTR_p_IY, gm.GMTR_p_IZ, gm.GMTR_p_JX, gm.GMTR_p_JY, gm.GMTR_p_JZ]
            out["geo.GMTR_p_IJ"] = np.ascontiguousarray(np.stack([gm.GMTR_p[:, :, K0, :, n] for n in idx], -1))
            out["geo.GRD_ZH"] = np.ascontiguousarray(m.grd.GRD_vz[:, :, :, :, m.grd.GRD_ZH])
            out["geo.GRD_zsfc"] = np.ascontiguousarray(m.grd.GRD_zs[:, :, K0, :, m.grd.GRD_ZSFC])
        out["geo.dcmip_flags"] = np.asarray([int(afdcmip.USE_Kessler), int(afdcmip.USE_SimpleMicrophys),
                                             int(afdcmip.SM_Latdepend_SST), int(afdcmip.SM_LargeScaleCond),
                                             int(afdcmip.USE_HeldSuarez), int(afdcmip.SM_MITC_SST_TYPE),
                                             int(afdcmip.SM_PBL_Bryan)])
        out["geo.GRD_Z"] = np.ascontiguousarray(m.grd.GRD_vz[:, :, :, :, m.grd.GRD_Z])
        out["geo.PRE00"] = np.asarray(m.cnst.CONST_PRE00)
        out["state0"], out["state0_pl"] = pv.copy(), pvp.copy()
        for s in range(NSTEPS):
            nic.run(1)
            out[f"state{s + 1}"], out[f"state{s + 1}_pl"] = m.prgv.PRG_var.copy(), m.prgv.PRG_var_pl.copy()
            out[f"precip{s + 1}"] = np.asarray(m.frc.precip).copy()
        if chem:   # the chemistry's history columns of the last state and what the diagnostics read
            m.io._diag_names, m.io._diag_names_2d = [], ["sl_cl", "sl_cl2", "sl_cly"]
            h = m.dyn.history_vars_step(m)
            assert sorted(h) == ["sl_cl", "sl_cl2", "sl_cly"]
            for k, v in h.items():
                out["hist." + k] = np.asarray(v)
            g, gm, cn, st = m.grd, m.gmtr, m.cnst, m.satr
            hg = dict(GRD_Z=g.GRD_vz[:, :, :, :, g.GRD_Z], GRD_LAT=g.GRD_LAT[:, :, K0, :],
                      GRD_zsfc=g.GRD_zs[:, :, K0, :, g.GRD_ZSFC], GRD_dgz=g.GRD_dgz, GMTR_area=gm.GMTR_area,
                      GMTR_p_IJ=np.stack([gm.GMTR_p[:, :, K0, :, i] for i in (
                          gm.GMTR_p_IX, gm.GMTR_p_IY, gm.GMTR_p_IZ, gm.GMTR_p_JX, gm.GMTR_p_JY, gm.GMTR_p_JZ)], -1),
                      LHV=cn.CONST_LHV, UNDEF=cn.CONST_UNDEF, PSAT0=cn.CONST_PSAT0, RTEM00=st.RTEM00,
                      CPovR_liq=st.CPovR_liq, CPovR_ice=st.CPovR_ice, LovR_liq=st.LovR_liq, LovR_ice=st.LovR_ice,
                      SAT_ULIMIT=st.SATURATION_ULIMIT_TEMP, SAT_LLIMIT=st.SATURATION_LLIMIT_TEMP,
                      NCHEM=np.asarray([m.rcnf.NCHEM_STR, m.rcnf.NCHEM_END]))
            for k in ("I_QV", "I_QC", "I_QR", "I_QI", "I_QS", "I_QG"):
                hg[k] = getattr(m.rcnf, k, -1)
            for k, v in hg.items():
                out["hgeo." + k] = np.ascontiguousarray(np.asarray(v))
    path = os.path.join(out_dir, f"gl03_z{VLAYERS.get(case, VL)}_{case}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--chem", action="store_true", help="the Kessler case with the terminator toy chemistry")
    ap.add_argument("--case", choices=sorted(CASES), default=None)
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out), args.case or ("kessler_chem" if args.chem else "kessler"))

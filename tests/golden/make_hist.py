"""Generate the history-diagnostics fixture by running the reference itself.

The gl03 z10 case of make_golden.py (reference prep tools, JW balanced jet,
sharp injected tracer, the same run as gl03_z10_trc.npz) with every derived
history diagnostic requested: after large step 1 and after large step 2 the
reference's own Dyn.history_vars_step (pynicamdc/nhm/dynamics/mod_dynamics.py:737,
pynicamdc/nhm/driver/mod_history_vars.py) computes the model-level fields
(ml_*), the pressure-level slices and column integrals (sl_*) and the
interval tendencies (ml_d*, seeded by the first call, one step apart at the
second).  Stores the extra setup the diagnostics read (height, latitude,
surface height, layer thicknesses, the saturation constants) and the second
call's outputs; the states are those of gl03_z10_trc.npz (checked here).

    python tests/golden/make_hist.py --ref <pyNICAM-DC checkout> --out tests/golden
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

GL, VL, ZTOP, DTL, GAMMA = 3, 10, 30000.0, 1200.0, 7.68e17

ML = ['ml_u', 'ml_v', 'ml_w', 'ml_th', 'ml_thv', 'ml_omg', 'ml_pres', 'ml_tem', 'ml_rho', 'ml_hgt', 'ml_mse',
      'ml_rh', 'ml_rha', 'ml_rhi', 'ml_du', 'ml_dv', 'ml_dw', 'ml_dtem', 'ml_dq', 'ml_ucos', 'ml_vcos',
      'ml_th_prime']
SL = ['sl_ps', 'sl_pw', 'sl_lwp', 'sl_iwp'] + [f'sl_{f}{lev}' for lev in ('850', '500', '250', '100')
                                              for f in ('u', 'v', 'w', 't')]


def run(ref: str, out_dir: str):
    import toml
    trc = np.load(os.path.join(out_dir, "gl03_z10_trc.npz"))
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "hist")
        MG.prep(ref, case_dir, GL, VL, ZTOP)
        c = toml.loads(MG.model_toml(ref, GL, VL, DTL, GAMMA, 2))
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

        class _NoIo:
            PRGout_interval = 10 ** 9
            PRGout_interval_2d = 10 ** 9
            PRGout_step0 = False
            PRGout_diagnostics = False
            _diag_names = ML
            _diag_names_2d = SL

            def IO_setup(self, *a, **k):
                pass

            def IO_PRGstep(self, *a, **k):
                pass

            def IO_finalize(self):
                pass
        mio.Io = _NoIo
        nic.initialize()
        m = nic.msc
        pv, pvp = m.prgv.PRG_var, m.prgv.PRG_var_pl
        kk = pv.shape[2]
        lat, lon = m.grd.GRD_LAT[:, :, 0, :], m.grd.GRD_LON[:, :, 0, :]
        latp, lonp = m.grd.GRD_LAT_pl[:, 0, :], m.grd.GRD_LON_pl[:, 0, :]
        pv[..., 6] = pv[..., 0] * np.moveaxis(MG.tracer_field(lat, lon, kk), -1, 2)
        pvp[..., 6] = pvp[..., 0] * np.moveaxis(MG.tracer_field(latp, lonp, kk), -1, 1)
        pv[:, :, 0, :, 6] = 0.0
        pv[:, :, -1, :, 6] = 0.0
        pvp[:, 0, :, 6] = 0.0
        pvp[:, -1, :, 6] = 0.0
        assert np.array_equal(pv, trc["state0"])
        dyn = m.dyn
        nic.run(1)
        assert np.array_equal(m.prgv.PRG_var, trc["state1"])
        h1 = dyn.history_vars_step(m)
        n1 = int(m.tim.TIME_cstep)
        nic.run(1)
        assert np.array_equal(m.prgv.PRG_var, trc["state2"])
        h2 = dyn.history_vars_step(m)
        n2 = int(m.tim.TIME_cstep)
        assert sorted(h2) == sorted(ML + SL), sorted(set(ML + SL) ^ set(h2))
        assert all(not np.any(h1[k]) for k in ('ml_du', 'ml_dv', 'ml_dw', 'ml_dtem', 'ml_dq'))

        K0 = m.adm.ADM_K0
        g, gm, cn, st = m.grd, m.gmtr, m.cnst, m.satr
        out = {"hist." + k: np.asarray(v) for k, v in h2.items()}
        out["hist.nstep1"], out["hist.nstep2"] = np.array(n1), np.array(n2)
        out["hist.dtl"] = np.array(m.tim.TIME_dtl)
        out["geo.GRD_Z"] = np.ascontiguousarray(g.GRD_vz[:, :, :, :, g.GRD_Z])
        out["geo.GRD_LAT"] = np.ascontiguousarray(g.GRD_LAT[:, :, K0, :])
        out["geo.GRD_zsfc"] = np.ascontiguousarray(g.GRD_zs[:, :, K0, :, g.GRD_ZSFC])
        out["geo.GRD_dgz"] = np.asarray(g.GRD_dgz)
        out["geo.GMTR_p_IJ"] = np.stack([gm.GMTR_p[:, :, K0, :, i] for i in (
            gm.GMTR_p_IX, gm.GMTR_p_IY, gm.GMTR_p_IZ, gm.GMTR_p_JX, gm.GMTR_p_JY, gm.GMTR_p_JZ)], axis=-1)
        out["geo.GMTR_area"] = np.ascontiguousarray(gm.GMTR_area)
        sat = dict(LHV=cn.CONST_LHV, LHS=cn.CONST_LHS, UNDEF=cn.CONST_UNDEF, PSAT0=cn.CONST_PSAT0,
                   RTEM00=st.RTEM00, CPovR_liq=st.CPovR_liq, CPovR_ice=st.CPovR_ice, LovR_liq=st.LovR_liq,
                   LovR_ice=st.LovR_ice, SAT_ULIMIT=st.SATURATION_ULIMIT_TEMP,
                   SAT_LLIMIT=st.SATURATION_LLIMIT_TEMP, I_QV=m.rcnf.I_QV)
        for k, v in sat.items():
            out["geo." + k] = np.array(v)
        for k in ("I_QC", "I_QR", "I_QI", "I_QS", "I_QG"):
            out["geo." + k] = np.array(getattr(m.rcnf, k, -1))
    path = os.path.join(out_dir, "gl03_z10_hist.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out))

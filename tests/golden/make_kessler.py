"""Generate the DCMIP Kessler forcing fixture by running the reference itself.

The gl03 z10 RAIN_TYPE WARM case of make_golden.py (reference prep tools, JW
balanced jet, seeded vapour / cloud / rain fields) with the reference's DCMIP
artificial forcing switched on with Kessler warm-rain microphysics only
(runconfparam AF_TYPE = 'DCMIP', forcing_dcmip_param USE_Kessler = true; the
scheme set of DCMIP2016 case 1-3): every large step is Dyn.dynamics_step
followed by Dyn.forcing_step (pynicamdc/api.py:724-730).  Stores the setup
arrays, the full-level heights GRD_vz[..., GRD_Z] the microphysics reads, and
the states before and after two forced steps.

    python tests/golden/make_kessler.py --ref <pyNICAM-DC checkout> --out tests/golden
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


def run(ref: str, out_dir: str):
    import toml
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "kessler")
        MG.prep(ref, case_dir, GL, VL, ZTOP)
        c = toml.loads(MG.model_toml(ref, GL, VL, DTL, GAMMA, NSTEPS, "WARM"))
        c["runconfparam"]["AF_TYPE"] = "DCMIP"
        c["forcing_dcmip_param"] = {"USE_Kessler": True}
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
        assert m.rcnf.AF_TYPE == "DCMIP" and afdcmip.USE_Kessler and not afdcmip.USE_SimpleMicrophys
        assert not afdcmip.USE_ToyChemistry and not afdcmip.USE_HeldSuarez
        assert m.rcnf.NQW_END == 2 and (m.rcnf.I_QV, m.rcnf.I_QC, m.rcnf.I_QR) == (0, 1, 2)
        assert not m.frc.NEGATIVE_FIXER and m.frc.UPDATE_TOT_DENS
        pv, pvp = m.prgv.PRG_var, m.prgv.PRG_var_pl
        kk = pv.shape[2]
        lat, lon = m.grd.GRD_LAT[:, :, 0, :], m.grd.GRD_LON[:, :, 0, :]
        latp, lonp = m.grd.GRD_LAT_pl[:, 0, :], m.grd.GRD_LON_pl[:, 0, :]
        for n in range(3):
            sc = MG.WATER_SCALE[n]
            pv[..., 6 + n] = pv[..., 0] * sc * np.moveaxis(MG.tracer_field(lat, lon, kk), -1, 2)
            pvp[..., 6 + n] = pvp[..., 0] * sc * np.moveaxis(MG.tracer_field(latp, lonp, kk), -1, 1)
            pv[:, :, 0, :, 6 + n] = 0.0
            pv[:, :, -1, :, 6 + n] = 0.0
            pvp[:, 0, :, 6 + n] = 0.0
            pvp[:, -1, :, 6 + n] = 0.0
        out = {"geo." + k: v for k, v in MG.geo_from_msc(m, pv.shape[-1] - 6).items()}
        out["geo.GRD_Z"] = np.ascontiguousarray(m.grd.GRD_vz[:, :, :, :, m.grd.GRD_Z])
        out["geo.PRE00"] = np.asarray(m.cnst.CONST_PRE00)
        out["state0"], out["state0_pl"] = pv.copy(), pvp.copy()
        for s in range(NSTEPS):
            nic.run(1)
            out[f"state{s + 1}"], out[f"state{s + 1}_pl"] = m.prgv.PRG_var.copy(), m.prgv.PRG_var_pl.copy()
            out[f"precip{s + 1}"] = np.asarray(m.frc.precip).copy()
    path = os.path.join(out_dir, "gl03_z10_kessler.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out))

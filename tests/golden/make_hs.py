"""Generate the Held-Suarez forcing fixture by running the reference itself.

The gl03 z10 case of make_golden.py (reference prep tools, JW balanced jet,
sharp injected tracer) with the reference's Held-Suarez artificial forcing
switched on (runconfparam AF_TYPE = 'HELD-SUAREZ'): every large step is
Dyn.dynamics_step followed by Dyn.forcing_step (pynicamdc/api.py:724-730).
Stores the setup arrays, the column latitudes GRD_LAT[:, :, K0, :] the forcing
reads, and the states before and after two forced steps.

    python tests/golden/make_hs.py --ref <pyNICAM-DC checkout> --out tests/golden
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
        case_dir = os.path.join(tmp, "hs")
        MG.prep(ref, case_dir, GL, VL, ZTOP)
        c = toml.loads(MG.model_toml(ref, GL, VL, DTL, GAMMA, NSTEPS))
        c["runconfparam"]["AF_TYPE"] = "HELD-SUAREZ"
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

            def IO_setup(self, *a, **k):
                pass

            def IO_PRGstep(self, *a, **k):
                pass

            def IO_finalize(self):
                pass
        mio.Io = _NoIo
        nic.initialize()
        m = nic.msc
        assert m.rcnf.AF_TYPE == "HELD-SUAREZ"
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
        out = {"geo." + k: v for k, v in MG.geo_from_msc(m, pv.shape[-1] - 6).items()}
        out["geo.GRD_LAT"] = np.ascontiguousarray(m.grd.GRD_LAT[:, :, m.adm.ADM_K0, :])
        out["state0"], out["state0_pl"] = pv.copy(), pvp.copy()
        for s in range(NSTEPS):
            nic.run(1)
            out[f"state{s + 1}"], out[f"state{s + 1}_pl"] = m.prgv.PRG_var.copy(), m.prgv.PRG_var_pl.copy()
    path = os.path.join(out_dir, "gl03_z10_hs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out))

"""Generate the offline tracer-advection fixture by running the reference itself.

DCMIP2012 test 1-1 (3-D deformational flow, four passive tracers) in the
reference's TRCADV mode (timeparam integ_type = "TRCADV", runconfparam
DCTEST_type = 'Traceradvection' / DCTEST_case = '1-1', CHEM_TYPE = 'PASSIVE',
init_type = 'Traceradvection'): each large step advects the tracers with the
current winds (MIURA2004 + Thuburn limiters) and then sets the prescribed
winds of the next time (mod_dynamics.py:2030-2085, nhm/forcing/mod_forcing.py
forcing_update, nhm/forcing/mod_af_trcadv.py test11_velocity).  Grid level 3,
10 EVEN layers to 12 km (the tracer case's vertical grid type), dtl 1200 s.
Stores the setup arrays, the column lon/lat, the full- and half-level heights
the wind formulas read, and the states before and after three steps.  With
--case 1-2 the same for test 1-2 (Hadley-like meridional circulation, one
tracer layer; test12_velocity), written to gl03_z10_trcadv12.npz.

    python tests/golden/make_trcadv.py --ref <pyNICAM-DC checkout> --out tests/golden
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

GL, VL, ZTOP, DTL, GAMMA, NSTEPS = 3, 10, 12000.0, 1200.0, 7.68e17, 3


def run(ref: str, out_dir: str, case: str = "1-1"):
    import toml
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "tr")
        MG.prep(ref, case_dir, GL, VL, ZTOP, layer_type="EVEN")
        c = toml.loads(MG.model_toml(ref, GL, VL, DTL, GAMMA, NSTEPS))
        c["timeparam"]["integ_type"] = "TRCADV"
        c["grdparam"]["topo_io_mode"] = "NONE"
        c["runconfparam"].update(CHEM_TYPE="PASSIVE", DCTEST_type="Traceradvection", DCTEST_case=case)
        c["dycoretestparam"].update(init_type="Traceradvection", test_case=case)
        c["chemvarparam"] = {"CHEM_TRC_vmax": 4}
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
        assert m.tim.TIME_integ_type == "TRCADV"
        pv, pvp = m.prgv.PRG_var, m.prgv.PRG_var_pl
        out = {"geo." + k: v for k, v in MG.geo_from_msc(m, pv.shape[-1] - 6).items()}
        g = m.grd
        K0 = m.adm.ADM_K0
        out["geo.GRD_LAT"] = np.ascontiguousarray(g.GRD_LAT[:, :, K0, :])
        out["geo.GRD_LON"] = np.ascontiguousarray(g.GRD_LON[:, :, K0, :])
        out["geo.GRD_LAT_pl"] = np.ascontiguousarray(g.GRD_LAT_pl[:, K0, :])
        out["geo.GRD_LON_pl"] = np.ascontiguousarray(g.GRD_LON_pl[:, K0, :])
        out["geo.GRD_Z"] = np.ascontiguousarray(g.GRD_vz[:, :, :, :, g.GRD_Z])
        out["geo.GRD_ZH"] = np.ascontiguousarray(g.GRD_vz[:, :, :, :, g.GRD_ZH])
        out["geo.GRD_Z_pl"] = np.ascontiguousarray(g.GRD_vz_pl[:, :, :, g.GRD_Z])
        out["geo.GRD_ZH_pl"] = np.ascontiguousarray(g.GRD_vz_pl[:, :, :, g.GRD_ZH])
        out["geo.integ_type"] = np.array("TRCADV")
        if case != "1-1":
            out["geo.trcadv_case"] = np.array(case)
        out["state0"], out["state0_pl"] = pv.copy(), pvp.copy()
        for s in range(NSTEPS):
            nic.run(1)
            out[f"state{s + 1}"], out[f"state{s + 1}_pl"] = m.prgv.PRG_var.copy(), m.prgv.PRG_var_pl.copy()
    path = os.path.join(out_dir, "gl03_z10_trcadv.npz" if case == "1-1" else "gl03_z10_trcadv12.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--case", default="1-1", choices=["1-1", "1-2"],
                    help="DCMIP2012 test: 1-1 deformational flow, 1-2 Hadley-like circulation")
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out), args.case)

"""Generate the restart (fio, input/output_io_mode "ADVANCED") fixture by
running the reference itself.

The gl03 z10 case of make_golden.py (the run of gl03_z10_trc.npz), one large
step, then the reference's own restart writer and reader
(nhm/share/mod_prgvar.py restart_output / restart_input with the prognostic
read, nhm/share/mod_fio.py, share/mod_comm.py COMM_var):

  * ``write``: the file restart_output writes for the state after step 1
    (header, the six prognostics and rhog<tracer>, big-endian float64);
  * ``read``: a file of the same state whose dummy levels hold a few
    non-finite values (as NICAM leaves its top dummy level), then the state
    restart_input makes of it: fio_read's dummy-level repair, the
    p2r-reverse pole-centre fill and the halo exchange of COMM_var.  The pole
    state is preset to NaN before the read, so every pole value comes from the
    read.

Stores both files (gzip), the state read back, and the metadata the writer
takes from the run (variable names, labels, units, layer name, region ids,
grid levels, the pole-centre source cells).

    python tests/golden/make_restart.py --ref <pyNICAM-DC checkout> --out tests/golden
"""
from __future__ import annotations

import argparse
import gzip
import os
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_golden as MG  # noqa: E402

GL, VL, ZTOP, DTL, GAMMA = 3, 10, 30000.0, 1200.0, 7.68e17
CTIME = 1200


def run(ref: str, out_dir: str):
    import toml
    trc = np.load(os.path.join(out_dir, "gl03_z10_trc.npz"))
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "rs")
        MG.prep(ref, case_dir, GL, VL, ZTOP)
        c = toml.loads(MG.model_toml(ref, GL, VL, DTL, GAMMA, 1))
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
        nic.run(1)
        prgv, rcnf = m.prgv, m.rcnf
        assert np.array_equal(prgv.PRG_var, trc["state1"])
        assert np.array_equal(prgv.PRG_var_pl, trc["state1_pl"])
        prgv.output_io_mode, prgv.output_prognostics, prgv.output_diagnostics = "ADVANCED", True, False
        base_w = os.path.join(tmp, "write.pe")
        prgv.restart_output(base_w, rcnf, np.float64, ctime=CTIME)
        with open(base_w + "000000", "rb") as f:
            write_bytes = f.read()
        # a file of the same state with non-finite dummy-level values
        keep = prgv.PRG_var.copy()
        prgv.PRG_var[1, 2, kk - 1, 3, 1] = np.nan
        prgv.PRG_var[:, :, kk - 1, 7, 5] = np.inf
        prgv.PRG_var[4, 4, 0, 12, 0] = np.nan
        base_r = os.path.join(tmp, "read.pe")
        prgv.restart_output(base_r, rcnf, np.float64, ctime=CTIME)
        with open(base_r + "000000", "rb") as f:
            read_bytes = f.read()
        prgv.PRG_var[...] = keep
        # the reference's prognostic restart read of that file
        prgv.PRG_var[...] = 0.0
        prgv.PRG_var_pl[...] = np.nan
        prgv.input_io_mode, prgv.input_diagnostics = "ADVANCED", False
        prgv.restart_input_basename = base_r
        prgv.restart_input(m.intoml, m.comm, m.gtl, m.cnst, rcnf, m.grd, m.vmtr, m.cnvv, m.tdyn, m.idi,
                           np.float64)
        read_state, read_state_pl = prgv.PRG_var.copy(), prgv.PRG_var_pl.copy()
        assert np.all(np.isfinite(read_state)) and np.all(np.isfinite(read_state_pl))

        adm, co = m.adm, m.comm
        items = prgv._restart_output_items(rcnf)
        names = [it[0] for it in items]
        assert [it[4] for it in items] == list(range(len(items)))
        # pole-centre sources of COMM_var's p2r-reverse copy (mod_comm.py:2249-2262)
        src = []
        cl = co.Copy_list_p2r
        for ipos in range(int(co.Copy_info_p2r[co.I_size])):
            l_from = int(cl[co.I_l_to, ipos])
            r_from = adm.RGNMNG_lp2r[l_from, co.Copy_info_p2r[co.I_prc_to]]
            if r_from == adm.RGNMNG_rgn4pl[adm.I_NPL] or r_from == adm.RGNMNG_rgn4pl[adm.I_SPL]:
                src.append([int(cl[co.I_gridi_from, ipos]), int(cl[co.I_l_from, ipos]),
                            int(cl[co.I_gridi_to, ipos]), int(cl[co.I_gridj_to, ipos]), l_from])
        out = {
            "write_file_gz": np.frombuffer(gzip.compress(write_bytes, 9), np.uint8),
            "read_file_gz": np.frombuffer(gzip.compress(read_bytes, 9), np.uint8),
            "read_state": read_state, "read_state_pl": read_state_pl,
            "names": np.array(names), "labels": np.array([it[1] for it in items]),
            "units": np.array([it[2] for it in items]), "layername": np.array(prgv.layername),
            "rgnid": np.array([int(adm.RGNMNG_lp2r[l, adm.ADM_prc_me]) for l in range(adm.ADM_lall)]),
            "glevel": np.array(adm.ADM_glevel), "rlevel": np.array(adm.ADM_rlevel), "ctime": np.array(CTIME),
            # rows: pole g, pole l, regional i, j, l (the pole centre takes the regional cell's value)
            "pole_src": np.array(src, np.int64),
        }
    path = os.path.join(out_dir, "gl03_z10_restart.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "pole sources", src)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    run(os.path.abspath(args.ref), os.path.abspath(args.out))

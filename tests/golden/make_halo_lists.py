"""Write halo_rl01.npz: the reference's single-rank halo copy lists for the
40-region (rlevel 1) icosahedral layout at grid levels 3..8.

The lists are the region/pole/singular-point copy tables that
``Comm.COMM_setup`` (share/mod_comm.py:177-1064, 1400-1561) derives from the
region topology; they are the index maps the device halo exchange must
reproduce exactly.  Run once, next to a reference checkout, with an rl01
single-process mnginfo file written by the reference's prep/mnginfo tool:

    python tests/golden/make_halo_lists.py <reference root> <rl01 mnginfo toml>

It writes pynicam-dc_b200/data/halo_rl01.npz.  Only this generator reads the
reference; the package reads the .npz.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

LEVELS = (3, 4, 5, 6, 7, 8)

_CHILD = r'''
import sys, numpy as np, toml
ref, mng, gl, out = sys.argv[1], sys.argv[2], int(sys.argv[3]), sys.argv[4]
sys.path.insert(0, ref)
from pynicamdc.share import comm_mode
comm_mode.set_mode("serial")
from pynicamdc.share.mod_backend import backend as bk
bk.configure("numpy", "float64")
tml = out + ".toml"
cfg = {"admparam": {"glevel": gl, "rlevel": 1, "vlayer": 1, "rgnmngfname": tml, "ADM_HGRID_SYSTEM": "ICO",
                    "debug": False},
       "rgnmngparam": {"RGNMNG_in_fname": mng, "RGNMNG_out_fname": "tempout"},
       "commparam": {"COMM_apply_barrier": False, "COMM_varmax": 15, "debug": False, "testonly": False},
       "param_io": {"h_source": "", "h_institute": "", "io_log_basename": "msg", "io_log_suppress": True,
                    "io_log_allnode": False, "io_log_nml_suppress": True, "io_aggregate": False},
       "cnstparam": {}, "param_prof": {"prof_mpi_barrier": False, "prof_rap_level": 0}}
toml.dump(cfg, open(tml, "w"))
from pynicamdc.share.mod_process import prc
from pynicamdc.share.mod_stdio import std
from pynicamdc.share.mod_prof import prf
from pynicamdc.share.mod_adm import adm
from pynicamdc.share.mod_const import Const
from pynicamdc.share.mod_comm import Comm
c = Const(np.float64); co = Comm()
prc.prc_mpistart(); std.io_setup("pyNICAM-DC", tml); std.io_log_setup(prc.prc_myrank, True)
prf.PROF_setup(tml, np.float64); c.CONST_setup(np.float64, tml); adm.ADM_setup(tml); co.COMM_setup(tml)
n = lambda info: int(info[co.I_size])
np.savez(out, r2r=co.Copy_list_r2r[:, :n(co.Copy_info_r2r)], p2r=co.Copy_list_p2r[:, :n(co.Copy_info_p2r)],
         r2p=co.Copy_list_r2p[:, :n(co.Copy_info_r2p)], sgp=co.Singular_list[:, :n(co.Singular_info)],
         have_sgp=np.asarray(adm.ADM_have_sgp))
'''


def main(ref_root: str, mnginfo: str):
    out = {}
    with tempfile.TemporaryDirectory() as td:
        child = os.path.join(td, "child.py")
        with open(child, "w") as f:
            f.write(_CHILD)
        for gl in LEVELS:
            f = os.path.join(td, f"gl{gl}.npz")
            subprocess.run([sys.executable, child, ref_root, os.path.abspath(mnginfo), str(gl), f], check=True,
                           cwd=td, stdout=subprocess.DEVNULL)
            z = np.load(f)
            for k in ("r2r", "p2r", "r2p", "sgp"):
                out[f"gl{gl:02d}_{k}"] = z[k].astype(np.int16)
            out["have_sgp"] = z["have_sgp"].astype(np.bool_)
    here = os.path.dirname(os.path.abspath(__file__))
    dst = os.path.join(here, "..", "..", "pynicam-dc_b200", "data", "halo_rl01.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst))


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])

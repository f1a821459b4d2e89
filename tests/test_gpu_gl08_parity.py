"""Parity at the benchmarked configuration: gl08 z40 (655,362 cells, 40
regions of 128x128), the case bench.py times, built by the same grid generator
and spring relaxation.  One large float64 step on the device and one oracle
step on the host from the same state: relative L2 per prognostic (bound
1e-12, the north star's one-step tolerance) and bit-for-bit equality, plus the
mass sums against the host's (relative; absolute for the JW tracer, whose
mass is zero).  Measured on B200: bit for bit, every prognostic and the
poles; the oracle step took 854 s.

Opt-in (NC_GL08_PARITY=1): the oracle step runs about a quarter of an hour on
one host core and holds tens of GB of host memory.  With NC_REPORT_DIR set
the result is written to gl08_parity.json there.
"""
import json
import os

import numpy as np
import pytest

from test_gpu_gl07 import _rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("NC_GL08_PARITY") != "1",
                                 reason="opt-in: NC_GL08_PARITY=1 (oracle step of ~15 min)")]


def test_gl08_step_matches_oracle(pkg):
    import time
    import bench
    from oracle import nicam_step as O
    geo, prg, prg_pl, _ = bench.make_case(8, 40, device="cuda")
    core = pkg.NicamCuda(geo, graph=True)
    try:
        core.upload(prg, prg_pl)
        core.step(1)
        out, out_pl = core.download()
        mass = core.mass_sums()
    finally:
        core.close()
    t = time.perf_counter()
    want, want_pl = O.dynamics_step(O.Geo(geo), prg, prg_pl)
    oracle_s = time.perf_counter() - t
    err, err_pl = _rel_l2(out, want), _rel_l2(out_pl, want_pl)
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    ks = slice(kmin, kmax + 1)
    w = geo["VMTR_VOLUME"][1:-1, 1:-1, ks] / geo["VMTR_GSGAM2"][1:-1, 1:-1, ks]
    w_pl = geo["VMTR_VOLUME_pl"][0, ks] / geo["VMTR_GSGAM2_pl"][0, ks]
    host = [float(np.sum(want[1:-1, 1:-1, ks, :, v] * w) + np.sum(want_pl[0, ks, :, v] * w_pl)) for v in (0, 6)]
    rep = {"grid": "gl08 z40", "rel_l2": err, "rel_l2_pole": err_pl,
           "bit_exact": bool(np.array_equal(out, want) and np.array_equal(out_pl, want_pl)),
           "differing_values": int(np.count_nonzero(out != want) + np.count_nonzero(out_pl != want_pl)),
           "mass_diff_vs_oracle": [abs(m - h) / abs(h) if h != 0 else abs(m) for m, h in zip(mass[:2], host)],
           "oracle_step_s": oracle_s}
    print("gl08 parity:", rep)
    out_dir = os.environ.get("NC_REPORT_DIR")
    if out_dir:
        with open(os.path.join(out_dir, "gl08_parity.json"), "w") as fh:
            json.dump(rep, fh, indent=1)
    assert max(err.values()) <= 1e-12 and max(err_pl.values()) <= 1e-12, (err, err_pl)
    assert rep["bit_exact"], rep["differing_values"]
    assert max(rep["mass_diff_vs_oracle"]) <= 1e-12

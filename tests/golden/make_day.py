"""One simulated day at gl05 z40: the oracle's digest, and the oracle pinned
to the reference over the same day.

The case: grid level 5 (40 regions of 16x16 + halo), 40 ULLRICH14 layers to
30 km, dtl = 600 s, 144 large steps (one day), gamma_h = alpha_d = 1.2e16,
the JW balanced jet + perturbation with the sharp analytic tracer of
make_golden.tracer_field in the first tracer slot.

Modes (all CPU):

  digest   builds the case with the package's own grid generator (host
           arithmetic at this level, so the identical case is rebuilt by the
           GPU test), runs the oracle for 144 steps and writes
           ``gl05_z40_day.npz``: hashes of the setup and the initial state,
           and after steps 1, 36 (6 h) and 144 (1 day) the state's SHA-256,
           per-prognostic interior sums of squares, a strided sample of the
           regional state (i, j in {2, 9, 16}, every level and region), the
           full pole state, and the host mass sums of every step.
  ref      runs the reference itself (numpy backend, serial, I/O stubbed) on
           its own generated gl05 grid for 144 steps; saves its setup, the
           initial state and the states after steps 1, 36 and 144 under
           --work.
  oracle   runs the oracle from the reference's saved setup and initial state
           (waits for ``ref`` to write them) and saves the same states.
  compare  compares the two runs and writes ``gl05_z40_day_pin.json``.

    python tests/golden/make_day.py --mode digest
    python tests/golden/make_day.py --mode ref --ref <pyNICAM-DC checkout> --work <scratch dir> &
    python tests/golden/make_day.py --mode oracle --ref <pyNICAM-DC checkout> --work <scratch dir>
    python tests/golden/make_day.py --mode compare --ref <pyNICAM-DC checkout> --work <scratch dir>
"""
from __future__ import annotations

import argparse
import hashlib
import importlib
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

GL, VL, ZTOP, DTL, GAMMA, NSTEPS = 5, 40, 30000.0, 600.0, 1.2e16, 144
RECORD = (1, 36, 144)
SAMPLE_IJ = (2, 9, 16)


def state_sha(s, s_pl) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(s).tobytes())
    h.update(np.ascontiguousarray(s_pl).tobytes())
    return h.hexdigest()


def geo_sha(geo: dict) -> str:
    """hash of the setup arrays (the surface-pressure diagnostic's heights,
    keys sfc_*, are not part of the setup the step reads; NQW_END = 0, the
    vapour as the only water tracer, is the default the step assumes without
    the key)"""
    h = hashlib.sha256()
    default = lambda k: k == "NQW_END" and int(np.asarray(geo[k])) == 0
    for k in sorted(k for k in geo if not k.startswith("sfc_") and not default(k)):
        h.update(k.encode())
        h.update(np.ascontiguousarray(np.asarray(geo[k])).tobytes())
    return h.hexdigest()


def sample(s):
    return s[np.ix_(SAMPLE_IJ, SAMPLE_IJ)].copy()


def interior_sumsq(s, kmin, kmax):
    """per-prognostic sum of squares over interior cells and levels"""
    v = s[1:-1, 1:-1, kmin:kmax + 1]
    return np.einsum("ijklv,ijklv->v", v, v)


def mass_host(geo, s, s_pl):
    """sum(rhog / GSGAM2 * VMTR_VOLUME) and the same of rhogq over interior
    cells, levels kmin..kmax, plus the two pole points (the volume-weighted
    sums of mod_embudget.py:74-80 with the poles included)"""
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    sl = (slice(1, -1), slice(1, -1), slice(kmin, kmax + 1))
    vol = geo["VMTR_VOLUME"][sl] / geo["VMTR_GSGAM2"][sl]
    vol_pl = geo["VMTR_VOLUME_pl"][0, kmin:kmax + 1] / geo["VMTR_GSGAM2_pl"][0, kmin:kmax + 1]
    out = []
    for v in [0] + list(range(6, s.shape[-1])):
        r = np.sum(s[sl + (slice(None), v)] * vol)
        p = np.sum(s_pl[0, kmin:kmax + 1, :, v] * vol_pl)
        out.append(r + p)
    return np.array(out)


def build_case():
    """the gl05 z40 one-day case from the package's grid generator"""
    from make_golden import tracer_field
    ig = importlib.import_module("pynicam-dc_b200.icogrid")
    g = ig.Grid(GL, vlayer=VL, ztop=ZTOP, device="cpu")
    geo = g.setup(dtl=DTL, gamma=GAMMA, nq=1)
    s, s_pl = g.jw_state(nq=1)
    lat = np.moveaxis(g.lat, 0, 2)
    lon = np.moveaxis(g.lon, 0, 2)
    lat_p, lon_p = ig._latlon(g.x_pl)
    lat_p, lon_p = np.moveaxis(lat_p, 0, 1), np.moveaxis(lon_p, 0, 1)
    kk = s.shape[2]
    s[..., 6] = s[..., 0] * np.moveaxis(tracer_field(lat, lon, kk), -1, 2)
    s_pl[..., 6] = s_pl[..., 0] * np.moveaxis(tracer_field(lat_p, lon_p, kk), -1, 1)
    s[:, :, 0, :, 6] = 0.0
    s[:, :, -1, :, 6] = 0.0
    s_pl[:, 0, :, 6] = 0.0
    s_pl[:, -1, :, 6] = 0.0
    return geo, s, s_pl


def mode_digest(out_path: str):
    from oracle import nicam_step as O
    t0 = time.time()
    geo, s, s_pl = build_case()
    G = O.Geo(geo)
    O.comm(G, s, s_pl)
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    out = {"geo_sha": np.array(geo_sha(geo)), "init_sha": np.array(state_sha(s, s_pl)),
           "record": np.array(RECORD), "sample_ij": np.array(SAMPLE_IJ)}
    mass = [mass_host(geo, s, s_pl)]
    print(f"case built in {time.time() - t0:.0f} s", flush=True)
    for n in range(1, NSTEPS + 1):
        s, s_pl = O.dynamics_step(G, s, s_pl)
        mass.append(mass_host(geo, s, s_pl))
        if n in RECORD:
            out[f"s{n}_sha"] = np.array(state_sha(s, s_pl))
            out[f"s{n}_sumsq"] = interior_sumsq(s, kmin, kmax)
            out[f"s{n}_sample"] = sample(s)
            out[f"s{n}_pl"] = s_pl.copy()
        if n % 12 == 0:
            print(f"step {n} {time.time() - t0:.0f} s", flush=True)
    out["mass"] = np.array(mass)
    np.savez_compressed(out_path, **out)
    print("wrote", out_path, os.path.getsize(out_path))


def mode_ref(ref: str, work: str):
    import make_golden as MG
    os.makedirs(work, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        case_dir = os.path.join(tmp, "day")
        MG.prep(ref, case_dir, GL, VL, ZTOP)
        with open(os.path.join(case_dir, "case", "config", "nhm_jw.toml"), "w") as f:
            f.write(MG.model_toml(ref, GL, VL, DTL, GAMMA, NSTEPS))
        with open(os.path.join(case_dir, "drv.toml"), "w") as f:
            f.write('[driver]\nbackend="numpy"\nprecision="float64"\ncomm="serial"\n'
                    'nhm_driver_cnf="./case/config/nhm_jw.toml"\n')
        os.chdir(case_dir)
        import types
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
        geo = {"geo." + k: v for k, v in MG.geo_from_msc(m, pv.shape[-1] - 6).items()}
        tmpf = os.path.join(work, "ref_setup.tmp.npz")
        np.savez(tmpf, **geo, state0=pv.copy(), state0_pl=pvp.copy())
        os.replace(tmpf, os.path.join(work, "ref_setup.npz"))
        t0 = time.time()
        for n in range(1, NSTEPS + 1):
            nic.run(1)
            if n in RECORD:
                np.savez(os.path.join(work, f"ref_s{n}.npz"), s=m.prgv.PRG_var, s_pl=m.prgv.PRG_var_pl)
            if n % 12 == 0:
                print(f"ref step {n} {time.time() - t0:.0f} s", flush=True)


def mode_oracle(work: str):
    from oracle import nicam_step as O
    from make_golden import load
    path = os.path.join(work, "ref_setup.npz")
    while not os.path.exists(path):
        time.sleep(10)
    geo, st = load(path)
    G = O.Geo(geo)
    s, s_pl = st["state0"], st["state0_pl"]
    t0 = time.time()
    for n in range(1, NSTEPS + 1):
        s, s_pl = O.dynamics_step(G, s, s_pl)
        if n in RECORD:
            np.savez(os.path.join(work, f"oracle_s{n}.npz"), s=s, s_pl=s_pl)
        if n % 12 == 0:
            print(f"oracle step {n} {time.time() - t0:.0f} s", flush=True)


def mode_compare(work: str, out_path: str):
    names = ["RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE", "RHOGQ1"]
    res = {"case": f"gl{GL:02d} z{VL} JW + sharp tracer, dtl {DTL} s, {NSTEPS} steps", "steps": {}}
    for n in RECORD:
        a = np.load(os.path.join(work, f"ref_s{n}.npz"))
        b = np.load(os.path.join(work, f"oracle_s{n}.npz"))
        d = {"bit_exact": bool(np.array_equal(a["s"], b["s"]) and np.array_equal(a["s_pl"], b["s_pl"]))}
        for v, nm in enumerate(names):
            x, y = a["s"][..., v], b["s"][..., v]
            den = float(np.sqrt(np.sum(x * x)))
            d[nm] = float(np.sqrt(np.sum((x - y) ** 2))) / den if den > 0 else 0.0
        res["steps"][str(n)] = d
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=("digest", "ref", "oracle", "compare"), default="digest")
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--work", default=os.path.join(tempfile.gettempdir(), "nicam_day"))
    args = ap.parse_args()
    if args.mode == "digest":
        mode_digest(os.path.join(HERE, "gl05_z40_day.npz"))
    elif args.mode == "ref":
        mode_ref(os.path.abspath(args.ref), os.path.abspath(args.work))
    elif args.mode == "oracle":
        mode_oracle(os.path.abspath(args.work))
    else:
        mode_compare(os.path.abspath(args.work), os.path.join(HERE, "gl05_z40_day_pin.json"))

"""Generate the golden fixtures by running the reference itself (CPU, numpy).

Run in a container where the reference tree is available (it is read-only and
is copied nowhere; the prep tools write into a scratch case directory):

    python tests/golden/make_golden.py --ref <pyNICAM-DC checkout> --out tests/golden

For each case this script
  1. builds the region table, the icosahedral grid (recursive division +
     spring dynamics + gravity centring) and a ULLRICH14 stretched vertical
     grid with the reference's own prep tools (prep/mnginfo/mkmnginfo.py,
     prep/hgrid/mkrawgrid.py --comm serial, prep/vgrid/mkvlayer.py);
  2. initialises pyNICAM (numpy backend, serial comm, I/O stubbed) with the
     Jablonowski-Williamson balanced jet + perturbation (init_type
     'Jablonowski', test_case '1'), RK3, DIRECT lap_order-2 hyperdiffusion and
     divergence damping, Thuburn limiters on;
  3. optionally replaces the (zero) water-vapour tracer by a seeded field with
     sharp cosine bells so that the MIURA2004 advection and both Thuburn
     limiters act on non-trivial data;
  4. runs NSTEPS large steps and stores the setup arrays (under the
     reference's attribute names) together with state0..stateN.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile
import types

import numpy as np

CASES = {
    # name: glevel, vlayer, ztop [m], dtl [s], gamma_h = alpha_d, nsteps, tracer
    "gl03_z10_trc": (3, 10, 30000.0, 1200.0, 7.68e17, 2, True),
    # RAIN_TYPE WARM: three water tracers (vapour, cloud, rain) in the
    # thermodynamics of the step (cv and qd over the water range)
    "gl03_z10_warm": (3, 10, 30000.0, 1200.0, 7.68e17, 2, True),
}
RAIN = {"gl03_z10_warm": "WARM"}
# numfilter options beyond DIRECT hyperdiffusion: NONLINEAR1 (the temperature-
# Laplacian-dependent Kh, mod_numfilter.py:1153-1207, as in the DCMIP2016
# tutorial cases) and the Rayleigh sponge (mod_numfilter.py:219-271, as in the
# mountain-wave cases), scaled to gl03 / dtl 1200 s
CASES["gl03_z10_nlhdiff"] = CASES["gl03_z10_trc"]
CASES["gl03_z10_rayleigh"] = CASES["gl03_z10_trc"]
NUMF = {"gl03_z10_nlhdiff": dict(hdiff_type="NONLINEAR1", Kh_coef_maxlim=7.68e18, Kh_coef_minlim=7.68e17,
                                 ZD_hdiff_nl=20000.0),
        "gl03_z10_rayleigh": dict(alpha_r=2.0e-4, ZD=15000.0)}
WATER_SCALE = (1.0, 0.05, 0.02)   # vapour, cloud, rain: multiples of the tracer field

MKRAWGRID_TOML = """[admparam]
glevel  = {gl}
rlevel  = 1
vlayer  = 1
rgnmngfname = '../../case/config/mkrawgrid.toml'
ADM_HGRID_SYSTEM = 'ICO'
debug = false
[param_mkgrd]
mkgrd_dospring    = true
mkgrd_doprerotate = false
mkgrd_dostretch   = false
mkgrd_doshrink    = false
mkgrd_dorotate    = false
mkgrd_in_basename = ''
mkgrd_in_io_mode  = ''
mkgrd_out_basename = 'rawgrid'
mkgrd_out_io_mode  = 'ADVANCED'
mkgrd_spring_beta      =  1.15
mkgrd_prerotation_tilt =  0.0
mkgrd_stretch_alpha    =  1.00
mkgrd_shrink_level     =  0.0
mkgrd_rotation_lon     =  0.0
mkgrd_rotation_lat     = 90.0
mkgrd_precision_single = false
[param_io]
h_source = 'src path'
h_institute = 'pyNICAM-DC team'
io_log_basename = 'msg'
io_log_suppress = false
io_log_allnode = true
io_log_nml_suppress = false
io_aggregate = false
[commparam]
COMM_apply_barrier= false
COMM_varmax = 15
debug = false
testonly = false
[cnstparam]
[param_prof]
prof_mpi_barrier = true
prof_rap_level = 10
[rgnmngparam]
RGNMNG_in_fname='../../case/prepdata/rl01-prc000001.toml'
RGNMNG_out_fname='tempout'
"""


def prep(ref: str, case_dir: str, gl: int, vl: int, ztop: float, layer_type: str = "ULLRICH14"):
    os.makedirs(os.path.join(case_dir, "case", "config"), exist_ok=True)
    os.makedirs(os.path.join(case_dir, "case", "prepdata"), exist_ok=True)
    work = os.path.join(case_dir, "a", "b")
    os.makedirs(work, exist_ok=True)
    cfg = os.path.join(case_dir, "case", "config")
    with open(os.path.join(cfg, "mkmnginfo.toml"), "w") as f:
        f.write("[mkmnginfo]\nrlevel = 1\nprc_num = 1\noutput_fname = '../../case/prepdata/rl01-prc000001.toml'\n")
    with open(os.path.join(cfg, "mkrawgrid.toml"), "w") as f:
        f.write(MKRAWGRID_TOML.format(gl=gl))
    with open(os.path.join(cfg, "mkvlayer.toml"), "w") as f:
        f.write(f"[mkvlayer]\nnum_of_layer = {vl}\nlayer_type = '{layer_type}'\nztop = {ztop}\n"
                "outfname = '../../case/prepdata/vgrid.json'\n")
    P = os.path.join(ref, "pynicamdc", "prep")
    run = lambda *a: subprocess.run([sys.executable, *a], cwd=work, check=True, capture_output=True)
    run(os.path.join(P, "mnginfo", "mkmnginfo.py"), "--config", "../../case/config/mkmnginfo.toml")
    run(os.path.join(P, "vgrid", "mkvlayer.py"), "--config", "../../case/config/mkvlayer.toml")
    run(os.path.join(P, "hgrid", "mkrawgrid.py"), "--config", "../../case/config/mkrawgrid.toml", "--comm", "serial")


NHM_TOML = os.path.join("tutorial", "case", "config", "nhm_jw.toml")


def model_toml(ref: str, gl: int, vl: int, dtl: float, gamma: float, nsteps: int, rain: str = "",
               numf: dict = None) -> str:
    """the reference's JW tutorial config, pointed at the scratch case"""
    import toml
    c = toml.load(os.path.join(ref, NHM_TOML))
    c["admparam"].update(glevel=gl, rlevel=1, vlayer=vl, rgnmngfname="./case/config/nhm_jw.toml")
    c["rgnmngparam"]["RGNMNG_in_fname"] = "./case/prepdata/rl01-prc000001.toml"
    c["grdparam"].update(hgrid_io_mode="npz", hgrid_fname="./case/prepdata/rawgrid.pe",
                         vgrid_fname="./case/prepdata/vgrid.json", topo_io_mode="IDEAL")
    c["timeparam"].update(integ_type="RK3", dtl=dtl, lstep_max=max(nsteps, 1))
    c["numfilterparam"].update(hdiff_type="DIRECT", lap_order_hdiff=2, gamma_h=gamma, divdamp_type="DIRECT",
                               lap_order_divdamp=2, alpha_d=gamma)
    if numf:
        c["numfilterparam"].update(numf)
    c["restartparam"]["input_io_mode"] = "IDEAL"
    c["dycoretestparam"].update(init_type="Jablonowski", test_case="1")
    c["runconfparam"]["THUBURN_LIM"] = True
    if rain:
        c["runconfparam"]["RAIN_TYPE"] = rain
    c.setdefault("embudgetparam", {})["MNT_ON"] = False
    c["ioparam"]["PRGout_interval"] = 10 ** 9
    return toml.dumps(c)


def tracer_field(lat, lon, kk):
    """seeded-free analytic tracer: two cosine bells with sharp edges and a band"""
    q = np.zeros(lat.shape + (kk,))
    for (c0, c1, R, a) in ((0.6, 1.0, 0.5, 4e-3), (-0.3, 3.5, 0.7, 2e-3)):
        r = np.arccos(np.clip(np.sin(c0) * np.sin(lat) + np.cos(c0) * np.cos(lat) * np.cos(lon - c1), -1, 1))
        bell = np.where(r < R, 0.5 * (1 + np.cos(np.pi * r / R)), 0.0)
        q += (a * bell)[..., None] * np.linspace(1.0, 0.2, kk)
    q += np.where(np.abs(lat - 0.2) < 0.15, 1e-3, 0.0)[..., None]
    return q + 1e-5


def geo_from_msc(m, nq: int) -> dict:
    """the reference's setup objects -> the flat setup dict used by the oracle
    and the CUDA backend"""
    g = {}
    a = m.adm
    g.update(kall=a.ADM_kall, kmin=a.ADM_kmin, kmax=a.ADM_kmax, gall_1d=a.ADM_gall_1d, gmin=a.ADM_gmin,
             gmax=a.ADM_gmax, lall=a.ADM_lall, have_sgp=np.asarray(a.ADM_have_sgp), nq=nq)
    g["pntmask"] = np.asarray(m.ppm.pntmask)
    c = m.cnst
    g.update(GRAV=c.CONST_GRAV, Rdry=c.CONST_Rdry, CVdry=c.CONST_CVdry, CPdry=c.CONST_CPdry, Rvap=c.CONST_Rvap,
             OHM=c.CONST_OHM, RADIUS=c.CONST_RADIUS, EPS=c.CONST_EPS, HUGE=c.CONST_HUGE, PRE00=c.CONST_PRE00)
    nf = m.numf
    g.update(rscale=m.grd.GRD_rscale, alpha=float(m.rcnf.NON_HYDRO_ALPHA), dtl=m.tim.TIME_dtl,
             dts=m.tim.TIME_dts, hdiff_fact_rho=nf.hdiff_fact_rho, Kh_coef=float(nf.gamma_h),
             divdamp_coef=float(nf.alpha_d))
    if nf.hdiff_nonlinear:   # NONLINEAR1: per-level upper bound, lower bound, mean cell area
        fact = np.zeros(a.ADM_kall)
        nf.height_factor(a.ADM_kall, m.grd.GRD_gz, m.grd.GRD_htop, nf.ZD_hdiff_nl, fact, m.cnst, np.float64)
        g["hdiff_nl_kh_max"] = (1.0 - fact) * nf.Kh_coef_maxlim + fact * nf.Kh_coef_minlim
        g["hdiff_nl_minlim"] = float(nf.Kh_coef_minlim)
        g["hdiff_nl_area"] = float(nf.AREA_ave)
    else:
        assert np.all(nf.Kh_coef == float(nf.gamma_h))
    assert np.all(nf.divdamp_coef == float(nf.alpha_d))
    if nf.NUMFILTER_DOrayleigh:   # the sponge coefficients per full and half level
        g["rayleigh_coef"] = np.asarray(nf.rayleigh_coef)
        g["rayleigh_coef_h"] = np.asarray(nf.rayleigh_coef_h)
        g["rayleigh_only_w"] = int(bool(nf.rayleigh_damp_only_w))
    g["sstep"] = np.asarray(m.dyn.num_of_iteration_sstep[:m.dyn.num_of_iteration_lstep])
    g["CVW"] = np.asarray(m.rcnf.CVW)
    g["NQW_END"] = int(m.rcnf.NQW_END)   # water tracers 0..NQW_END (NQW_STR = I_QV = 0)
    co = m.comm
    g["copy_r2r"] = co.Copy_list_r2r[:, :int(co.Copy_info_r2r[co.I_size])].astype(np.int64)
    g["copy_p2r"] = co.Copy_list_p2r[:, :int(co.Copy_info_p2r[co.I_size])].astype(np.int64)
    g["copy_r2p"] = co.Copy_list_r2p[:, :int(co.Copy_info_r2p[co.I_size])].astype(np.int64)
    g["copy_sgp"] = co.Singular_list[:, :int(co.Singular_info[co.I_size])].astype(np.int64)
    for k, v in vars(m.vmtr).items():
        if k.startswith("VMTR_") and isinstance(v, np.ndarray):
            g[k] = v
    for k in ("GRD_x", "GRD_x_pl", "GRD_xr", "GRD_xr_pl", "GRD_afact", "GRD_bfact", "GRD_cfact", "GRD_dfact",
              "GRD_rdgz", "GRD_rdgzh", "GRD_gz", "GRD_gzh"):
        g[k] = getattr(m.grd, k)
    for k in ("OPRT_coef_div", "OPRT_coef_grad", "OPRT_coef_lap", "OPRT_coef_intp", "OPRT_coef_diff"):
        g[k] = getattr(m.oprt, k)
        g[k + "_pl"] = getattr(m.oprt, k + "_pl")
    for k in ("GMTR_t", "GMTR_a", "GMTR_p"):
        g[k] = getattr(m.gmtr, k)
        g[k + "_pl"] = getattr(m.gmtr, k + "_pl")
    for k in ("rho_bs", "pre_bs", "tem_bs"):
        g[k] = getattr(m.bsst, k)
        g[k + "_pl"] = getattr(m.bsst, k + "_pl")
    return {k: np.asarray(v) for k, v in g.items()}


def run_case(ref: str, name: str, out_dir: str, scratch: str):
    gl, vl, ztop, dtl, gamma, nsteps, tracer = CASES[name]
    case_dir = os.path.join(scratch, name)
    prep(ref, case_dir, gl, vl, ztop)
    with open(os.path.join(case_dir, "case", "config", "nhm_jw.toml"), "w") as f:
        f.write(model_toml(ref, gl, vl, dtl, gamma, nsteps, RAIN.get(name, ""), NUMF.get(name)))
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
    if tracer:
        kk = pv.shape[2]
        lat, lon = m.grd.GRD_LAT[:, :, 0, :], m.grd.GRD_LON[:, :, 0, :]
        latp, lonp = m.grd.GRD_LAT_pl[:, 0, :], m.grd.GRD_LON_pl[:, 0, :]
        nw = int(m.rcnf.NQW_END) + 1 if name in RAIN else 1
        for n in range(nw):
            sc = WATER_SCALE[n]
            pv[..., 6 + n] = pv[..., 0] * sc * np.moveaxis(tracer_field(lat, lon, kk), -1, 2)
            pvp[..., 6 + n] = pvp[..., 0] * sc * np.moveaxis(tracer_field(latp, lonp, kk), -1, 1)
            pv[:, :, 0, :, 6 + n] = 0.0
            pv[:, :, -1, :, 6 + n] = 0.0
            pvp[:, 0, :, 6 + n] = 0.0
            pvp[:, -1, :, 6 + n] = 0.0
    out = {"geo." + k: v for k, v in geo_from_msc(m, pv.shape[-1] - 6).items()}
    out["state0"], out["state0_pl"] = pv.copy(), pvp.copy()
    for s in range(nsteps):
        nic.run(1)
        out[f"state{s + 1}"], out[f"state{s + 1}_pl"] = m.prgv.PRG_var.copy(), m.prgv.PRG_var_pl.copy()
    path = os.path.join(out_dir, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


def load(path: str):
    """fixture -> (geo dict, states dict)"""
    d = np.load(path)
    geo = {k[4:]: d[k] for k in d.files if k.startswith("geo.")}
    st = {k: d[k] for k in d.files if k.startswith("state")}
    return geo, st


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of a pyNICAM-DC checkout")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--case", default="gl03_z10_trc")
    args = ap.parse_args()
    out = os.path.abspath(args.out)
    with tempfile.TemporaryDirectory() as tmp:
        run_case(os.path.abspath(args.ref), args.case, out, tmp)

"""ctypes binding of libnicamcuda.so and the device-resident dynamics object.

``NicamCuda`` owns one C-ABI handle: it turns a setup dict (the reference's
geometry/metric/operator arrays under their attribute names) into the
``nc_array`` table of ``nc_create``, and exposes the step, marshal and budget
calls.  The library is loaded from this package directory only; if it is
missing or cannot be loaded, construction raises -- there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import halo

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libnicamcuda.so"
LIB_PATH = os.path.join(_HERE, LIB_NAME)

NC_F64, NC_I32, NC_I64, NC_BOOL = 0, 1, 2, 3


class NcArray(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("data", ctypes.c_void_p), ("dtype", ctypes.c_int32),
                ("ndim", ctypes.c_int32), ("shape", ctypes.c_int64 * 8)]


_lib = None

# every entry point declared in include/nicam_cuda.h and include/nicam_cuda_debug.h
EXPORTS = ("nc_create", "nc_upload_state", "nc_download_state", "nc_download_state_async", "nc_join_copies",
           "nc_upload_state_device", "nc_download_state_device", "nc_check_finite", "nc_set_block", "nc_get_block",
           "nc_step", "nc_set_graph", "nc_run_phases", "nc_sync", "nc_mass_sums", "nc_get_field", "nc_state_pointers", "nc_kernel_launches", "nc_stream", "nc_profile",
           "nc_kernel_stats", "nc_grid_spring", "nc_mass_sum_noalloc", "nc_forcing_step", "nc_history_vars", "nc_restart_pack",
           "nc_restart_unpack", "nc_restart_finish", "nc_divide_known", "nc_vsolve", "nc_vadv_lin", "nc_laplacian",
           "nc_trc_step_lin", "nc_set_time", "nc_trc_prepare", "nc_divergence", "nc_gradient", "nc_diffusion", "nc_divdamp3d", "nc_divdamp2d", "nc_exchange", "nc_diffusion_kh", "nc_forcing_precip", "nc_last_error", "nc_destroy")


def load_library(path: str = LIB_PATH):
    """Load (once) and type the C ABI.  Raises OSError if the library is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{LIB_NAME} not built: run __graft_entry__.build() (expected at {path})")
    lib = ctypes.CDLL(path)
    vp, i32, i64, dp = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p
    lib.nc_create.argtypes = [ctypes.POINTER(NcArray), i32, ctypes.POINTER(vp)]
    lib.nc_upload_state.argtypes = [vp, dp, dp]
    lib.nc_download_state.argtypes = [vp, dp, dp]
    lib.nc_download_state_async.argtypes = [vp, dp, dp]
    lib.nc_join_copies.argtypes = [vp]
    lib.nc_upload_state_device.argtypes = [vp, dp, dp, vp]
    lib.nc_download_state_device.argtypes = [vp, dp, dp, vp]
    lib.nc_check_finite.argtypes = [vp]
    lib.nc_set_block.argtypes = [vp, ctypes.c_char_p, i32]
    lib.nc_get_block.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(i32)]
    lib.nc_step.argtypes = [vp, i32]
    lib.nc_set_graph.argtypes = [vp, i32]
    lib.nc_run_phases.argtypes = [vp, i32]
    lib.nc_sync.argtypes = [vp]
    lib.nc_mass_sums.argtypes = [vp, dp, i32]
    lib.nc_get_field.argtypes = [vp, ctypes.c_char_p, dp, dp]
    lib.nc_state_pointers.argtypes = [vp, i32, ctypes.POINTER(vp), ctypes.POINTER(vp)]
    lib.nc_kernel_launches.argtypes = [vp]
    lib.nc_kernel_launches.restype = i64
    lib.nc_last_error.restype = ctypes.c_char_p
    lib.nc_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.nc_profile.argtypes = [vp, i32]
    lib.nc_kernel_stats.argtypes = [vp, i32, ctypes.c_char_p, dp, dp]
    lib.nc_kernel_stats.restype = ctypes.c_int
    lib.nc_mass_sum_noalloc.argtypes = [dp] * 8 + [i32] * 5 + [dp, vp]
    lib.nc_mass_sum_noalloc.restype = ctypes.c_int
    lib.nc_grid_spring.argtypes = [i32, i32, dp, dp, dp, dp, dp, i32, dp, dp, i32, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, i64, ctypes.POINTER(i64)]
    lib.nc_grid_spring.restype = ctypes.c_int
    lib.nc_forcing_step.argtypes = [vp]
    lib.nc_forcing_step.restype = ctypes.c_int
    lib.nc_divide_known.argtypes = [dp, dp, dp, i64, ctypes.c_double]
    lib.nc_history_vars.argtypes = [vp, dp, i32, i64, ctypes.c_double, dp]
    lib.nc_history_vars.restype = ctypes.c_int
    for f in ("nc_restart_pack", "nc_restart_unpack"):
        getattr(lib, f).argtypes = [vp, i32, vp]
        getattr(lib, f).restype = ctypes.c_int
    lib.nc_restart_finish.argtypes = [vp, dp, i32]
    lib.nc_restart_finish.restype = ctypes.c_int
    lib.nc_divide_known.restype = ctypes.c_int
    lib.nc_vsolve.argtypes = [vp, i32, i32] + [dp] * 9 + [vp]
    lib.nc_vadv_lin.argtypes = [vp, i32, i32] + [dp] * 6 + [ctypes.c_double, ctypes.c_double, i32, vp]
    lib.nc_laplacian.argtypes = [vp, i32, dp, dp, dp, dp, vp]
    lib.nc_trc_step_lin.argtypes = [vp, i32] + [dp] * 6 + [vp]
    lib.nc_set_time.argtypes = [vp, ctypes.c_double]
    lib.nc_trc_prepare.argtypes = [vp]
    lib.nc_divergence.argtypes = [vp, i32, dp, dp, dp, dp, vp]
    lib.nc_forcing_precip.argtypes = [vp, dp]
    lib.nc_forcing_precip.restype = ctypes.c_int
    lib.nc_gradient.argtypes = [vp, i32, dp, dp, dp, dp, vp]
    lib.nc_diffusion.argtypes = [vp, i32, dp, dp, dp, dp, dp, dp, vp]
    lib.nc_divdamp3d.argtypes = [vp, i32, dp, dp, dp, dp, vp]
    lib.nc_divdamp2d.argtypes = [vp, i32, dp, dp, dp, dp, vp]
    lib.nc_exchange.argtypes = [vp, i32, dp, dp, i32, vp]
    lib.nc_diffusion_kh.argtypes = [vp, dp, dp, dp, dp, dp, dp, vp]
    for f in ("nc_vsolve", "nc_vadv_lin", "nc_laplacian", "nc_trc_step_lin", "nc_set_time", "nc_trc_prepare",
              "nc_divergence", "nc_gradient", "nc_diffusion", "nc_divdamp3d", "nc_divdamp2d", "nc_exchange", "nc_diffusion_kh"):
        getattr(lib, f).restype = ctypes.c_int
    lib.nc_destroy.argtypes = [vp]
    lib.nc_destroy.restype = None
    for f in ("nc_create", "nc_upload_state", "nc_download_state", "nc_download_state_async", "nc_join_copies",
              "nc_upload_state_device", "nc_download_state_device", "nc_check_finite", "nc_set_block",
              "nc_get_block", "nc_step", "nc_set_graph", "nc_run_phases", "nc_sync", "nc_mass_sums", "nc_get_field", "nc_state_pointers", "nc_stream", "nc_profile"):
        getattr(lib, f).restype = ctypes.c_int
    _lib = lib
    return lib


NC_ERR_ARG, NC_ERR_CUDA, NC_ERR_STATE, NC_ERR_NONFINITE = 1, 2, 3, 4


class NicamError(RuntimeError):
    """a non-zero status of the C ABI; ``status`` holds the code"""

    def __init__(self, msg: str, status: int = 0):
        super().__init__(msg)
        self.status = status


class NonFiniteStateError(NicamError):
    """NC_ERR_NONFINITE: the device state holds a NaN or an infinity"""


def grid_spring(x, x_pl, have_sgp, plan, lam, dbar, dt, crit, max_iter):
    """Spring relaxation on the device (nc_grid_spring); x (L,G,G,3) and
    x_pl (2,6,3) are updated in place.  Returns the iteration count."""
    lib = load_library()
    x = np.ascontiguousarray(x, np.float64)
    x_pl = np.ascontiguousarray(x_pl, np.float64)
    sg = np.ascontiguousarray(have_sgp, np.uint8)
    r_dst, r_src, p_dst, p_src = (np.ascontiguousarray(a, np.int64) for a in plan)
    it = ctypes.c_int64(0)
    rc = lib.nc_grid_spring(x.shape[0], x.shape[1], x.ctypes.data, x_pl.ctypes.data, sg.ctypes.data,
                            r_dst.ctypes.data, r_src.ctypes.data, len(r_dst), p_dst.ctypes.data, p_src.ctypes.data,
                            len(p_dst), lam, dbar, dt, crit, int(max_iter), ctypes.byref(it))
    if rc != 0:
        raise NicamError(f"nc_grid_spring status {rc}: {lib.nc_last_error().decode(errors='replace')}")
    return x, x_pl, int(it.value)


def divide_known(x, b) -> np.ndarray:
    """x / b on the device with the kernels' division by a known divisor
    (nc_divide_known): b a float (constant divisor, reciprocal pair from the
    host) or an array like x (per-element reciprocal formed on the device).
    The result should equal numpy's x / b bit for bit."""
    lib = load_library()
    x = np.ascontiguousarray(x, np.float64)
    q = np.empty_like(x)
    if np.ndim(b) == 0:
        rc = lib.nc_divide_known(x.ctypes.data, None, q.ctypes.data, x.size, float(b))
    else:
        y = np.ascontiguousarray(b, np.float64)
        if y.shape != x.shape:
            raise ValueError("divisor array must have the shape of x")
        rc = lib.nc_divide_known(x.ctypes.data, y.ctypes.data, q.ctypes.data, x.size, 0.0)
    if rc != 0:
        raise NicamError(f"nc_divide_known status {rc}: {lib.nc_last_error().decode(errors='replace')}")
    return q


def _check(rc: int, lib=None):
    if rc != 0:
        msg = (lib or _lib).nc_last_error().decode(errors="replace")
        cls = NonFiniteStateError if rc == NC_ERR_NONFINITE else NicamError
        raise cls(f"libnicamcuda status {rc}: {msg}", rc)


def _dtype_code(a: np.ndarray) -> int:
    if a.dtype == np.float64:
        return NC_F64
    if a.dtype == np.int32:
        return NC_I32
    if a.dtype == np.int64:
        return NC_I64
    if a.dtype == np.bool_:
        return NC_BOOL
    raise TypeError(f"unsupported dtype {a.dtype}")


def _scalar(a):
    """the single value of a 0-d or one-element array (or a Python number)"""
    return np.asarray(a).reshape(-1)[0].item()


# derived history diagnostics: item names in the order of nc_history_vars's ids
# (the reference's I/O order, share/mod_io.py:251-260), the constants and the
# tracer indices of its setup entries
HIST_ITEMS = ('ml_u', 'ml_v', 'ml_w', 'ml_th', 'ml_thv', 'ml_omg', 'ml_pres', 'ml_tem', 'ml_rho', 'ml_hgt',
              'ml_mse', 'ml_rh', 'ml_rha', 'ml_rhi', 'ml_du', 'ml_dv', 'ml_dw', 'ml_dtem', 'ml_dq', 'ml_ucos',
              'ml_vcos', 'ml_th_prime', 'sl_ps', 'sl_pw', 'sl_lwp', 'sl_iwp') + tuple(
    f'sl_{f}{lev}' for lev in ('850', '500', '250', '100') for f in ('u', 'v', 'w', 't')) + (
    'sl_cl', 'sl_cl2', 'sl_cly')
HIST_CHEM = ('sl_cl', 'sl_cl2', 'sl_cly')   # AF_TYPE 'DCMIP' with the terminator chemistry only
HIST_N3 = 22
HIST_CONSTS = ("LHV", "UNDEF", "PSAT0", "RTEM00", "CPovR_liq", "CPovR_ice", "LovR_liq", "LovR_ice", "SAT_LLIMIT",
               "SAT_ULIMIT")
HIST_TRACERS = ("I_QV", "I_QC", "I_QR", "I_QI", "I_QS", "I_QG")


def dcmip_sst(lat, latdepend: bool, held_suarez: bool = False, mitc_type: int = 1):
    """the sea-surface temperature of the DCMIP simple physics per column
    (nhm/forcing/simple_physics.py:152-197 _sst_tsurf): for moist Held-Suarez
    the Gaussian-in-latitude profile of MITC type 1, 2 or 3, else the moist
    baroclinic wave's latitude profile, or 302.15 K everywhere; the
    reference's numpy expressions, so the device reads the reference's values"""
    import math
    pi = math.pi
    if held_suarez:
        if mitc_type == 1:
            return 29.0 * np.exp(-0.5 * lat * lat / (26.0 / 180.0 * pi) ** 2) + 271.0
        if mitc_type in (2, 3):
            amp, w, c0 = (29.0, 20.0, 17.0) if mitc_type == 2 else (32.0, 23.0, 12.0)
            dphi2, dphi0 = (w / 180.0 * pi) ** 2, (c0 / 180.0 * pi)
            return amp * np.exp(-0.5 * np.maximum(np.abs(lat) - dphi0, 0.0) ** 2 / dphi2) + 271.0
        raise ValueError(f"MITC_TYPE out of range: {mitc_type}")
    if not latdepend:
        return np.full_like(lat, 302.15)
    T00, u0, a, omega, q0, eta0, rair, rh2o = 288.0, 35.0, 6371220.0, 7.29212e-5, 0.021, 0.252, 287.0, 461.5
    zvir = (rh2o / rair) - 1.0
    etav, latw = (1.0 - eta0) * 0.5 * pi, 2.0 * pi / 9.0
    sinl, cosl = np.sin(lat), np.cos(lat)
    termA = (-2.0 * sinl ** 6 * (cosl ** 2 + 1.0 / 3.0) + 10.0 / 63.0) * u0 * (math.cos(etav)) ** 1.5
    termB = (8.0 / 5.0 * cosl ** 3 * (sinl ** 2 + 2.0 / 3.0) - pi / 4.0) * a * omega * 0.5
    pref = pi * u0 / rair * 1.5 * math.sin(etav) * (math.cos(etav)) ** 0.5
    return (T00 + pref * (termA + termB)) / (1.0 + zvir * q0 * np.exp(-(lat / latw) ** 4))


def setup_table(geo: dict) -> dict:
    """Host arrays handed to ``nc_create`` (names as in include/nicam_cuda.h).

    ``geo`` holds the reference's arrays under their attribute names (the
    layout of ``tests/golden`` fixtures).  Column subsets the device needs are
    cut here: GMTR_t weights W1..W3, GMTR_a outward normals HNX..HNZ of the
    three edges, GMTR_p inverse area.
    """
    t = {}
    for k in ("kall", "kmin", "kmax", "gall_1d", "gmin", "gmax", "lall", "nq"):
        t[k] = np.asarray(int(_scalar(geo[k])), np.int64)
    for k in ("GRAV", "Rdry", "CVdry", "CPdry", "Rvap", "OHM", "EPS", "HUGE", "rscale", "alpha", "dtl", "dts",
              "Kh_coef", "divdamp_coef", "hdiff_fact_rho"):
        t[k] = np.asarray(float(_scalar(geo[k])), np.float64)
    t["CVW"] = np.ascontiguousarray(geo["CVW"], np.float64)
    if "NQW_END" in geo:   # water tracers 0..NQW_END (RAIN_TYPE); the vapour alone when absent
        t["NQW_END"] = np.asarray(float(_scalar(geo["NQW_END"])), np.float64)
    t["sstep"] = np.ascontiguousarray(geo["sstep"], np.int64)
    if "hdiff_nl_kh_max" in geo:   # hyperdiffusion NONLINEAR1: the Kh bounds and 2 AREA_ave^2 / dtl
        area = float(_scalar(geo["hdiff_nl_area"]))
        t["hdiff_nl_kh_max"] = np.ascontiguousarray(geo["hdiff_nl_kh_max"], np.float64)
        t["hdiff_nl_area"] = np.asarray(area, np.float64)
        t["hdiff_nl_minlim"] = np.asarray(float(_scalar(geo["hdiff_nl_minlim"])), np.float64)
        t["hdiff_nl_c1"] = np.asarray(2.0 * (area ** 2) / float(_scalar(geo["dtl"])), np.float64)
    if "rayleigh_coef" in geo:   # Rayleigh sponge on the full and half levels
        t["rayleigh_coef"] = np.ascontiguousarray(geo["rayleigh_coef"], np.float64)
        t["rayleigh_coef_h"] = np.ascontiguousarray(geo["rayleigh_coef_h"], np.float64)
        t["rayleigh_only_w"] = np.asarray(float(_scalar(geo.get("rayleigh_only_w", 0))), np.float64)
    for k in ("GRD_afact", "GRD_bfact", "GRD_cfact", "GRD_dfact", "GRD_rdgz", "GRD_rdgzh"):
        t[k] = np.ascontiguousarray(geo[k], np.float64)
    for k in ("VMTR_GSGAM2", "VMTR_GSGAM2H", "VMTR_RGSGAM2", "VMTR_RGSGAM2H", "VMTR_RGSQRTH", "VMTR_RGAM",
              "VMTR_RGAMH", "VMTR_GAM2H", "VMTR_PHI", "VMTR_C2Wfact", "VMTR_W2Cfact", "VMTR_C2WfactGz",
              "VMTR_VOLUME", "rho_bs", "pre_bs", "tem_bs",
              "OPRT_coef_div", "OPRT_coef_grad", "OPRT_coef_lap", "OPRT_coef_intp", "OPRT_coef_diff",
              "GRD_x", "GRD_xr"):
        t[k] = np.ascontiguousarray(geo[k], np.float64)
        pk = k + "_pl"
        if pk in geo:
            t[pk] = np.ascontiguousarray(geo[pk], np.float64)
    for k in ("GMTR_t_pl", "GMTR_a_pl", "GMTR_p_pl"):
        t[k] = np.ascontiguousarray(geo[k], np.float64)
    t["GMTR_t_W"] = np.ascontiguousarray(np.asarray(geo["GMTR_t"])[..., 2:5], np.float64)
    t["GMTR_a_HN"] = np.ascontiguousarray(np.asarray(geo["GMTR_a"])[..., 0:3], np.float64)
    t["GMTR_p_RAREA"] = np.ascontiguousarray(np.asarray(geo["GMTR_p"])[..., 1:2], np.float64)
    trcadv = str(np.asarray(geo.get("integ_type", "RK3"))) == "TRCADV"
    if trcadv:   # offline tracer advection: the coordinates the prescribed winds are computed from
        # 1: the DCMIP 1-1 winds, 2: the DCMIP 1-2 winds (Hadley-like circulation)
        t["trcadv"] = np.asarray(2.0 if str(np.asarray(geo.get("trcadv_case", "1-1"))) == "1-2" else 1.0, np.float64)
        G, L = int(_scalar(geo["gall_1d"])), int(_scalar(geo["lall"]))
        for k in ("GRD_LON", "GRD_LAT"):
            t[k] = np.ascontiguousarray(np.asarray(geo[k], np.float64).reshape(G, G, 1, L))
        for k in ("GRD_Z", "GRD_ZH", "GRD_LON_pl", "GRD_LAT_pl", "GRD_Z_pl", "GRD_ZH_pl"):
            t[k] = np.ascontiguousarray(geo[k], np.float64)
    if "GRD_LAT" in geo and not trcadv:   # Held-Suarez forcing: latitude terms with the reference's numpy expressions
        lat = np.asarray(geo["GRD_LAT"], np.float64)
        lat = lat.reshape(lat.shape[0], lat.shape[1], 1, lat.shape[-1])
        sinlat, coslat = np.abs(np.sin(lat)), np.abs(np.cos(lat))
        t["AF_hs_lat_terms"] = np.ascontiguousarray(np.stack([sinlat ** 2, coslat ** 2, coslat ** 4], axis=-1))
        t["PRE00"] = np.asarray(float(_scalar(geo["PRE00"])), np.float64)
    if int(np.asarray(geo.get("AF_dcmip_kessler", 0))):   # DCMIP forcing, Kessler microphysics only
        t["AF_dcmip_kessler_zf"] = np.ascontiguousarray(geo["GRD_Z"], np.float64)
        t["PRE00"] = np.asarray(float(_scalar(geo["PRE00"])), np.float64)
        for k in ("AF_negative_fixer", "AF_update_tot_dens"):
            if k in geo:
                t[k] = np.asarray(float(_scalar(geo[k])), np.float64)
        if "AF_dcmip_schemes" in geo:
            # [Kessler, simple physics, latitude-dependent SST, condensation(, moist Held-Suarez, MITC SST
            # type(, Bryan boundary layer))]
            fl = [int(x) for x in np.asarray(geo["AF_dcmip_schemes"]).reshape(-1)]
            kes, sm, latdep, lsc = fl[:4]
            hs, mitc = (fl[4], fl[5]) if len(fl) >= 6 else (0, 1)
            bryan = fl[6] if len(fl) >= 7 else 0
            t["AF_dcmip_schemes"] = np.asarray([kes, sm, lsc, hs, bryan], np.int64)
            G, L = int(_scalar(geo["gall_1d"])), int(_scalar(geo["lall"]))
            if sm or hs:
                lat = np.asarray(geo["AF_dcmip_lat"], np.float64).reshape(G, G, 1, L)
            if sm:
                t["AF_dcmip_zh"] = np.ascontiguousarray(geo["AF_dcmip_zh"], np.float64)
                t["AF_dcmip_zsfc"] = np.ascontiguousarray(np.asarray(geo["AF_dcmip_zsfc"], np.float64).reshape(G, G, 1, L))
                t["AF_dcmip_ij"] = np.ascontiguousarray(np.asarray(geo["AF_dcmip_ij"], np.float64).reshape(G, G, 1, L, 6))
                t["AF_dcmip_tsurf"] = np.ascontiguousarray(dcmip_sst(lat, bool(latdep), bool(hs), mitc))
            if hs:   # the Held-Suarez latitude terms, as for AF_TYPE 'HELD-SUAREZ'
                sinlat, coslat = np.abs(np.sin(lat)), np.abs(np.cos(lat))
                t["AF_dcmip_hs_lat_terms"] = np.ascontiguousarray(np.stack([sinlat ** 2, coslat ** 2, coslat ** 4], -1))
        if "AF_dcmip_chem" in geo:   # terminator toy chemistry: (Cl, Cl2) tracer indices, column lat / lon
            G, L = int(_scalar(geo["gall_1d"])), int(_scalar(geo["lall"]))
            t["AF_dcmip_chem"] = np.ascontiguousarray(np.asarray(geo["AF_dcmip_chem"]).reshape(2), np.int64)
            for k in ("AF_dcmip_lat", "AF_dcmip_lon"):
                t[k] = np.ascontiguousarray(np.asarray(geo[k], np.float64).reshape(G, G, 1, L))
    if "hist_hgt" in geo:   # derived history diagnostics (nc_history_vars)
        G, L = int(_scalar(geo["gall_1d"])), int(_scalar(geo["lall"]))
        plane = lambda x: np.ascontiguousarray(np.asarray(x, np.float64).reshape(G, G, 1, L))
        t["HIST_hgt"] = np.ascontiguousarray(geo["hist_hgt"], np.float64)
        t["HIST_coslat"] = plane(np.cos(np.asarray(geo["hist_lat"], np.float64)))
        t["HIST_zsfc"] = plane(geo["hist_zsfc"])
        t["HIST_area"] = plane(geo["hist_area"])
        t["HIST_IJ"] = np.ascontiguousarray(np.asarray(geo["hist_IJ"], np.float64).reshape(G, G, 1, L, 6))
        t["HIST_dgz"] = np.ascontiguousarray(geo["hist_dgz"], np.float64)
        t["HIST_consts"] = np.ascontiguousarray([float(_scalar(geo["hist_" + k])) for k in HIST_CONSTS], np.float64)
        t["HIST_tracers"] = np.ascontiguousarray([int(_scalar(geo["hist_" + k])) for k in HIST_TRACERS], np.int64)
        if "hist_NCHEM" in geo:   # the terminator chemistry's tracers (NCHEM_STR, NCHEM_END)
            t["HIST_chem"] = np.ascontiguousarray(np.asarray(geo["hist_NCHEM"]).reshape(2), np.int64)
        t["PRE00"] = np.asarray(float(_scalar(geo["PRE00"])), np.float64)
    t["pntmask"] = np.ascontiguousarray(geo["pntmask"], np.int32)
    t["have_sgp"] = np.ascontiguousarray(geo["have_sgp"], np.bool_)
    if "halo_plan" in geo:   # composed elsewhere (ensemble.stack_setup: members stacked along the regions)
        plan = geo["halo_plan"]
    else:
        plan = halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"], geo["copy_sgp"],
                            int(_scalar(geo["gall_1d"])), int(_scalar(geo["lall"])))
    if "members" in geo:
        t["members"] = np.asarray(int(_scalar(geo["members"])), np.int64)
    for k, v in zip(("halo_r_dst", "halo_r_src", "halo_p_dst", "halo_p_src"), plan):
        t[k] = np.ascontiguousarray(v, np.int64)
    return t


PRECISIONS = ("float64", "mixed")


class NicamCuda:
    """One device-resident NICAM-DC dynamical core (one C-ABI handle).

    ``precision`` is "float64" (the reference's numpy arithmetic, bit for
    bit) or "mixed": float32 work fields, metrics and stencil / advection /
    hyperdiffusion arithmetic, with the tridiagonal (HEVI) elimination and its
    matrix, the pressure and density deviations from the reference state and
    the mass sums in float64.  The host-side state stays float64 in both."""

    def __init__(self, geo: dict, graph: bool = True, precision: str = "float64"):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {PRECISIONS}, got {precision!r}")
        lib = load_library()
        self._lib = lib
        self.precision = precision
        self._tab = setup_table(geo)
        self._tab["precision"] = np.asarray(1.0 if precision == "mixed" else 0.0, np.float64)
        names, arrs = [], []
        entries = (NcArray * len(self._tab))()
        for n, (k, a) in enumerate(self._tab.items()):
            a = np.ascontiguousarray(a)
            self._tab[k] = a
            names.append(k.encode())
            e = entries[n]
            e.name = names[-1]
            e.data = a.ctypes.data
            e.dtype = _dtype_code(a)
            e.ndim = a.ndim
            for d in range(a.ndim):
                e.shape[d] = a.shape[d]
        self._names = names
        h = ctypes.c_void_p()
        _check(lib.nc_create(entries, len(self._tab), ctypes.byref(h)))
        self._h = h
        _check(lib.nc_set_graph(h, 1 if graph else 0))
        G, K, L, nq = (int(_scalar(self._tab[k])) for k in ("gall_1d", "kall", "lall", "nq"))
        self.shape = (G, G, K, L, 6 + nq)
        LP = 2 * (int(_scalar(self._tab["members"])) if "members" in self._tab else 1)
        self.shape_pl = (6, K, LP, 6 + nq)
        self.kmin, self.kmax = int(_scalar(self._tab["kmin"])), int(_scalar(self._tab["kmax"]))

    # ---- state marshal (host arrays in the reference layout)
    def upload(self, prg: np.ndarray, prg_pl: np.ndarray):
        if prg.shape != self.shape or prg_pl.shape != self.shape_pl:
            raise ValueError(f"state shape {prg.shape}/{prg_pl.shape}, expected {self.shape}/{self.shape_pl}")
        prg = np.ascontiguousarray(prg, np.float64)
        prg_pl = np.ascontiguousarray(prg_pl, np.float64)
        self._keep = (prg, prg_pl)
        _check(self._lib.nc_upload_state(self._h, prg.ctypes.data, prg_pl.ctypes.data))

    def upload_ptr(self, prg_ptr: int, prg_pl_ptr: int):
        """upload from raw host pointers (e.g. pinned torch tensors)"""
        _check(self._lib.nc_upload_state(self._h, prg_ptr, prg_pl_ptr))

    def download(self, prg: np.ndarray = None, prg_pl: np.ndarray = None):
        if prg is None:
            prg = np.empty(self.shape)
        if prg_pl is None:
            prg_pl = np.empty(self.shape_pl)
        _check(self._lib.nc_download_state(self._h, prg.ctypes.data, prg_pl.ctypes.data))
        return prg, prg_pl

    def download_ptr(self, prg_ptr: int, prg_pl_ptr: int):
        _check(self._lib.nc_download_state(self._h, prg_ptr, prg_pl_ptr))

    def upload_tensor(self, prg, prg_pl):
        """marshal-in from CUDA tensors (torch.float64, contiguous, the
        reference layout and shapes), ordered on torch's current stream"""
        self._check_tensors(prg, prg_pl)
        import torch
        st = torch.cuda.current_stream(prg.device).cuda_stream
        _check(self._lib.nc_upload_state_device(self._h, prg.data_ptr(), prg_pl.data_ptr(), st))

    def download_tensor(self, prg=None, prg_pl=None):
        """marshal-out into CUDA tensors (allocated when not given), ordered
        on torch's current stream; returns (prg, prg_pl)"""
        import torch
        if prg is None:
            prg = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        if prg_pl is None:
            prg_pl = torch.empty(self.shape_pl, dtype=torch.float64, device=prg.device)
        self._check_tensors(prg, prg_pl)
        st = torch.cuda.current_stream(prg.device).cuda_stream
        _check(self._lib.nc_download_state_device(self._h, prg.data_ptr(), prg_pl.data_ptr(), st))
        return prg, prg_pl

    def _check_tensors(self, prg, prg_pl):
        import torch
        for t, shp in ((prg, self.shape), (prg_pl, self.shape_pl)):
            if (not t.is_cuda or t.dtype != torch.float64 or tuple(t.shape) != tuple(shp)
                    or not t.is_contiguous()):
                raise ValueError(f"expected a contiguous float64 CUDA tensor of shape {shp}, got "
                                 f"{t.dtype} {tuple(t.shape)} on {t.device}")

    # ---- tangent-linear / adjoint operators on device-layout tensors
    # (regional [l][k][j][i] = shape (lall, kall, gall_1d, gall_1d), pole
    # [g][k][lp] = shape (6, kall, 2); float64 handles only)
    @property
    def field_shape(self):
        G, K, L = self.shape[0], self.shape[2], self.shape[3]
        return (L, K, G, G)

    @property
    def field_shape_pl(self):
        return (6, self.shape[2], self.shape_pl[2])

    def _dev(self, t, pole: bool = False, comps: int = 0):
        import torch
        shp = self.field_shape_pl if pole else self.field_shape
        if comps:
            shp = (comps,) + shp
        if t is None:
            return None
        if not t.is_cuda or t.dtype != torch.float64 or tuple(t.shape) != shp or not t.is_contiguous():
            raise ValueError(f"expected a contiguous float64 CUDA tensor of shape {shp}, got "
                             f"{t.dtype} {tuple(t.shape)} on {t.device}")
        return t.data_ptr()

    def vsolve(self, Mc, Mu, Ml, b, x, pole: bool = False, transpose: bool = False, x_fwd=None, gM=None):
        """nc_vsolve: x = M^-1 b (M^-T b with transpose); with x_fwd and
        gM = (gMc, gMu, gMl) also the matrix cotangents"""
        import torch
        st = torch.cuda.current_stream(b.device).cuda_stream
        g = gM if gM is not None else (None, None, None)
        _check(self._lib.nc_vsolve(self._h, int(pole), int(transpose), *(self._dev(t, pole) for t in (Mc, Mu, Ml, b, x)),
                                   self._dev(x_fwd, pole), *(self._dev(t, pole) for t in g), st))

    def vadv_lin(self, mode: int, rhogq, den, flx_v, frhog, inp, out, dt: float, bcoef: float = 0.0,
                 clamp: bool = True, pole: bool = False):
        """nc_vadv_lin: mode 0 F(rhogq), 1 dF(inp), 2 dF^T(inp) into out"""
        import torch
        st = torch.cuda.current_stream(out.device).cuda_stream
        _check(self._lib.nc_vadv_lin(self._h, int(pole), int(mode), *(self._dev(t, pole) for t in
                                                                      (rhogq, den, flx_v, frhog, inp, out)),
                                     float(dt), float(bcoef), int(bool(clamp)), st))

    def laplacian(self, q, q_pl, y, y_pl, transpose: bool = False):
        """nc_laplacian: y = L(C(q)), or C^T L^T q with transpose"""
        import torch
        st = torch.cuda.current_stream(q.device).cuda_stream
        _check(self._lib.nc_laplacian(self._h, int(transpose), self._dev(q), self._dev(q_pl, True), self._dev(y),
                                      self._dev(y_pl, True), st))

    @property
    def trcadv(self) -> bool:
        return "trcadv" in self._tab and float(_scalar(self._tab["trcadv"])) != 0.0

    def set_time(self, time: float):
        """the model time of the prescribed winds of an offline-advection
        (trcadv) handle (nc_set_time); it starts at 0 and each step adds dtl"""
        _check(self._lib.nc_set_time(self._h, float(time)))

    def divergence(self, v, v_pl, y, y_pl, transpose: bool = False):
        """nc_divergence: y = D(C(v)) (v of shape (3,) + field shape), or
        v = C^T D^T y with transpose"""
        import torch
        st = torch.cuda.current_stream(y.device).cuda_stream
        _check(self._lib.nc_divergence(self._h, int(transpose), self._dev(v, comps=3), self._dev(v_pl, True, 3),
                                       self._dev(y), self._dev(y_pl, True), st))

    def gradient(self, q, q_pl, g, g_pl, transpose: bool = False):
        """nc_gradient: g = Grad(C(q)) (g of shape (3,) + field shape), or
        q = C^T Grad^T g with transpose"""
        import torch
        st = torch.cuda.current_stream(q.device).cuda_stream
        _check(self._lib.nc_gradient(self._h, int(transpose), self._dev(q), self._dev(q_pl, True),
                                     self._dev(g, comps=3), self._dev(g_pl, True, 3), st))

    def diffusion(self, kh, kh_pl, s, s_pl, y, y_pl, transpose: bool = False):
        """nc_diffusion: y = Dk(C(s)), the kh-weighted diffusion after the halo
        exchange, or s = C^T Dk^T y with transpose (kh fixed)"""
        import torch
        st = torch.cuda.current_stream(s.device).cuda_stream
        _check(self._lib.nc_diffusion(self._h, int(transpose), self._dev(kh), self._dev(kh_pl, True), self._dev(s),
                                      self._dev(s_pl, True), self._dev(y), self._dev(y_pl, True), st))

    def diffusion_kh(self, s, s_pl, y, y_pl, gkh, gkh_pl):
        """nc_diffusion_kh: gkh = d<y, Dk(C(s))>/dkh"""
        import torch
        st = torch.cuda.current_stream(s.device).cuda_stream
        _check(self._lib.nc_diffusion_kh(self._h, self._dev(s), self._dev(s_pl, True), self._dev(y),
                                         self._dev(y_pl, True), self._dev(gkh), self._dev(gkh_pl, True), st))

    def exchange(self, x, x_pl, transpose: bool = False):
        """nc_exchange: the halo exchange of x (nf,) + field shape (or one
        field) in place, or its adjoint with transpose"""
        import torch
        nf = x.shape[0] if x.dim() == len(self.field_shape) + 1 else 0
        st = torch.cuda.current_stream(x.device).cuda_stream
        _check(self._lib.nc_exchange(self._h, int(transpose), self._dev(x, comps=nf), self._dev(x_pl, True, nf),
                                     max(nf, 1), st))

    def divdamp3d(self, v, v_pl, y, y_pl, transpose: bool = False):
        """nc_divdamp3d: y = D3(C(v)) (v of shape (4,) + field shape: the four
        momenta; y (3,) + field shape), or v = C^T D3^T y with transpose"""
        import torch
        st = torch.cuda.current_stream(y.device).cuda_stream
        _check(self._lib.nc_divdamp3d(self._h, int(transpose), self._dev(v, comps=4), self._dev(v_pl, True, 4),
                                      self._dev(y, comps=3), self._dev(y_pl, True, 3), st))

    def divdamp2d(self, v, v_pl, y, y_pl, transpose: bool = False):
        """nc_divdamp2d: y = D2(C(v)) (v and y of shape (3,) + field shape), or
        v = C^T D2^T y with transpose"""
        import torch
        st = torch.cuda.current_stream(y.device).cuda_stream
        _check(self._lib.nc_divdamp2d(self._h, int(transpose), self._dev(v, comps=3), self._dev(v_pl, True, 3),
                                      self._dev(y, comps=3), self._dev(y_pl, True, 3), st))

    def trc_prepare(self):
        """offline advection: the uploaded state's winds onto the handle as
        its step's tracer advection reads them, without stepping
        (nc_trc_prepare)"""
        _check(self._lib.nc_trc_prepare(self._h))

    def trc_step_lin(self, mode: int, x0, x0_pl, inp, inp_pl, out, out_pl):
        """nc_trc_step_lin: the tracer advection of the handle's last step
        applied to the tracer mass x0 (mode 0), its tangent-linear (1) or
        adjoint (2) applied to inp, into out"""
        import torch
        st = torch.cuda.current_stream(out.device).cuda_stream
        _check(self._lib.nc_trc_step_lin(self._h, int(mode), self._dev(x0), self._dev(x0_pl, True), self._dev(inp),
                                         self._dev(inp_pl, True), self._dev(out), self._dev(out_pl, True), st))

    def set_block(self, kernel: str, threads: int):
        """threads per block of a column / point kernel (nc_set_block)"""
        _check(self._lib.nc_set_block(self._h, kernel.encode(), int(threads)))

    def get_block(self, kernel: str) -> int:
        t = ctypes.c_int32(0)
        _check(self._lib.nc_get_block(self._h, kernel.encode(), ctypes.byref(t)))
        return int(t.value)

    def check_finite(self):
        """raise NonFiniteStateError if the device state holds a NaN or an
        infinity (nc_check_finite)"""
        _check(self._lib.nc_check_finite(self._h))

    def download_ptr_async(self, prg_ptr: int, prg_pl_ptr: int):
        """download into raw (pinned) host pointers without waiting; the data
        are there after sync()"""
        _check(self._lib.nc_download_state_async(self._h, prg_ptr, prg_pl_ptr))

    def join_copies(self):
        """order the library stream after the last upload / download copies"""
        _check(self._lib.nc_join_copies(self._h))

    def step(self, nsteps: int = 1):
        _check(self._lib.nc_step(self._h, int(nsteps)))

    def forcing_step(self):
        """Dyn.forcing_step for AF_TYPE 'HELD-SUAREZ' (nc_forcing_step); the
        handle must have been built from a setup with GRD_LAT"""
        _check(self._lib.nc_forcing_step(self._h))

    def forcing_precip(self) -> np.ndarray:
        """the precipitation rate of the last DCMIP Kessler forcing step,
        (gall_1d, gall_1d, lall) (nc_forcing_precip)"""
        out = np.empty((self.shape[0], self.shape[1], self.shape[3]))
        _check(self._lib.nc_forcing_precip(self._h, out.ctypes.data))
        return out

    def history_vars(self, names, nstep: int, dt: float) -> dict:
        """the derived history diagnostics ``names`` (from ``HIST_ITEMS``) of
        the device state (nc_history_vars): {name: host array}, model-level
        fields (gall_1d, gall_1d, kall, lall), slices and column integrals
        (gall_1d, gall_1d, lall)"""
        ids = []
        for n in names:
            if n not in HIST_ITEMS:
                raise NotImplementedError(f"history diagnostic {n!r} is not built on the device")
            ids.append(HIST_ITEMS.index(n))
        G, K, L = self.shape[0], self.shape[2], self.shape[3]
        res = {n: np.empty((G, G, K, L) if i < HIST_N3 else (G, G, L)) for n, i in zip(names, ids)}
        idarr = np.ascontiguousarray(ids, np.int32)
        ptrs = np.ascontiguousarray([res[n].ctypes.data for n in names], np.uint64)
        _check(self._lib.nc_history_vars(self._h, idarr.ctypes.data if ids else None, len(ids), int(nstep),
                                         float(dt), ptrs.ctypes.data if ids else None))
        return res

    # ---- restart payloads (fio "ADVANCED" byte order; see restart.py)
    def restart_pack(self, var: int, buf: np.ndarray):
        """the big-endian file payload of prognostic ``var`` into ``buf``
        (lall*kall*gall_1d^2 float64 slots)"""
        if buf.nbytes != 8 * self.shape[0] * self.shape[1] * self.shape[2] * self.shape[3]:
            raise ValueError("restart payload buffer has the wrong size")
        _check(self._lib.nc_restart_pack(self._h, int(var), buf.ctypes.data))

    def restart_unpack(self, var: int, buf: np.ndarray):
        if buf.nbytes != 8 * self.shape[0] * self.shape[1] * self.shape[2] * self.shape[3]:
            raise ValueError("restart payload has the wrong size")
        buf = np.ascontiguousarray(buf)
        _check(self._lib.nc_restart_unpack(self._h, int(var), buf.ctypes.data))

    def restart_finish(self, pole_src):
        ps = np.ascontiguousarray(pole_src, np.int64).reshape(-1, 5)
        _check(self._lib.nc_restart_finish(self._h, ps.ctypes.data if len(ps) else None, len(ps)))

    def run_phases(self, nphases: int):
        """debugging: run the first ``nphases`` phases of one step"""
        _check(self._lib.nc_run_phases(self._h, int(nphases)))

    def sync(self):
        _check(self._lib.nc_sync(self._h))

    def mass_sums(self):
        n = 1 + int(_scalar(self._tab["nq"]))
        out = np.zeros(n)
        _check(self._lib.nc_mass_sums(self._h, out.ctypes.data, n))
        return out

    def field(self, name: str):
        """a named device work field in the reference layout (debug / parity)"""
        reg = np.empty(self.shape[:4])
        pl = np.empty(self.shape_pl[:3])
        _check(self._lib.nc_get_field(self._h, name.encode(), reg.ctypes.data, pl.ctypes.data))
        return reg, pl

    def kernel_launches(self) -> int:
        return int(self._lib.nc_kernel_launches(self._h))

    def stream_ptr(self) -> int:
        """cudaStream_t of the handle (for CUDA events on the same stream)"""
        p = ctypes.c_void_p()
        _check(self._lib.nc_stream(self._h, ctypes.byref(p)))
        return int(p.value or 0)

    def profile(self, enable: bool):
        _check(self._lib.nc_profile(self._h, 1 if enable else 0))

    def kernel_stats(self) -> dict:
        """{kernel name: (total ms, launches)} of the profiled steps"""
        n = self._lib.nc_kernel_stats(self._h, 0, None, None, None)
        if n < 0:
            _check(-n)
        names = ctypes.create_string_buffer(48 * max(n, 1))
        ms = np.zeros(max(n, 1))
        cnt = np.zeros(max(n, 1), np.int64)
        self._lib.nc_kernel_stats(self._h, n, names, ms.ctypes.data, cnt.ctypes.data)
        out = {}
        for k in range(n):
            nm = names.raw[48 * k:48 * (k + 1)].split(b"\0", 1)[0].decode()
            out[nm] = (float(ms[k]), int(cnt[k]))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.nc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

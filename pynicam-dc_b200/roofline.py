"""Algorithmic HBM bytes of one large step: the roofline's numerator.

Every regional kernel of the step is listed with the 3-D arrays it reads and
writes once per launch and the 2-D coefficient planes it reads once, named as
in the kernels' argument structs (csrc/nc_*.cuh).  A 3-D array is one pass of
lall * kall * gall_1d^2 values; a plane is lall * gall_1d^2 values.  The
element size follows the array's class:

* ``f``   work and state fields: 8 bytes (float64 form) or 4 (mixed form);
* ``f64`` the float64 islands of the mixed form (the deviations pregd /
          rhogd and the implicit matrix Mc / Mu / Ml): 8 bytes in both forms;
* ``m``   3-D metrics and ``p`` 2-D coefficient planes: 8 or 4 bytes, like
          ``f``.

Reads of neighbouring cells or levels of an array count once (the tiles and
the L2 keep them on chip; the ncu captures confirm DRAM traffic at or below
these bytes for the stencils).  The gamma-factor metrics RGAM / RGAMH / GAM2H
are not counted where the kernels skip them on a shallow atmosphere (every
value exactly 1: ``gam_at``), and are counted where a kernel reads them
unconditionally (vp0_h, path1, trc_hflux).  Pole kernels (12 columns) and the
halo-index reads of the exchanges are left out; the exchanges count their
halo values read and written.  Boundary rows touched by one or two levels of
a kernel are not counted.
"""
from __future__ import annotations

PROG = ("RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE")


def _n(prefix, n, start=0):
    return tuple(f"{prefix}{i}" for i in range(start, start + n))


# kernel -> (reads, writes, planes); entries are (name, class)
def _f(*names):
    return tuple((n, "f") for n in names)


def _m(*names):
    return tuple((n, "m") for n in names)


def _f64(*names):
    return tuple((n, "f64") for n in names)


C2WGZ = _m(*_n("C2WGz.", 6))
KERNELS = {
    # Pre_Post: diagnostics, boundary conditions, eth, deviations, merged velocity (k_diag)
    "diag": (_f(*PROG, "RHOGQ1") + _m("GSGAM2", "C2W.0", "C2W.1", "pre_bs", "rho_bs"),
             _f("pre", "tem", "vx", "vy", "vz", "w", "rho", "ein", "eth", "vvx", "vvy", "vvz") + _f64("pregd", "rhogd"),
             _n("GRD_x.", 3)),
    # momentum advection (k_advmom_t)
    "advmom": (_f(*PROG[:5], "vvx", "vvy", "vvz") + C2WGZ + _m("RGSQRTH", "C2W.0", "C2W.1"),
               _f(*_n("gadv.", 4)),
               _n("coef_div.", 21) + _n("GRD_x.", 3)),
    # hyperdiffusion, first and second Laplacian pass (k_hdiff1, k_hdiff2_l)
    "hdiff1": (_f("vx", "vy", "vz", "w", "tem", "rho") + _m("tem_bs", "rho_bs"), _f(*_n("vt.", 6)),
               _n("coef_lap.", 7)),
    "hdiff2": (_f(*_n("vt.", 6), "RHOG"), _f(*_n("vt2.", 6)),
               _n("intp_w.", 18) + _n("coef_lap.", 7) + _n("coef_diff.", 18)),
    # large-step tendency (k_gtend)
    "gtend": (_f(*_n("vt2.", 6), "RHOG", *_n("gadv.", 4)) + _m("C2W.0", "C2W.1"), _f(*_n("gT0.", 6), "frhog"),
              _n("GRD_x.", 3)),
    # PROG_split / PROG_mean initialisation (k_split_init); the first stage reads no PROG0
    "split_init": (_f(*_n("PROG0.", 6), *PROG), _f(*_n("PS.", 6), *_n("PM.", 5)), ()),
    "split_init_first": (_f(*PROG), _f(*_n("PS.", 6), *_n("PM.", 5)), ()),
    # 3-D divergence damping (k_dd3d_t): momenta of PROG or PROG_split
    "dd3d": (_f("RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW") + C2WGZ + _m("RGSQRTH"), _f(*_n("vtmp2.", 3)),
             _n("coef_intp.", 18) + _n("coef_diff.", 18)),
    # vp0 horizontal terms (k_vp0_hl) and column part with the implicit matrix (k_vp0_cr)
    "vp0_h": (_f("eth", "RHOGVX", "RHOGVY", "RHOGVZ", *_n("vtmp2.", 3)) + _f64("pregd") +
              _m("RGAM", "RGAMH") + C2WGZ,
              _f(*_n("vph.", 8)),
              _n("GRD_x.", 3) + _n("coef_div.", 21) + _n("coef_intp.", 18) + _n("coef_diff.", 18) +
              _n("coef_grad.", 21)),
    "vp0_c": (_f(*PROG[:5], "eth", *_n("vph.", 8), "vx", "vy", "vz", *_n("gT0.", 6)) + _f64("pregd", "rhogd") +
              _m("RGSQRTH", "C2W.0", "C2W.1", "W2C.0", "W2C.1", "RGSGAM2", "PHI") + C2WGZ,
              _f(*_n("gT.", 6), "ethtot0") + _f64("Mc", "Mu", "Ml"), ()),
    # acoustic loop: path 1 (k_path1_l), vi_main horizontal divergences (k_vimain_a_l),
    # Thomas solve (k_vi_solve) and energy update (k_vi_energy_p)
    "path1": (_f(*_n("vtmp2.", 3), "PS.5", "PS.1", "PS.2", "PS.3", "gT.1", "gT.2", "gT.3", "PM.1", "PM.2", "PM.3") +
              _m("RGAM", "RGAMH") + C2WGZ,
              _f("dvh.0", "dvh.1", "dvh.2", "PM.1", "PM.2", "PM.3"),
              _n("GRD_x.", 3) + _n("coef_intp.", 18) + _n("coef_diff.", 18) + _n("coef_grad.", 21)),
    "vimain_a": (_f("eth", "ethtot0", "dvh.0", "dvh.1", "dvh.2", "RHOGVX", "RHOGVY", "RHOGVZ"),
                 _f("hdiv.0", "hdiv.1", "hdiv.2"), _n("coef_div.", 21)),
    "vi_solve": (_f("dvh.0", "dvh.1", "dvh.2", "eth", "PS.0", "PS.4", "PS.5", "hdiv.0", "hdiv.1", "gT.0", "gT.4", "gT.5",
                    "PM.0", "PM.4") + _f64("Mc", "Mu", "Ml") + C2WGZ + _m("RGSQRTH", "RGSGAM2", "GSGAM2H"),
                 _f("dwe.0", "dwe.1", "PM.0", "PM.4"), ()),
    "vi_energy": (_f(*PROG[:5], "PS.0", "PS.1", "PS.2", "PS.3", "PS.4", "PS.5", "dwe.0", "dwe.1", "dvh.0", "dvh.1", "dvh.2",
                     "hdiv.2", "ethtot0", "gT0.5") + _m("C2W.0", "C2W.1", "W2C.0", "W2C.1", "RGSQRTH", "PHI") + C2WGZ,
                  _f("dwe.2"), ()),
    # PROG += PROG_split with the projection (k_post)
    "post": (_f(*PROG, *_n("PS.", 6)), _f(*PROG), _n("GRD_x.", 3)),
    # tracer advection (nc_tracer.cuh)
    "trc_vflux": (_f("PM.1", "PM.2", "PM.3", "PM.4", "PROG0.0", "frhog") + C2WGZ + _m("RGSQRTH"), _f("flx_v", "rhog_t"),
                  ()),
    "trc_vadv": (_f("RHOGQ1", "den", "flx_v", "frhog"), _f("RHOGQ1"), ()),
    "trc_hflux": (_f("PM.0", "PM.1", "PM.2", "PM.3", "rhog_t") + _m("RGAM"),
                  _f(*_n("flx.", 6), *_n("xc.", 9), *_n("ch.", 6), *_n("cm.", 6)),
                  _n("GMTR_t.", 6) + _n("GMTR_p.", 1) + _n("GMTR_a.", 9) + _n("GRD_xr.", 9)),
    "trc_grad": (_f("RHOGQ1", "rhog_t"), _f("q", "gq.0", "gq.1", "gq.2"), _n("coef_grad.", 21)),
    "trc_remap": (_f("q", "gq.0", "gq.1", "gq.2", *_n("xc.", 9), "cm.0", "cm.1", "cm.2"), _f("qa.0", "qa.1", "qa.2"),
                  _n("GRD_x.", 3)),
    "trc_qout": (_f("q", "cm.0", "cm.1", "cm.2", *_n("ch.", 6), "frhog", "rhog_t"), _f("Qmin", "Qmax"), ()),
    "trc_apply": (_f("cm.0", "cm.1", "cm.2", "qa.0", "qa.1", "qa.2", "q", "Qmin", "Qmax", *_n("flx.", 6), "RHOGQ1"),
                  _f("RHOGQ1"), ()),
    "trc_rhog": (_f("rhog_t", *_n("flx.", 6), "frhog"), _f("rhog_t"), ()),
}


def esize(cls: str, precision: str) -> int:
    if cls == "f64":
        return 8
    return 4 if precision == "mixed" else 8


def kernel_bytes(name: str, npt: int, npt2: int, precision: str = "float64") -> int:
    """algorithmic bytes of one launch of a regional kernel"""
    reads, writes, planes = KERNELS[name]
    b = sum(esize(c, precision) for _, c in reads + writes) * npt
    return b + len(planes) * esize("p", precision) * npt2


def kernel_passes(name: str) -> tuple:
    """(3-D array passes, planes) of one launch"""
    reads, writes, planes = KERNELS[name]
    return len(reads) + len(writes), len(planes)


def step_launches(sstep=(2, 3, 6), nq: int = 1) -> dict:
    """regional launches of each kernel in one large step (RK3, the acoustic
    steps sstep per stage, nq tracers)"""
    ns = sum(sstep)
    nst = len(sstep)
    return {"diag": nst, "advmom": nst, "hdiff1": nst, "hdiff2": nst, "gtend": nst, "split_init": nst - 1,
            "split_init_first": 1, "dd3d": nst + ns, "vp0_h": nst, "vp0_c": nst, "path1": ns, "vimain_a": ns,
            "vi_solve": ns, "vi_energy": ns, "post": nst, "trc_vflux": 1, "trc_vadv": 2 * nq, "trc_hflux": 1,
            "trc_grad": nq, "trc_remap": nq, "trc_qout": nq, "trc_apply": nq, "trc_rhog": 1}


def exchange_fields(sstep=(2, 3, 6), nq: int = 1) -> int:
    """fields moved by the halo exchanges of one large step"""
    ns = sum(sstep)
    nst = len(sstep)
    per_stage = 6 + 6 + 3 + 5          # hyperdiffusion x2, vp0 divergence damping, PROG_mean
    per_small = 3 + 3 + 3              # divergence damping, diff_vh, (rhog, rhogw, rhoge)_split
    return nst * per_stage + ns * per_small + (nst - 1) * 6 + nq * (3 + 2) + 6 + nq


def step_bytes(npt: int, npt2: int, halo_points: int, sstep=(2, 3, 6), nq: int = 1,
               precision: str = "float64") -> dict:
    """algorithmic bytes of one large step: the kernels (by name), the halo
    exchanges (halo_points = halo values per level and field: regional halo
    cells + pole neighbours; kall levels), and the PROG0 snapshot copy"""
    e = esize("f", precision)
    out = {k: n * kernel_bytes(k, npt, npt2, precision) for k, n in step_launches(sstep, nq).items()}
    kall_pts = npt // max(npt2, 1)
    out["comm"] = 2 * e * halo_points * kall_pts * exchange_fields(sstep, nq)
    out["prog0_copy"] = 2 * 6 * e * npt
    out["total"] = sum(out.values())
    return out


def field_passes(sstep=(2, 3, 6), nq: int = 1, kall: int = 42) -> float:
    """F: float64-equivalent field passes per step (3-D passes + planes / kall),
    the halo exchanges and the PROG0 copy included at their own sizes"""
    F = 0.0
    for k, n in step_launches(sstep, nq).items():
        f3, p2 = kernel_passes(k)
        F += n * (f3 + p2 / kall)
    return F + 12

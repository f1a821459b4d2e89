"""CPU oracle: float64 numpy restatement of the NICAM-DC dynamics step.

TEST INFRASTRUCTURE ONLY.  This module is the checker the CUDA path is compared
against; it is imported by ``tests/``, by ``__graft_entry__.smoke()`` and by the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` and by nothing else.
The product path never calls it.

It restates, operator by operator and in the same floating-point association
order, the reference's numpy backend of ``Dyn.dynamics_step``
(pynicamdc/nhm/dynamics/mod_dynamics.py:1725-2741) for the configuration the
reference runs in its JW baroclinic-wave case: RK3 HEVI, DIRECT lap_order-2
hyperdiffusion and divergence damping, NOBASE reference state, MIURA2004
tracer advection with the Thuburn limiters, TEM/TEM thermal and FREE/RIGID
momentum boundaries, one rank holding all regions and both poles.

Array layout is the reference's: regional ``(i, j, k, l)`` (+ trailing
component axis), pole ``(g, k, l)`` with g = 0 the pole point and 1..5 its
neighbours.  ``geo`` is the flat setup dict written by the fixture generator
(keys are the reference's attribute names, e.g. ``VMTR_RGAM``).

Pinned against the reference: ``tests/test_oracle_golden.py`` replays the
committed golden states produced by the reference itself
(``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import numpy as np

I_RHOG, I_RHOGVX, I_RHOGVY, I_RHOGVZ, I_RHOGW, I_RHOGE = 0, 1, 2, 3, 4, 5
I_pre, I_tem, I_vx, I_vy, I_vz, I_w = 0, 1, 2, 3, 4, 5
XDIR, YDIR, ZDIR = 0, 1, 2
TI, TJ = 0, 1
AI, AIJ, AJ = 0, 1, 2
W1, W2, W3 = 2, 3, 4            # GMTR_t column indices
P_RAREA = 1                      # GMTR_p column index
HNX, HNY, HNZ = 0, 1, 2          # GMTR_a column indices (regional and pole)


class Geo:
    """Run constants of one grid: a thin attribute view of the setup dict."""

    def __init__(self, d):
        self.d = d
        c = lambda k: d[k].item() if np.ndim(d[k]) == 0 else d[k]
        self.kall = int(c("kall"))
        self.kmin = int(c("kmin"))
        self.kmax = int(c("kmax"))
        self.gall_1d = int(c("gall_1d"))
        self.gmin = int(c("gmin"))
        self.gmax = int(c("gmax"))
        self.lall = int(c("lall"))
        self.have_sgp = np.asarray(d["have_sgp"], bool)
        self.pntmask = np.asarray(d["pntmask"])
        self.nq = int(c("nq"))
        for k in ("GRAV", "Rdry", "CVdry", "CPdry", "Rvap", "OHM", "RADIUS",
                  "EPS", "HUGE", "PRE00", "rscale", "alpha", "dtl", "dts",
                  "Kh_coef", "divdamp_coef", "hdiff_fact_rho"):
            setattr(self, k, float(c(k)))
        self.sstep = [int(x) for x in np.asarray(d["sstep"])]
        self.CVW = np.asarray(d["CVW"], np.float64)
        # water tracers 0..NQW_END (mod_runconf.py RUNCONF_tracer_setup: NQW_STR = I_QV = 0)
        self.nqw = int(c("NQW_END")) + 1 if "NQW_END" in d else 1

    def __getattr__(self, k):
        d = self.__dict__.get("d")
        if d is not None and k in d:
            return d[k]
        raise AttributeError(k)


# --------------------------------------------------------------------------
# halo exchange  (share/mod_comm.py:1563-1644, single rank: local copies only)
# --------------------------------------------------------------------------
def comm(g, var, var_pl):
    """In-place region-edge / pole / singular-point copy of ``var (i,j,k,l,v)``
    and ``var_pl (g,k,l,v)``; copy order and read-before-write semantics follow
    mod_comm.py:1613-1641."""
    c = g.copy_r2r
    if c.shape[1]:
        var[c[3], c[4], :, c[5], :] = var[c[0], c[1], :, c[2], :]
    c = g.copy_p2r
    if c.shape[1]:
        var[c[3], c[4], :, c[5], :] = var_pl[c[0], :, c[2], :]
    c = g.copy_r2p
    if c.shape[1]:
        var_pl[c[3], :, c[5], :] = var[c[0], c[1], :, c[2], :]
    c = g.copy_sgp
    if c.shape[1]:
        var[c[3], c[4], :, c[5], :] = var[c[0], c[1], :, c[2], :].copy()


def comm1(g, a, a_pl):
    """COMM of a single (i,j,k,l) field."""
    v = a[..., None].copy()
    vp = a_pl[..., None].copy()
    comm(g, v, vp)
    a[...] = v[..., 0]
    a_pl[...] = vp[..., 0]


# --------------------------------------------------------------------------
# Pre_Post: diagnostics, boundary conditions, deviations
# --------------------------------------------------------------------------
def diagnostics(g, PROG, PROGq, DIAG, PROG_pl, PROGq_pl, DIAG_pl):
    """kernels/diag.py:53-143 (regional) and mod_dynamics.py:1163-1196 (pole).
    Returns rho, ein, q (+pole) and writes DIAG/DIAG_pl in place."""
    kmin, kmax = g.kmin, g.kmax
    out = []
    for P, Pq, D, GS, C2W in ((PROG, PROGq, DIAG, g.VMTR_GSGAM2, g.VMTR_C2Wfact),
                              (PROG_pl, PROGq_pl, DIAG_pl, g.VMTR_GSGAM2_pl, g.VMTR_C2Wfact_pl)):
        RHOG = P[..., I_RHOG]
        rho = RHOG / GS
        D[..., I_vx] = P[..., I_RHOGVX] / RHOG
        D[..., I_vy] = P[..., I_RHOGVY] / RHOG
        D[..., I_vz] = P[..., I_RHOGVZ] / RHOG
        ein = P[..., I_RHOGE] / RHOG
        q = Pq / RHOG[..., None]
        # kernels/diag.py:97-115: cv and qd over the water range, sums in index order
        qw = q[..., 0:g.nqw]
        qd = 1.0 - np.sum(qw, axis=-1)
        cv = np.sum(qw * g.CVW[0:g.nqw], axis=-1) + qd * g.CVdry
        tem = ein / cv
        D[..., I_tem] = tem
        D[..., I_pre] = rho * tem * (qd * g.Rdry + q[..., 0] * g.Rvap)
        ks = [slice(None)] * (P.ndim - 1)
        kin, kdn = list(ks), list(ks)
        kax = P.ndim - 3
        kin[kax] = slice(kmin + 1, kmax + 1)
        kdn[kax] = slice(kmin, kmax)
        kin, kdn = tuple(kin), tuple(kdn)
        D[kin + (I_w,)] = P[kin + (I_RHOGW,)] / (C2W[kin + (0,)] * RHOG[kin] + C2W[kin + (1,)] * RHOG[kdn])
        out += [rho, ein, q]
    return out


def _kidx(a, k):
    """index k on the level axis of a regional (i,j,k,l) or pole (g,k,l) array"""
    return a[:, :, k, :] if a.ndim == 4 else a[:, k, :]


def _kset(a, k, v):
    if a.ndim == 4:
        a[:, :, k, :] = v
    else:
        a[:, k, :] = v


def bndcnd_all(g, DIAG, PROG, rho, ein, pole=False):
    """share/mod_bndcnd.py:182-264 with kernels/bndcnd.py (TEM/TEM, FREE top,
    RIGID bottom); in place."""
    kmin, kmax = g.kmin, g.kmax
    sfx = "_pl" if pole else ""
    GS = getattr(g, "VMTR_GSGAM2" + sfx)
    C2W = getattr(g, "VMTR_C2Wfact" + sfx)
    C2WGz = getattr(g, "VMTR_C2WfactGz" + sfx)
    PHI = getattr(g, "VMTR_PHI" + sfx)
    tem = DIAG[..., I_tem]
    pre = DIAG[..., I_pre]
    K = lambda a, k: _kidx(a, k)
    tem_top = K(tem, kmax).copy()
    tem_btm = K(tem, kmin).copy()
    pre_top = K(pre, kmax - 1) - K(rho, kmax) * (K(PHI, kmax + 1) - K(PHI, kmax - 1))
    pre_btm = K(pre, kmin + 1) - K(rho, kmin) * (K(PHI, kmin - 1) - K(PHI, kmin + 1))
    rho_top = pre_top / (g.Rdry * tem_top)
    rho_btm = pre_btm / (g.Rdry * tem_btm)
    _kset(tem, kmax + 1, tem_top); _kset(tem, kmin - 1, tem_btm)
    _kset(pre, kmax + 1, pre_top); _kset(pre, kmin - 1, pre_btm)
    _kset(rho, kmax + 1, rho_top); _kset(rho, kmin - 1, rho_btm)
    rhog = PROG[..., I_RHOG]
    _kset(rhog, kmax + 1, K(rho, kmax + 1) * K(GS, kmax + 1))
    _kset(rhog, kmin - 1, K(rho, kmin - 1) * K(GS, kmin - 1))
    _kset(ein, kmax + 1, g.CVdry * K(tem, kmax + 1))
    _kset(ein, kmin - 1, g.CVdry * K(tem, kmin - 1))
    _kset(PROG[..., I_RHOGE], kmax + 1, K(rhog, kmax + 1) * K(ein, kmax + 1))
    _kset(PROG[..., I_RHOGE], kmin - 1, K(rhog, kmin - 1) * K(ein, kmin - 1))
    # momentum: FREE top (sgn +1), RIGID bottom (sgn -1)
    for iv in (I_RHOGVX, I_RHOGVY, I_RHOGVZ):
        v = PROG[..., iv]
        top = 1.0 * (K(v, kmax) / K(rhog, kmax)) * K(rhog, kmax + 1)
        btm = -1.0 * (K(v, kmin) / K(rhog, kmin)) * K(rhog, kmin - 1)
        _kset(v, kmax + 1, top)
        _kset(v, kmin - 1, btm)
    for kk in (kmax + 1, kmin - 1):
        for iv, idg in ((I_RHOGVX, I_vx), (I_RHOGVY, I_vy), (I_RHOGVZ, I_vz)):
            _kset(DIAG[..., idg], kk, K(PROG[..., iv], kk) / K(rhog, kk))
    rw = PROG[..., I_RHOGW]
    vx, vy, vz = PROG[..., I_RHOGVX], PROG[..., I_RHOGVY], PROG[..., I_RHOGVZ]
    cz = lambda k, c: K(C2WGz[..., c], k)
    rw_top = -(cz(kmax + 1, 0) * K(vx, kmax + 1) + cz(kmax + 1, 1) * K(vx, kmax)
               + cz(kmax + 1, 2) * K(vy, kmax + 1) + cz(kmax + 1, 3) * K(vy, kmax)
               + cz(kmax + 1, 4) * K(vz, kmax + 1) + cz(kmax + 1, 5) * K(vz, kmax))
    _kset(rw, kmax + 1, rw_top)
    _kset(rw, kmin, np.zeros_like(K(rw, kmin)))
    _kset(rw, kmin - 1, 0.0)
    w = DIAG[..., I_w]
    _kset(w, kmax + 1, K(rw, kmax + 1) / (K(C2W[..., 0], kmax + 1) * K(rhog, kmax + 1)
                                          + K(C2W[..., 1], kmax + 1) * K(rhog, kmax)))
    _kset(w, kmin, K(rw, kmin) / (K(C2W[..., 0], kmin) * K(rhog, kmin)
                                  + K(C2W[..., 1], kmin) * K(rhog, kmin - 1)))
    _kset(w, kmin - 1, 0.0)


# --------------------------------------------------------------------------
# horizontal operators (kernels/oprt*.py)
# --------------------------------------------------------------------------
def _pad2(inner, i, j, lo=1):
    out = np.zeros((i, j) + inner.shape[2:], inner.dtype)
    out[lo:lo + inner.shape[0], lo:lo + inner.shape[1]] = inner
    return out


def divergence(g, vx, vy, vz):
    """kernels/fluxconv.py:52-78 (coef_div 7-point, zero border)."""
    i, j = vx.shape[:2]
    c = g.OPRT_coef_div[1:i - 1, 1:j - 1]

    def st(v, d):
        return (c[..., d, 0] * v[1:i - 1, 1:j - 1] + c[..., d, 1] * v[2:i, 1:j - 1]
                + c[..., d, 2] * v[2:i, 2:j] + c[..., d, 3] * v[1:i - 1, 2:j]
                + c[..., d, 4] * v[0:i - 2, 1:j - 1] + c[..., d, 5] * v[0:i - 2, 0:j - 2]
                + c[..., d, 6] * v[1:i - 1, 0:j - 2])
    return _pad2(st(vx, XDIR) + st(vy, YDIR) + st(vz, ZDIR), i, j)


def divergence_pl(g, vx, vy, vz):
    """kernels/fluxconv.py:81-108: only the pole row, summed over v = 0..5."""
    c = g.OPRT_coef_div_pl
    per_v = (c[:, 0, :, XDIR][:, None, :] * vx + c[:, 0, :, YDIR][:, None, :] * vy
             + c[:, 0, :, ZDIR][:, None, :] * vz)
    out = np.zeros_like(vx)
    out[0] = per_v.sum(axis=0)
    return out


def gradient(g, s):
    """kernels/oprtgradient.py:45-70 (and presgrad.py:64-97), returns (i,j,k,l,3)."""
    i, j = s.shape[:2]
    stk = np.stack([s[1:i - 1, 1:j - 1], s[2:i, 1:j - 1], s[2:i, 2:j], s[1:i - 1, 2:j],
                    s[0:i - 2, 1:j - 1], s[0:i - 2, 0:j - 2], s[1:i - 1, 0:j - 2]], axis=4)
    cg = g.OPRT_coef_grad[1:i - 1, 1:j - 1]
    comps = [np.sum(cg[..., d, :] * stk, axis=4) for d in (XDIR, YDIR, ZDIR)]
    return _pad2(np.stack(comps, axis=4), i, j)


def gradient_pl(g, s_pl):
    """kernels/oprtgradient.py:73-88: pole row, per-direction sequential sum."""
    cg = g.OPRT_coef_grad_pl[:, 0]                       # (6, l, 3)
    row = (cg[:, None, :, :] * s_pl[..., None]).sum(axis=0)
    out = np.zeros(s_pl.shape + (3,))
    out[0] = row
    return out


def laplacian(g, s):
    """kernels/oprtlaplacian.py:41-55."""
    i, j = s.shape[:2]
    c = g.OPRT_coef_lap[1:i - 1, 1:j - 1]
    inner = (c[..., 0] * s[1:i - 1, 1:j - 1] + c[..., 1] * s[2:i, 1:j - 1]
             + c[..., 2] * s[2:i, 2:j] + c[..., 3] * s[1:i - 1, 2:j]
             + c[..., 4] * s[0:i - 2, 1:j - 1] + c[..., 5] * s[0:i - 2, 0:j - 2]
             + c[..., 6] * s[1:i - 1, 0:j - 2])
    return _pad2(inner, i, j)


def laplacian_pl(g, s_pl):
    """kernels/oprtlaplacian.py:58-70."""
    out = np.zeros_like(s_pl)
    out[0] = (g.OPRT_coef_lap_pl * s_pl).sum(axis=0)
    return out


def _sgp_corner(g, tTI, tTJ):
    """singular-point fix at the (0,0) vertex (kernels/oprtdiffusion.py:91-96)."""
    fdt = tTI.dtype
    m0 = g.pntmask[0, :, 0].astype(fdt)
    m1 = g.pntmask[0, :, 1].astype(fdt)
    m0 = m0.reshape((1, 1, 1, -1) + (1,) * (tTI.ndim - 4))
    m1 = m1.reshape((1, 1, 1, -1) + (1,) * (tTI.ndim - 4))
    tTI = tTI.copy()
    tTI[0:1, 0:1] = tTI[0:1, 0:1] * m0 + tTJ[1:2, 0:1] * m1
    return tTI


def diffusion(g, s, kh):
    """kernels/oprtdiffusion.py:59-134."""
    i, j = s.shape[:2]
    gmin, gmax = g.gmin, g.gmax
    bi, bj, bip, bjp = slice(0, i - 1), slice(0, j - 1), slice(1, i), slice(1, j)
    s0 = s[bi, bj][..., None]
    s_ip = s[bip, bj][..., None]
    s_d = s[bip, bjp][..., None]
    s_jp = s[bi, bjp][..., None]
    cti = g.OPRT_coef_intp[bi, bj, :, :, :, :, TI]
    ctj = g.OPRT_coef_intp[bi, bj, :, :, :, :, TJ]
    c1i, c2i, c3i = cti[..., 0], cti[..., 1], cti[..., 2]
    c1j, c2j, c3j = ctj[..., 0], ctj[..., 1], ctj[..., 2]
    tTI = ((2.0 * c1i - c2i - c3i) * s0 + (-c1i + 2.0 * c2i - c3i) * s_ip
           + (-c1i - c2i + 2.0 * c3i) * s_d) / 3.0
    tTJ = ((2.0 * c1j - c2j - c3j) * s0 + (-c1j + 2.0 * c2j - c3j) * s_d
           + (-c1j - c2j + 2.0 * c3j) * s_jp) / 3.0
    tTI = _sgp_corner(g, tTI, tTJ)
    sl, slp, slm = slice(gmin, gmax + 1), slice(gmin + 1, gmax + 2), slice(gmin - 1, gmax)
    kh0 = kh[sl, sl]
    kf = [0.5 * (kh0 + kh[slp, slp]), 0.5 * (kh0 + kh[sl, slp]), 0.5 * (kh0 + kh[slm, sl]),
          0.5 * (kh0 + kh[slm, slm]), 0.5 * (kh0 + kh[sl, slm]), 0.5 * (kh0 + kh[slp, sl])]
    II, IIm = slice(gmin, gmax + 1), slice(gmin - 1, gmax)
    a_ti, a_tj = tTI[II, II], tTJ[II, II]
    b_ti = tTI[IIm, II]
    c_tj, c_ti = tTJ[IIm, IIm], tTI[IIm, IIm]
    d_tj = tTJ[II, IIm]
    inner = None
    for d in range(3):
        cd = g.OPRT_coef_diff[II, II, :, :, d, :]
        blk = (kf[0] * cd[..., 0] * (a_ti[..., d] + a_tj[..., d])
               + kf[1] * cd[..., 1] * (a_tj[..., d] + b_ti[..., d])
               + kf[2] * cd[..., 2] * (b_ti[..., d] + c_tj[..., d])
               + kf[3] * cd[..., 3] * (c_tj[..., d] + c_ti[..., d])
               + kf[4] * cd[..., 4] * (c_ti[..., d] + d_tj[..., d])
               + kf[5] * cd[..., 5] * (d_tj[..., d] + a_ti[..., d]))
        inner = blk if inner is None else inner + blk
    return _pad2(inner, i, j, lo=gmin)


def diffusion_pl(g, s_pl, kh_pl):
    """kernels/oprtdiffusion.py:137-177."""
    sv = s_pl[1:6]
    svp1 = np.roll(sv, -1, axis=0)
    cI = g.OPRT_coef_intp_pl[1:6, 0]                     # (5, l, 3, 3)
    c0 = cI[..., 0][:, None]
    c1 = cI[..., 1][:, None]
    c2 = cI[..., 2][:, None]
    vt = ((2.0 * c0 - c1 - c2) * s_pl[0][None, :, :, None] + (-c0 + 2.0 * c1 - c2) * sv[..., None]
          + (-c0 - c1 + 2.0 * c2) * svp1[..., None]) / 3.0
    vsum = np.roll(vt, 1, axis=0) + vt
    kh_avg = 0.5 * (kh_pl[0][None] + kh_pl[1:6])
    cd = g.OPRT_coef_diff_pl[1:6, 0][:, None]
    contrib = kh_avg * (cd * vsum).sum(axis=-1)
    out = np.zeros_like(s_pl)
    out[0] = contrib.sum(axis=0)
    return out


def horizontalize(g, vx, vy, vz):
    """kernels/horizontalizevec.py:34-55; interior only, border kept (in place)."""
    i, j = vx.shape[:2]
    gv = g.GRD_x[1:i - 1, 1:j - 1, 0]
    gx, gy, gz = (gv[..., d][:, :, None, :] for d in (XDIR, YDIR, ZDIR))
    r = g.rscale
    sx, sy, sz = vx[1:i - 1, 1:j - 1], vy[1:i - 1, 1:j - 1], vz[1:i - 1, 1:j - 1]
    prd = (sx * gx + sy * gy + sz * gz) / r
    nx = sx - prd * gx / r
    ny = sy - prd * gy / r
    nz = sz - prd * gz / r
    vx[1:i - 1, 1:j - 1] = nx
    vy[1:i - 1, 1:j - 1] = ny
    vz[1:i - 1, 1:j - 1] = nz


def horizontalize_pl(g, vx, vy, vz):
    """kernels/horizontalizevec.py:58-71 (in place)."""
    gx, gy, gz = (g.GRD_x_pl[:, 0, :, d][:, None, :] for d in (XDIR, YDIR, ZDIR))
    r = g.rscale
    prd = vx * gx / r + vy * gy / r + vz * gz / r
    nx = vx - prd * gx / r
    ny = vy - prd * gy / r
    nz = vz - prd * gz / r
    vx[...] = nx
    vy[...] = ny
    vz[...] = nz


def _sclt(g, c, vx, vy, vz, R, Rp1):
    """sclt_TI / sclt_TJ of kernels/oprtdivdamp.py:73-94."""
    ti = (c[..., XDIR, 0, TI] * vx[R, R] + c[..., XDIR, 1, TI] * vx[Rp1, R] + c[..., XDIR, 2, TI] * vx[Rp1, Rp1]
          + c[..., YDIR, 0, TI] * vy[R, R] + c[..., YDIR, 1, TI] * vy[Rp1, R] + c[..., YDIR, 2, TI] * vy[Rp1, Rp1]
          + c[..., ZDIR, 0, TI] * vz[R, R] + c[..., ZDIR, 1, TI] * vz[Rp1, R] + c[..., ZDIR, 2, TI] * vz[Rp1, Rp1])
    tj = (c[..., XDIR, 0, TJ] * vx[R, R] + c[..., XDIR, 1, TJ] * vx[Rp1, Rp1] + c[..., XDIR, 2, TJ] * vx[R, Rp1]
          + c[..., YDIR, 0, TJ] * vy[R, R] + c[..., YDIR, 1, TJ] * vy[Rp1, Rp1] + c[..., YDIR, 2, TJ] * vy[R, Rp1]
          + c[..., ZDIR, 0, TJ] * vz[R, R] + c[..., ZDIR, 1, TJ] * vz[Rp1, Rp1] + c[..., ZDIR, 2, TJ] * vz[R, Rp1])
    return ti, tj


def _ddivd(g, sTI, sTJ, d):
    G = g.gmax + 1
    II, IIm = slice(1, G), slice(0, G - 1)
    a_ti, a_tj = sTI[II, II], sTJ[II, II]
    b_ti = sTI[IIm, II]
    c_tj, c_ti = sTJ[IIm, IIm], sTI[IIm, IIm]
    d_tj = sTJ[II, IIm]
    cd = g.OPRT_coef_diff[II, II, :, :, d, :]
    return (cd[..., 0] * (a_ti + a_tj) + cd[..., 1] * (a_tj + b_ti) + cd[..., 2] * (b_ti + c_tj)
            + cd[..., 3] * (c_tj + c_ti) + cd[..., 4] * (c_ti + d_tj) + cd[..., 5] * (d_tj + a_ti))


def divdamp(g, vx, vy, vz):
    """kernels/oprtdivdamp.py:54-122 -> (dx, dy, dz)."""
    i, j = vx.shape[:2]
    G = g.gmax + 1
    R, Rp1 = slice(0, G), slice(1, G + 1)
    c = g.OPRT_coef_intp[R, R]
    sTI, sTJ = _sclt(g, c, vx, vy, vz, R, Rp1)
    return [_pad2(_ddivd(g, sTI, sTJ, d), i, j) for d in (XDIR, YDIR, ZDIR)]


def divdamp_pl(g, vx, vy, vz):
    """kernels/oprtdivdamp.py:125-173."""
    sx, sy, sz = vx[0], vy[0], vz[0]
    ijx, ijy, ijz = vx[1:6], vy[1:6], vz[1:6]
    px, py, pz = np.roll(ijx, -1, 0), np.roll(ijy, -1, 0), np.roll(ijz, -1, 0)
    cI = g.OPRT_coef_intp_pl[1:6, 0]
    b = lambda a: a[:, None, :]
    sclt = (b(cI[:, :, XDIR, 0]) * sx + b(cI[:, :, XDIR, 1]) * ijx + b(cI[:, :, XDIR, 2]) * px
            + b(cI[:, :, YDIR, 0]) * sy + b(cI[:, :, YDIR, 1]) * ijy + b(cI[:, :, YDIR, 2]) * py
            + b(cI[:, :, ZDIR, 0]) * sz + b(cI[:, :, ZDIR, 1]) * ijz + b(cI[:, :, ZDIR, 2]) * pz)
    pair = np.roll(sclt, 1, 0) + sclt
    cd = g.OPRT_coef_diff_pl[1:6, 0]
    outs = []
    for d in (XDIR, YDIR, ZDIR):
        o = np.zeros_like(vx)
        o[0] = (b(cd[:, :, d]) * pair).sum(axis=0)
        outs.append(o)
    return outs


def _rhogw_vm(g, vx, vy, vz, w, pole=False):
    """kernels/oprt3ddivdamp.py:50-82 (== fluxconv rhogw_vmh with vflag 1)."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    cz = getattr(g, "VMTR_C2WfactGz" + sfx)
    RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
    RGSQRTH = getattr(g, "VMTR_RGSQRTH" + sfx)
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    K = (lambda a, s: a[:, :, s]) if not pole else (lambda a, s: a[:, s])
    horiz = (K(cz, ks)[..., 0] * K(vx, ks) + K(cz, ks)[..., 1] * K(vx, km)
             + K(cz, ks)[..., 2] * K(vy, ks) + K(cz, ks)[..., 3] * K(vy, km)
             + K(cz, ks)[..., 4] * K(vz, ks) + K(cz, ks)[..., 5] * K(vz, km))
    out = np.zeros_like(w)
    if pole:
        out[:, ks] = horiz * RGAMH[:, ks] + w[:, ks] * RGSQRTH[:, ks]
    else:
        out[:, :, ks] = horiz * RGAMH[:, :, ks] + w[:, :, ks] * RGSQRTH[:, :, ks]
    return out


def divdamp3d(g, rvx, rvy, rvz, rw):
    """kernels/oprt3ddivdamp.py:85-173."""
    i, j, kall = rvx.shape[:3]
    kmin, kmax = g.kmin, g.kmax
    G = g.gmax + 1
    rwv = _rhogw_vm(g, rvx, rvy, rvz, rw)
    K = slice(kmin, kmax + 1)
    RG = g.VMTR_RGAM[:, :, K]
    vmx, vmy, vmz = rvx[:, :, K] * RG, rvy[:, :, K] * RG, rvz[:, :, K] * RG
    R, Rp1 = slice(0, G), slice(1, G + 1)
    UP, DN = slice(kmin + 1, kmax + 2), slice(kmin, kmax + 1)
    rdz = g.GRD_rdgz[K][None, None, :, None]
    wTI = ((rwv[R, R, UP] + rwv[Rp1, R, UP] + rwv[Rp1, Rp1, UP])
           - (rwv[R, R, DN] + rwv[Rp1, R, DN] + rwv[Rp1, Rp1, DN])) / 3.0 * rdz
    wTJ = ((rwv[R, R, UP] + rwv[Rp1, Rp1, UP] + rwv[R, Rp1, UP])
           - (rwv[R, R, DN] + rwv[Rp1, Rp1, DN] + rwv[R, Rp1, DN])) / 3.0 * rdz
    c = g.OPRT_coef_intp[R, R]
    sTI, sTJ = _sclt(g, c, vmx, vmy, vmz, R, Rp1)
    sTI = sTI + wTI
    sTJ = sTJ + wTJ
    sTI = _sgp_corner(g, sTI, sTJ)
    outs = []
    for d in (XDIR, YDIR, ZDIR):
        o = np.zeros(rvx.shape)
        o[1:G, 1:G, K] = _ddivd(g, sTI, sTJ, d)
        outs.append(o)
    return outs


def divdamp3d_pl(g, rvx, rvy, rvz, rw):
    """kernels/oprt3ddivdamp.py:176-237."""
    kmin, kmax = g.kmin, g.kmax
    rwv = _rhogw_vm(g, rvx, rvy, rvz, rw, pole=True)
    K = slice(kmin, kmax + 1)
    RG = g.VMTR_RGAM_pl[:, K]
    vmx, vmy, vmz = rvx[:, K] * RG, rvy[:, K] * RG, rvz[:, K] * RG
    sx, sy, sz = vmx[0], vmy[0], vmz[0]
    ijx, ijy, ijz = vmx[1:6], vmy[1:6], vmz[1:6]
    px, py, pz = np.roll(ijx, -1, 0), np.roll(ijy, -1, 0), np.roll(ijz, -1, 0)
    UP, DN = slice(kmin + 1, kmax + 2), slice(kmin, kmax + 1)
    r_n_up, r_n_dn = rwv[0, UP], rwv[0, DN]
    r_ij_up, r_ij_dn = rwv[1:6, UP], rwv[1:6, DN]
    sclt_w = ((r_n_up + r_ij_up + np.roll(r_ij_up, -1, 0))
              - (r_n_dn + r_ij_dn + np.roll(r_ij_dn, -1, 0))) / 3.0 * g.GRD_rdgz[K][None, :, None]
    cI = g.OPRT_coef_intp_pl[1:6, 0]
    b = lambda a: a[:, None, :]
    sclt = (b(cI[:, :, XDIR, 0]) * sx + b(cI[:, :, XDIR, 1]) * ijx + b(cI[:, :, XDIR, 2]) * px
            + b(cI[:, :, YDIR, 0]) * sy + b(cI[:, :, YDIR, 1]) * ijy + b(cI[:, :, YDIR, 2]) * py
            + b(cI[:, :, ZDIR, 0]) * sz + b(cI[:, :, ZDIR, 1]) * ijz + b(cI[:, :, ZDIR, 2]) * pz
            + sclt_w)
    pair = np.roll(sclt, 1, 0) + sclt
    cd = g.OPRT_coef_diff_pl[1:6, 0]
    outs = []
    for d in (XDIR, YDIR, ZDIR):
        o = np.zeros_like(rvx)
        o[0, K] = (b(cd[:, :, d]) * pair).sum(axis=0)
        outs.append(o)
    return outs


# --------------------------------------------------------------------------
# source terms (kernels/advconv.py, fluxconv.py, presgrad.py, buoyancy.py)
# --------------------------------------------------------------------------
def flux_convergence(g, rvx, rvy, rvz, rw, vertical=True, pole=False):
    """kernels/fluxconv.py:111-208 (fluxtype default / horizontal)."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    RGAM = getattr(g, "VMTR_RGAM" + sfx)
    RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
    RGSQRTH = getattr(g, "VMTR_RGSQRTH" + sfx)
    cz_all = getattr(g, "VMTR_C2WfactGz" + sfx)
    vflag = 1.0 if vertical else 0.0
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    K = (lambda a, s: a[:, :, s]) if not pole else (lambda a, s: a[:, s])
    vxm, vym, vzm = rvx * RGAM, rvy * RGAM, rvz * RGAM
    cz = K(cz_all, ks)
    horiz = (cz[..., 0] * K(rvx, ks) + cz[..., 1] * K(rvx, km) + cz[..., 2] * K(rvy, ks)
             + cz[..., 3] * K(rvy, km) + cz[..., 4] * K(rvz, ks) + cz[..., 5] * K(rvz, km))
    horiz = horiz * K(RGAMH, ks)
    vert = vflag * K(rw, ks) * K(RGSQRTH, ks)
    vmh = np.zeros_like(rw)
    if pole:
        vmh[:, ks] = horiz + vert
        div = divergence_pl(g, vxm, vym, vzm)
    else:
        vmh[:, :, ks] = horiz + vert
        div = divergence(g, vxm, vym, vzm)
    kc, kcp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
    out = np.zeros_like(rw)
    if pole:
        rdz = g.GRD_rdgz[kc][None, :, None]
        out[:, kc] = -div[:, kc] - (vmh[:, kcp] - vmh[:, kc]) * rdz
    else:
        rdz = g.GRD_rdgz[kc][None, None, :, None]
        out[:, :, kc] = -div[:, :, kc] - (vmh[:, :, kcp] - vmh[:, :, kc]) * rdz
    return out


def scaled_fluxes(g, rvx, rvy, rvz, rw, scl, vertical=True, pole=False):
    """kernels/advconv.py:42-108."""
    kmin, kmax = g.kmin, g.kmax
    sx, sy, sz = rvx * scl, rvy * scl, rvz * scl
    sw = np.zeros_like(rw)
    if vertical:
        af = g.GRD_afact[kmin:kmax + 2]
        bf = g.GRD_bfact[kmin:kmax + 2]
        if pole:
            sw[:, kmin:kmax + 2] = rw[:, kmin:kmax + 2] * (af[None, :, None] * scl[:, kmin:kmax + 2]
                                                           + bf[None, :, None] * scl[:, kmin - 1:kmax + 1])
        else:
            sw[:, :, kmin:kmax + 2] = rw[:, :, kmin:kmax + 2] * (
                af[None, None, :, None] * scl[:, :, kmin:kmax + 2]
                + bf[None, None, :, None] * scl[:, :, kmin - 1:kmax + 1])
    return sx, sy, sz, sw


def advection_convergence(g, rvx, rvy, rvz, rw, scl, vertical=True, pole=False):
    """mod_src.py:499-623 = scaled fluxes then flux convergence."""
    sx, sy, sz, sw = scaled_fluxes(g, rvx, rvy, rvz, rw, scl, vertical, pole)
    return flux_convergence(g, sx, sy, sz, sw, vertical, pole)


def pres_gradient(g, P, P_pl, vertical=True):
    """kernels/presgrad.py:126-265 with first_layer_remedy and horizontalize."""
    kmin, kmax = g.kmin, g.kmax
    i, j, kall, l = P.shape
    out = []
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        PP = P_pl if pole else P
        RGAM = getattr(g, "VMTR_RGAM" + sfx)
        RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
        czall = getattr(g, "VMTR_C2WfactGz" + sfx)
        if pole:
            Pvm = PP * RGAM * 1.0      # * plmask (== 1 here)
            gh = gradient_pl(g, Pvm)
            K = lambda a, s: a[:, s]
        else:
            Pvm = PP * RGAM
            gh = gradient(g, Pvm)
            K = lambda a, s: a[:, :, s]
        cz = K(czall, slice(kmin, kmax + 2))
        rgh = K(RGAMH, slice(kmin, kmax + 2))
        Pk = K(PP, slice(kmin, kmax + 2))
        Pkm1 = K(PP, slice(kmin - 1, kmax + 1))
        pvmh = np.stack([(cz[..., 0] * Pk + cz[..., 1] * Pkm1) * rgh,
                         (cz[..., 2] * Pk + cz[..., 3] * Pkm1) * rgh,
                         (cz[..., 4] * Pk + cz[..., 5] * Pkm1) * rgh], axis=-1)
        if pole:
            rdz = g.GRD_rdgz[kmin:kmax + 1][None, :, None, None]
            vterm = (pvmh[:, 1:] - pvmh[:, :-1]) * rdz
            gf = gh[:, kmin:kmax + 1] + vterm
            Pg = gh.copy()
            Pg[:, kmin - 1] = 0.0
            Pg[:, kmin] = gf[:, 1]
            Pg[:, kmin + 1:kmax + 1] = gf[:, 1:]
            Pg[:, kmax + 1] = 0.0
            horizontalize_pl(g, Pg[..., 0], Pg[..., 1], Pg[..., 2])
        else:
            rdz = g.GRD_rdgz[kmin:kmax + 1][None, None, :, None, None]
            vterm = (pvmh[:, :, 1:] - pvmh[:, :, :-1]) * rdz
            gf = gh[:, :, kmin:kmax + 1] + vterm
            Pg = gh.copy()
            Pg[:, :, kmin - 1] = 0.0
            Pg[:, :, kmin] = gf[:, :, 1]
            Pg[:, :, kmin + 1:kmax + 1] = gf[:, :, 1:]
            Pg[:, :, kmax + 1] = 0.0
            Pgx, Pgy, Pgz = Pg[..., 0].copy(), Pg[..., 1].copy(), Pg[..., 2].copy()
            horizontalize(g, Pgx, Pgy, Pgz)
            Pg = np.stack([Pgx, Pgy, Pgz], axis=-1)
        Pgw = np.zeros_like(PP)
        if vertical:
            GAM2H = getattr(g, "VMTR_GAM2H" + sfx)
            RGSGAM2 = getattr(g, "VMTR_RGSGAM2" + sfx)
            ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
            if pole:
                rdh = g.GRD_rdgzh[ks][None, :, None]
                Pgw[:, ks] = GAM2H[:, ks] * (PP[:, ks] * RGSGAM2[:, ks] - PP[:, km] * RGSGAM2[:, km]) * rdh
            else:
                rdh = g.GRD_rdgzh[ks][None, None, :, None]
                Pgw[:, :, ks] = GAM2H[:, :, ks] * (PP[:, :, ks] * RGSGAM2[:, :, ks]
                                                   - PP[:, :, km] * RGSGAM2[:, :, km]) * rdh
        out += [Pg, Pgw]
    return out            # Pgrad, Pgradw, Pgrad_pl, Pgradw_pl


def buoyancy(g, rhog, pole=False):
    """kernels/buoyancy.py:40-81."""
    sfx = "_pl" if pole else ""
    C2W = getattr(g, "VMTR_C2Wfact" + sfx)
    kmin, kmax = g.kmin, g.kmax
    out = np.zeros_like(rhog)
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    if pole:
        out[:, ks] = -g.GRAV * (C2W[:, ks, :, 0] * rhog[:, ks] + C2W[:, ks, :, 1] * rhog[:, km])
    else:
        out[:, :, ks] = -g.GRAV * (C2W[:, :, ks, :, 0] * rhog[:, :, ks] + C2W[:, :, ks, :, 1] * rhog[:, :, km])
    return out


def advection_momentum(g, DIAG, PROG, DIAG_pl, PROG_pl):
    """mod_src.py:96-497 with kernels/advconvmom.py (sphere).  Returns
    (gvx, gvy, gvz, gw) regional and pole."""
    kmin, kmax = g.kmin, g.kmax
    res = []
    for pole in (False, True):
        D = DIAG_pl if pole else DIAG
        P = PROG_pl if pole else PROG
        gx = (g.GRD_x_pl[:, 0] if pole else g.GRD_x[:, :, 0])
        gxs = [gx[..., d] for d in (XDIR, YDIR, ZDIR)]
        kc, kp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
        cf, df = g.GRD_cfact[kc], g.GRD_dfact[kc]
        w = D[..., I_w]
        if pole:
            wc = cf[None, :, None] * w[:, kp] + df[None, :, None] * w[:, kc]
            gb = [a[:, None, :] for a in gxs]
        else:
            wc = cf[None, None, :, None] * w[:, :, kp] + df[None, None, :, None] * w[:, :, kc]
            gb = [a[:, :, None, :] for a in gxs]
        vv = []
        for idg, gd in zip((I_vx, I_vy, I_vz), gb):
            a = np.zeros_like(w)
            if pole:
                a[:, kc] = D[:, kc, :, idg] + (wc * gd / g.rscale)
            else:
                a[:, :, kc] = D[:, :, kc, :, idg] + wc * gd / g.rscale
            vv.append(a)
        rvx, rvy, rvz, rw = P[..., I_RHOGVX], P[..., I_RHOGVY], P[..., I_RHOGVZ], P[..., I_RHOGW]
        dv = [advection_convergence(g, rvx, rvy, rvz, rw, s, True, pole) for s in vv]
        Kc = (lambda a: a[:, kc]) if pole else (lambda a: a[:, :, kc])
        rh = Kc(P[..., I_RHOG])
        dvx = Kc(dv[0]) - (-2.0 * rh * (g.OHM * Kc(vv[1])))
        dvy = Kc(dv[1]) - (2.0 * rh * (g.OHM * Kc(vv[0])))
        dvz = Kc(dv[2])
        gg = [a / g.rscale for a in gb]
        prd = dvx * gg[0] + dvy * gg[1] + dvz * gg[2]
        outs = [np.zeros_like(w) for _ in range(4)]
        gwc = prd * g.alpha
        C2W = g.VMTR_C2Wfact_pl if pole else g.VMTR_C2Wfact
        ks = slice(kmin + 1, kmax + 1)
        if pole:
            outs[0][:, kc] = dvx - prd * gg[0]
            outs[1][:, kc] = dvy - prd * gg[1]
            outs[2][:, kc] = dvz - prd * gg[2]
            outs[3][:, ks] = C2W[:, ks, :, 0] * gwc[:, 1:] + C2W[:, ks, :, 1] * gwc[:, :-1]
        else:
            outs[0][:, :, kc] = dvx - prd * gg[0]
            outs[1][:, :, kc] = dvy - prd * gg[1]
            outs[2][:, :, kc] = dvz - prd * gg[2]
            outs[3][:, :, ks] = C2W[:, :, ks, :, 0] * gwc[:, :, 1:] + C2W[:, :, ks, :, 1] * gwc[:, :, :-1]
        res.append(outs)
    return res


# --------------------------------------------------------------------------
# numerical filters (mod_numfilter.py)
# --------------------------------------------------------------------------
def hdiffusion(g, rhog, rho, DIAG, rhog_pl, rho_pl, DIAG_pl):
    """mod_numfilter.py:845-1469 (DIRECT, lap_order 2, tracer part off) with
    _hdiff_tendency_host :1519-1578 and the final horizontalize.  Returns
    f_TEND (i,j,k,l,6) and f_TEND_pl."""
    kmin, kmax = g.kmin, g.kmax
    Kh = g.Kh_coef
    rhog_h = np.zeros_like(rhog)
    rhog_h[:, :, kmin:kmax + 2] = (g.VMTR_C2Wfact[:, :, kmin:kmax + 2, :, 0] * rhog[:, :, kmin:kmax + 2]
                                   + g.VMTR_C2Wfact[:, :, kmin:kmax + 2, :, 1] * rhog[:, :, kmin - 1:kmax + 1])
    rhog_h[:, :, kmin - 1] = 0.0
    rhog_h_pl = np.zeros_like(rhog_pl)
    rhog_h_pl[:, kmin:kmax + 2] = (g.VMTR_C2Wfact_pl[:, kmin:kmax + 2, :, 0] * rhog_pl[:, kmin:kmax + 2]
                                   + g.VMTR_C2Wfact_pl[:, kmin:kmax + 2, :, 1] * rhog_pl[:, kmin - 1:kmax + 1])
    rhog_h_pl[:, kmin - 1] = 0.0
    vt = np.stack([DIAG[..., I_vx], DIAG[..., I_vy], DIAG[..., I_vz], DIAG[..., I_w],
                   DIAG[..., I_tem] - g.tem_bs, rho - g.rho_bs], axis=-1)
    vtp = np.stack([DIAG_pl[..., I_vx], DIAG_pl[..., I_vy], DIAG_pl[..., I_vz], DIAG_pl[..., I_w],
                    DIAG_pl[..., I_tem] - g.tem_bs_pl, rho_pl - g.rho_bs_pl], axis=-1)
    KhA = np.full(rhog.shape, Kh)
    KhA_pl = np.full(rhog_pl.shape, Kh)
    KhH, KhH_pl = KhA, KhA_pl
    nonlinear = "hdiff_nl_kh_max" in g.d
    for p in range(2):
        v2 = np.zeros_like(vt)
        v2p = np.zeros_like(vtp)
        for n in range(4):
            v2[..., n] = laplacian(g, vt[..., n])
            v2p[..., n] = laplacian_pl(g, vtp[..., n])
        if p == 1:
            if nonlinear:
                KhA, KhA_pl = hdiff_nonlinear_coef(g, vt[..., 4], vtp[..., 4])
                KhH, KhH_pl = hdiff_nonlinear_coef_h(g, KhA), hdiff_nonlinear_coef_h(g, KhA_pl, pole=True)
            wk = rhog * g.CVdry * KhA
            wkp = rhog_pl * g.CVdry * KhA_pl
            v2[..., 4] = diffusion(g, vt[..., 4], wk)
            v2p[..., 4] = diffusion_pl(g, vtp[..., 4], wkp)
            wk = rhog * g.hdiff_fact_rho * KhA
            wkp = rhog_pl * g.hdiff_fact_rho * KhA_pl
            v2[..., 5] = diffusion(g, vt[..., 5], wk)
            v2p[..., 5] = diffusion_pl(g, vtp[..., 5], wkp)
        else:
            v2[..., 4] = laplacian(g, vt[..., 4])
            v2p[..., 4] = laplacian_pl(g, vtp[..., 4])
            v2[..., 5] = laplacian(g, vt[..., 5])
            v2p[..., 5] = laplacian_pl(g, vtp[..., 5])
        vt = -v2
        vtp = -v2p
        comm(g, vt, vtp)
    f = np.zeros(rhog.shape + (6,))
    fp = np.zeros(rhog_pl.shape + (6,))
    zero = 0.0 * 0.0
    for (F, V, RG, RGH, KA, KH) in ((f, vt, rhog, rhog_h, KhA, KhH), (fp, vtp, rhog_pl, rhog_h_pl, KhA_pl, KhH_pl)):
        F[..., I_RHOGVX] = -(V[..., 0] * KA + zero) * RG
        F[..., I_RHOGVY] = -(V[..., 1] * KA + zero) * RG
        F[..., I_RHOGVZ] = -(V[..., 2] * KA + zero) * RG
        F[..., I_RHOGW] = -(V[..., 3] * KH + zero) * RGH
        F[..., I_RHOGE] = -(V[..., 4] + zero)
        F[..., I_RHOG] = -(V[..., 5] + zero)
    a, b, c = f[..., I_RHOGVX].copy(), f[..., I_RHOGVY].copy(), f[..., I_RHOGVZ].copy()
    horizontalize(g, a, b, c)
    f[..., I_RHOGVX], f[..., I_RHOGVY], f[..., I_RHOGVZ] = a, b, c
    a, b, c = fp[..., I_RHOGVX].copy(), fp[..., I_RHOGVY].copy(), fp[..., I_RHOGVZ].copy()
    horizontalize_pl(g, a, b, c)
    fp[..., I_RHOGVX], fp[..., I_RHOGVY], fp[..., I_RHOGVZ] = a, b, c
    return f, fp


def hdiff_nonlinear_coef(g, lapT, lapT_pl):
    """mod_numfilter.py:1153-1184 (hdiff_type NONLINEAR1): Kh from the
    temperature-deviation Laplacian after the first Laplacian pass,
    cfact AREA^2 / dt * |lapT| / T0 * AREA with cfact 2, T0 300 K, clipped to
    [Kh_coef_minlim, kh_max(k)] (kh_max from height_factor, mod_numfilter.py:
    832-843, 920-922).  Returns Kh (i,j,k,l) and pole."""
    A, lo, hi = float(g.hdiff_nl_area), float(g.hdiff_nl_minlim), np.asarray(g.hdiff_nl_kh_max)
    c1 = 2.0 * (A ** 2) / g.dtl
    kh = np.clip(c1 * (np.abs(lapT) / 300.0 * A), lo, hi[None, None, :, None])
    kh_pl = np.clip(c1 * (np.abs(lapT_pl) / 300.0 * A), lo, hi[None, :, None])
    return kh, kh_pl


def hdiff_nonlinear_coef_h(g, kh, pole=False):
    """mod_numfilter.py:1186-1206: the half-level average of the nonlinear Kh
    on kmin+1..kmax, zero at kmin-1, kmin and kmax+1"""
    kmin, kmax = g.kmin, g.kmax
    out = np.zeros_like(kh)
    if pole:
        out[:, kmin + 1:kmax + 1] = 0.5 * (kh[:, kmin + 1:kmax + 1] + kh[:, kmin:kmax])
    else:
        out[:, :, kmin + 1:kmax + 1] = 0.5 * (kh[:, :, kmin + 1:kmax + 1] + kh[:, :, kmin:kmax])
    return out


def rayleigh_damping(g, f, fp, rhog, rhog_pl, DIAG, DIAG_pl):
    """mod_numfilter.py:240-271 numfilter_rayleigh_damping on the
    hyperdiffusion tendency (in place): the momentum tendencies lose
    rayleigh_coef(k) rhog v (unless only w is damped), the w tendency
    rayleigh_coef_h(k) w (C2Wa rhog(k) + C2Wb rhog(k-1)), rhog(-1) = 0."""
    rc, rch = np.asarray(g.rayleigh_coef), np.asarray(g.rayleigh_coef_h)
    if not int(g.rayleigh_only_w):
        coef = rc[None, None, :, None] * rhog
        for n, v in ((I_RHOGVX, I_vx), (I_RHOGVY, I_vy), (I_RHOGVZ, I_vz)):
            f[..., n] -= coef * DIAG[..., v]
        coef_pl = rc[None, :, None] * rhog_pl
        for n, v in ((I_RHOGVX, I_vx), (I_RHOGVY, I_vy), (I_RHOGVZ, I_vz)):
            fp[..., n] -= coef_pl * DIAG_pl[..., v]
    km1 = np.zeros_like(rhog)
    km1[:, :, 1:] = rhog[:, :, :-1]
    f[..., I_RHOGW] -= rch[None, None, :, None] * DIAG[..., I_w] * (
        g.VMTR_C2Wfact[..., 0] * rhog + g.VMTR_C2Wfact[..., 1] * km1)
    km1p = np.zeros_like(rhog_pl)
    km1p[:, 1:] = rhog_pl[:, :-1]
    fp[..., I_RHOGW] -= rch[None, :, None] * DIAG_pl[..., I_w] * (
        g.VMTR_C2Wfact_pl[..., 0] * rhog_pl + g.VMTR_C2Wfact_pl[..., 1] * km1p)


def numfilter_divdamp(g, rvx, rvy, rvz, rw, rvx_pl, rvy_pl, rvz_pl, rw_pl):
    """mod_numfilter.py:2032-2268 (lap_order 2: 3-D divdamp, COMM, post-COMM
    island kernels/divdamppostcomm.py:29-81).  Returns gd(x,y,z) and pole."""
    d = divdamp3d(g, rvx, rvy, rvz, rw)
    dp = divdamp3d_pl(g, rvx_pl, rvy_pl, rvz_pl, rw_pl)
    v2 = np.stack(d, axis=-1)
    v2p = np.stack(dp, axis=-1)
    comm(g, v2, v2p)
    o = divdamp(g, -v2[..., 0], -v2[..., 1], -v2[..., 2])
    op = divdamp_pl(g, -v2p[..., 0], -v2p[..., 1], -v2p[..., 2])
    gd = [g.divdamp_coef * a for a in o]
    gdp = [g.divdamp_coef * a for a in op]
    horizontalize(g, gd[0], gd[1], gd[2])
    horizontalize_pl(g, gdp[0], gdp[1], gdp[2])
    return gd, gdp


# --------------------------------------------------------------------------
# HEVI vertical implicit (mod_vi.py, kernels/vimatrix.py, virhowsolver.py,
# rhogkin.py, vimain.py, vipath1.py)
# --------------------------------------------------------------------------
def rhow_matrix(g, eth_h, gz, dt, pole=False):
    """kernels/vimatrix.py:67-164 (pre-combined coefficients)."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    ks, ksp, ksm = slice(kmin + 1, kmax + 1), slice(kmin + 2, kmax + 2), slice(kmin, kmax)
    RGSGAM2 = getattr(g, "VMTR_RGSGAM2" + sfx)
    GAM2H = getattr(g, "VMTR_GAM2H" + sfx)
    RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
    RGSQRTH = getattr(g, "VMTR_RGSQRTH" + sfx)
    GCVovR = g.GRAV * g.CVdry / g.Rdry
    ACVovRt2 = g.alpha * g.CVdry / g.Rdry / (dt * dt)
    if pole:
        K = lambda a, s: a[:, s]
        b1 = lambda v: v[None, :, None]
    else:
        K = lambda a, s: a[:, :, s]
        b1 = lambda v: v[None, None, :, None]
    rg, rgm = b1(g.GRD_rdgz[ks]), b1(g.GRD_rdgz[ksm])
    Ca = (K(RGSGAM2, ks) * rg + K(RGSGAM2, ksm) * rgm) * K(GAM2H, ks)
    Cb = b1(g.GRD_dfact[ks] - g.GRD_cfact[ksm])
    Cu1 = K(RGSGAM2, ks) * rg * K(GAM2H, ksp)
    Cu2 = K(GAM2H, ksp) * K(RGAMH, ks) ** 2 * GCVovR
    Cl1 = K(RGSGAM2, ks) * rg * K(GAM2H, ksm)
    Cl2 = K(GAM2H, ksm) * K(RGAMH, ks) ** 2 * GCVovR
    rgh = b1(g.GRD_rdgzh[ks])
    cf = b1(g.GRD_cfact[ks])
    dfm = b1(g.GRD_dfact[ksm])
    Mc = ACVovRt2 / K(RGSQRTH, ks) + rgh * (Ca * K(eth_h, ks) - Cb * (K(gz, ks) + GCVovR))
    Mu = -rgh * (Cu1 * K(eth_h, ksp) + cf * (K(gz, ksp) + Cu2))
    Ml = -rgh * (Cl1 * K(eth_h, ksm) - dfm * (K(gz, ksm) + Cl2))
    return Mc, Mu, Ml            # interior k = kmin+1..kmax


def rhow_solver(g, rhogw, rhogw0, preg0, rhog0, Srho, Sw, Spre, Mc, Mu, Ml, dt, pole=False):
    """kernels/virhowsolver.py:42-172 (Thomas solve on k = kmin+1..kmax)."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    ks, ksm = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
    RGSGAM2 = getattr(g, "VMTR_RGSGAM2" + sfx)
    RGAM = getattr(g, "VMTR_RGAM" + sfx)
    RGSGAM2H = getattr(g, "VMTR_RGSGAM2H" + sfx)
    GSGAM2H = getattr(g, "VMTR_GSGAM2H" + sfx)
    CVovRt2 = g.CVdry / g.Rdry / (dt * dt)
    if pole:
        K = lambda a, s: a[:, s]
        b1 = lambda v: v[None, :, None]
    else:
        K = lambda a, s: a[:, :, s]
        b1 = lambda v: v[None, None, :, None]
    rgh, af, bf = b1(g.GRD_rdgzh[ks]), b1(g.GRD_afact[ks]), b1(g.GRD_bfact[ks])
    Sall = ((K(rhogw0, ks) * g.alpha + dt * K(Sw, ks)) * K(RGAMH, ks) ** 2
            - ((K(preg0, ks) + dt * K(Spre, ks)) * K(RGSGAM2, ks)
               - (K(preg0, ksm) + dt * K(Spre, ksm)) * K(RGSGAM2, ksm)) * dt * rgh
            - ((K(rhog0, ks) + dt * K(Srho, ks)) * K(RGAM, ks) ** 2 * af
               + (K(rhog0, ksm) + dt * K(Srho, ksm)) * K(RGAM, ksm) ** 2 * bf) * dt * g.GRAV
            ) * CVovRt2
    rw_kmin = _kidx(rhogw, kmin) * _kidx(RGSGAM2H, kmin)
    rw_kmaxp1 = _kidx(rhogw, kmax + 1) * _kidx(RGSGAM2H, kmax + 1)
    N = kmax - kmin
    S = [_kidx(Sall, n) for n in range(N)]
    C = [_kidx(Mc, n) for n in range(N)]
    U = [_kidx(Mu, n) for n in range(N)]
    L = [_kidx(Ml, n) for n in range(N)]
    S[0] = S[0] - L[0] * rw_kmin
    S[N - 1] = S[N - 1] - U[N - 1] * rw_kmaxp1
    beta = C[0]
    u = [S[0] / beta]
    gam = [None] * N
    for n in range(1, N):
        gg = U[n - 1] / beta
        beta = C[n] - L[n] * gg
        u.append((S[n] - L[n] * u[n - 1]) / beta)
        gam[n] = gg
    x = [None] * N
    x[N - 1] = u[N - 1]
    for n in range(N - 2, -1, -1):
        x[n] = u[n] - gam[n + 1] * x[n + 1]
    out = rhogw.copy()
    for n in range(N):
        _kset(out, kmin + 1 + n, x[n] * _kidx(GSGAM2H, kmin + 1 + n))
    _kset(out, kmin, rw_kmin * _kidx(GSGAM2H, kmin))
    _kset(out, kmax + 1, rw_kmaxp1 * _kidx(GSGAM2H, kmax + 1))
    return out


def rhogkin(g, rhog, rvx, rvy, rvz, rw, pole=False):
    """kernels/rhogkin.py:38-119."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    C2W = getattr(g, "VMTR_C2Wfact" + sfx)
    W2C = getattr(g, "VMTR_W2Cfact" + sfx)
    kc, kvi, kcm = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    K = (lambda a, s: a[:, s]) if pole else (lambda a, s: a[:, :, s])
    kh = 0.5 * (K(rvx, kc) ** 2 + K(rvy, kc) ** 2 + K(rvz, kc) ** 2) / K(rhog, kc)
    denom = K(C2W, kvi)[..., 0] * K(rhog, kvi) + K(C2W, kvi)[..., 1] * K(rhog, kcm)
    v_int = 0.5 * K(rw, kvi) ** 2 / denom
    kax = 1 if pole else 2
    z = np.zeros_like(np.take(v_int, [0], axis=kax))
    vb = np.concatenate([z, v_int, z], axis=kax)
    vup = np.take(vb, range(1, vb.shape[kax]), axis=kax)
    vdn = np.take(vb, range(0, vb.shape[kax] - 1), axis=kax)
    tot = kh + K(W2C, kc)[..., 0] * vup + K(W2C, kc)[..., 1] * vdn
    out = np.zeros_like(rhog)
    if pole:
        out[:, kc] = tot
    else:
        out[:, :, kc] = tot
    return out


def vi_main(g, P, dt, pole):
    """kernels/vimain.py:127-262 (TIME_split) for one of regional / pole.
    ``P`` holds the arrays named as in the reference's P dict."""
    sfx = "_pl" if pole else ""
    PHI = getattr(g, "VMTR_PHI" + sfx)
    C2WGz = getattr(g, "VMTR_C2WfactGz" + sfx)
    kmin, kmax = g.kmin, g.kmax
    drhog = flux_convergence(g, P["rhogvx_s1"], P["rhogvy_s1"], P["rhogvz_s1"], P["rhogw_s0"], False, pole)
    drhoge = advection_convergence(g, P["rhogvx_s1"], P["rhogvy_s1"], P["rhogvz_s1"], P["rhogw_s0"],
                                   P["eth0"], False, pole)
    grhog1 = P["grhog"] + drhog
    grhoge1 = P["grhoge"] + drhoge
    gpre = grhoge1 * g.Rdry / g.CVdry
    vx, vy, vz = P["rhogvx_s1"], P["rhogvy_s1"], P["rhogvz_s1"]
    K = lambda a, k: _kidx(a, k)
    cz = lambda c: K(C2WGz[..., c], kmax + 1)
    rw_top = -(cz(0) * K(vx, kmax + 1) + cz(1) * K(vx, kmax) + cz(2) * K(vy, kmax + 1)
               + cz(3) * K(vy, kmax) + cz(4) * K(vz, kmax + 1) + cz(5) * K(vz, kmax))
    rhogw_s1 = np.zeros_like(vx)
    _kset(rhogw_s1, kmin, np.zeros_like(K(vx, kmin)))
    _kset(rhogw_s1, kmax + 1, rw_top)
    Mc, Mu, Ml = P["Mc"], P["Mu"], P["Ml"]
    rhogw_s1 = rhow_solver(g, rhogw_s1, P["rhogw_s0"], P["preg_s0"], P["rhog_s0"], grhog1, P["grhogw"],
                           gpre, Mc, Mu, Ml, dt, pole)
    drhog2 = flux_convergence(g, vx, vy, vz, rhogw_s1, True, pole)
    rhog_s1 = P["rhog_s0"] + (P["grhog"] + drhog2) * dt
    kin0 = rhogkin(g, P["rhog0"], P["rhogvx0"], P["rhogvy0"], P["rhogvz0"], P["rhogw0"], pole)
    kin10 = rhogkin(g, P["rhog0"] + P["rhog_s0"], P["rhogvx0"] + P["rhogvx_s0"], P["rhogvy0"] + P["rhogvy_s0"],
                    P["rhogvz0"] + P["rhogvz_s0"], P["rhogw0"] + P["rhogw_s0"], pole)
    rhogvx1b = P["rhogvx0"] + vx
    rhogvy1b = P["rhogvy0"] + vy
    rhogvz1b = P["rhogvz0"] + vz
    rhogw1b = P["rhogw0"] + rhogw_s1
    kin11 = rhogkin(g, P["rhog0"] + rhog_s1, rhogvx1b, rhogvy1b, rhogvz1b, rhogw1b, pole)
    ethtot0 = P["eth0"] + kin0 / P["rhog0"] + PHI
    drhogetot = advection_convergence(g, rhogvx1b, rhogvy1b, rhogvz1b, rhogw1b, ethtot0, True, pole)
    rhoge_s1 = (P["rhoge_s0"] + (P["grhogetot"] + drhogetot) * dt + (kin10 - kin11)
                + (P["rhog_s0"] - rhog_s1) * PHI)
    return rhog_s1, rhogw_s1, rhoge_s1


def vi_small_step(g, PROG, PROG_pl, DIAG, DIAG_pl, eth, eth_pl, rhogd, rhogd_pl, pregd, pregd_pl,
                  g_TEND0, g_TEND0_pl, PROG_split, PROG_split_pl, nitr, dt):
    """mod_vi.py:104-1590 numpy path.  Updates PROG/PROG_pl in place and
    returns PROG_mean, PROG_mean_pl (post-COMM)."""
    kmin, kmax = g.kmin, g.kmax
    RovCV = g.Rdry / g.CVdry
    alpha = g.alpha
    res = {}
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        P = PROG_pl if pole else PROG
        eth_ = eth_pl if pole else eth
        C2W = getattr(g, "VMTR_C2Wfact" + sfx)
        K = (lambda a, s: a[:, s]) if pole else (lambda a, s: a[:, :, s])
        ks_, ksm_ = slice(kmin, kmax + 2), slice(kmin - 1, kmax + 1)
        rhog_h = np.zeros_like(P[..., 0])
        eth_h = np.zeros_like(P[..., 0])
        if pole:
            rhog_h[:, ks_] = C2W[:, ks_, :, 0] * P[:, ks_, :, I_RHOG] + C2W[:, ks_, :, 1] * P[:, ksm_, :, I_RHOG]
            eth_h[:, ks_] = (g.GRD_afact[ks_][None, :, None] * eth_[:, ks_]
                             + g.GRD_bfact[ks_][None, :, None] * eth_[:, ksm_])
            eth_h[:, kmin - 1] = eth_h[:, kmin]
            rhog_h[:, kmin - 1] = rhog_h[:, kmin]
        else:
            rhog_h[:, :, ks_] = (C2W[:, :, ks_, :, 0] * P[:, :, ks_, :, I_RHOG]
                                 + C2W[:, :, ks_, :, 1] * P[:, :, ksm_, :, I_RHOG])
            eth_h[:, :, ks_] = (g.GRD_afact[ks_][None, None, :, None] * eth_[:, :, ks_]
                                + g.GRD_bfact[ks_][None, None, :, None] * eth_[:, :, ksm_])
            rhog_h[:, :, kmin - 1] = rhog_h[:, :, kmin]
            eth_h[:, :, kmin - 1] = eth_h[:, :, kmin]
        res["rhog_h" + sfx] = rhog_h
        res["eth_h" + sfx] = eth_h
        res["drhog" + sfx] = flux_convergence(g, P[..., I_RHOGVX], P[..., I_RHOGVY], P[..., I_RHOGVZ],
                                              P[..., I_RHOGW], True, pole)
    gd, gdp = numfilter_divdamp(g, PROG[..., I_RHOGVX], PROG[..., I_RHOGVY], PROG[..., I_RHOGVZ],
                                PROG[..., I_RHOGW], PROG_pl[..., I_RHOGVX], PROG_pl[..., I_RHOGVY],
                                PROG_pl[..., I_RHOGVZ], PROG_pl[..., I_RHOGW])
    dpg, dpgw, dpg_pl, dpgw_pl = pres_gradient(g, pregd, pregd_pl, True)
    g_TEND, g_TEND_pl = {}, {}
    gz = {}
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        P = PROG_pl if pole else PROG
        D = DIAG_pl if pole else DIAG
        G0 = g_TEND0_pl if pole else g_TEND0
        dbuo = buoyancy(g, rhogd_pl if pole else rhogd, pole)
        drhoge = advection_convergence(g, P[..., I_RHOGVX], P[..., I_RHOGVY], P[..., I_RHOGVZ], P[..., I_RHOGW],
                                       eth_pl if pole else eth, True, pole)
        dg, dgw = (dpg_pl, dpgw_pl) if pole else (dpg, dpgw)
        gzt = g.GRAV - (dgw - dbuo) / res["rhog_h" + sfx]
        pwh = -gzt * P[..., I_RHOGW]
        W2C = getattr(g, "VMTR_W2Cfact" + sfx)
        kc, kp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
        pw = np.zeros_like(pwh)
        if pole:
            pw[:, kc] = (D[:, kc, :, I_vx] * dg[:, kc, :, XDIR] + D[:, kc, :, I_vy] * dg[:, kc, :, YDIR]
                         + D[:, kc, :, I_vz] * dg[:, kc, :, ZDIR] + W2C[:, kc, :, 0] * pwh[:, kp]
                         + W2C[:, kc, :, 1] * pwh[:, kc])
        else:
            pw[:, :, kc] = (D[:, :, kc, :, I_vx] * dg[:, :, kc, :, XDIR] + D[:, :, kc, :, I_vy] * dg[:, :, kc, :, YDIR]
                            + D[:, :, kc, :, I_vz] * dg[:, :, kc, :, ZDIR] + W2C[:, :, kc, :, 0] * pwh[:, :, kp]
                            + W2C[:, :, kc, :, 1] * pwh[:, :, kc])
        dd = gdp if pole else gd
        zero = np.zeros_like(pw)
        T = np.zeros(pw.shape + (6,))
        T[..., I_RHOG] = G0[..., I_RHOG] + res["drhog" + sfx]
        T[..., I_RHOGVX] = G0[..., I_RHOGVX] - dg[..., XDIR] + dd[0] + zero
        T[..., I_RHOGVY] = G0[..., I_RHOGVY] - dg[..., YDIR] + dd[1] + zero
        T[..., I_RHOGVZ] = G0[..., I_RHOGVZ] - dg[..., ZDIR] + dd[2] + zero
        T[..., I_RHOGW] = G0[..., I_RHOGW] + zero * alpha - dgw + dbuo
        T[..., I_RHOGE] = G0[..., I_RHOGE] + drhoge + pw
        if pole:
            g_TEND_pl = T
        else:
            g_TEND = T
        gz[sfx] = gzt
    rweight = 1.0 / float(nitr)
    PROG_mean = PROG[..., 0:5].copy()
    PROG_mean_pl = PROG_pl[..., 0:5].copy()
    Mats = {}
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        Mats[sfx] = rhow_matrix(g, res["eth_h" + sfx], gz[sfx], dt, pole)
    PS, PSp = PROG_split, PROG_split_pl
    for ns in range(nitr):
        preg_s = PS[..., I_RHOGE] * RovCV
        _kset(preg_s, kmin - 1, _kidx(preg_s, kmin)); _kset(preg_s, kmax + 1, _kidx(preg_s, kmax))
        _kset(PS[..., I_RHOGE], kmin - 1, _kidx(PS[..., I_RHOGE], kmin))
        _kset(PS[..., I_RHOGE], kmax + 1, _kidx(PS[..., I_RHOGE], kmax))
        preg_sp = PSp[..., I_RHOGE] * RovCV
        _kset(preg_sp, kmin - 1, _kidx(preg_sp, kmin)); _kset(preg_sp, kmax + 1, _kidx(preg_sp, kmax))
        _kset(PSp[..., I_RHOGE], kmin - 1, _kidx(PSp[..., I_RHOGE], kmin))
        _kset(PSp[..., I_RHOGE], kmax + 1, _kidx(PSp[..., I_RHOGE], kmax))
        dd, ddp = numfilter_divdamp(g, PS[..., I_RHOGVX], PS[..., I_RHOGVY], PS[..., I_RHOGVZ], PS[..., I_RHOGW],
                                    PSp[..., I_RHOGVX], PSp[..., I_RHOGVY], PSp[..., I_RHOGVZ], PSp[..., I_RHOGW])
        # _vi_path1_fused (kernels/vipath1.py:68-160), gradtype horizontal
        Pg, _, Pg_pl, _ = pres_gradient(g, preg_s, preg_sp, False)
        dvh, dvhp = [], []
        drw = {}
        for pole in (False, True):
            T = g_TEND_pl if pole else g_TEND
            pg = Pg_pl if pole else Pg
            ddd = ddp if pole else dd
            S = PSp if pole else PS
            P = PROG_pl if pole else PROG
            zero = np.zeros_like(T[..., 0])
            dx = T[..., I_RHOGVX] - pg[..., XDIR] + ddd[0] + zero
            dy = T[..., I_RHOGVY] - pg[..., YDIR] + ddd[1] + zero
            dz = T[..., I_RHOGVZ] - pg[..., ZDIR] + ddd[2] + zero
            drw["_pl" if pole else ""] = T[..., I_RHOGW] + zero * alpha
            vx_ = S[..., I_RHOGVX] + dx * dt
            vy_ = S[..., I_RHOGVY] + dy * dt
            vz_ = S[..., I_RHOGVZ] + dz * dt
            rg = P[..., I_RHOG]
            for v in (vx_, vy_, vz_):
                top = 1.0 * (_kidx(v, kmax) / _kidx(rg, kmax)) * _kidx(rg, kmax + 1)
                btm = -1.0 * (_kidx(v, kmin) / _kidx(rg, kmin)) * _kidx(rg, kmin - 1)
                _kset(v, kmax + 1, top)
                _kset(v, kmin - 1, btm)
            arr = np.stack([vx_, vy_, vz_], axis=-1)
            (dvhp if pole else dvh).append(arr)
        dvh, dvhp = dvh[0], dvhp[0]
        comm(g, dvh, dvhp)
        dwe = np.zeros(PS.shape[:-1] + (3,))
        dwep = np.zeros(PSp.shape[:-1] + (3,))
        for pole in (False, True):
            sfx = "_pl" if pole else ""
            S = PSp if pole else PS
            P = PROG_pl if pole else PROG
            T = g_TEND_pl if pole else g_TEND
            G0 = g_TEND0_pl if pole else g_TEND0
            V = dvhp if pole else dvh
            Mc, Mu, Ml = Mats[sfx]
            Pd = {
                "rhogvx_s1": V[..., 0], "rhogvy_s1": V[..., 1], "rhogvz_s1": V[..., 2],
                "rhog_s0": S[..., I_RHOG], "rhogvx_s0": S[..., I_RHOGVX], "rhogvy_s0": S[..., I_RHOGVY],
                "rhogvz_s0": S[..., I_RHOGVZ], "rhogw_s0": S[..., I_RHOGW], "rhoge_s0": S[..., I_RHOGE],
                "preg_s0": preg_sp if pole else preg_s,
                "rhog0": P[..., I_RHOG], "rhogvx0": P[..., I_RHOGVX], "rhogvy0": P[..., I_RHOGVY],
                "rhogvz0": P[..., I_RHOGVZ], "rhogw0": P[..., I_RHOGW], "eth0": eth_pl if pole else eth,
                "grhog": T[..., I_RHOG], "grhogw": drw[sfx], "grhoge": T[..., I_RHOGE],
                "grhogetot": G0[..., I_RHOGE], "Mc": Mc, "Mu": Mu, "Ml": Ml,
            }
            r1, rw1, re1 = vi_main(g, Pd, dt, pole)
            W = dwep if pole else dwe
            W[..., 0], W[..., 1], W[..., 2] = r1, rw1, re1
        comm(g, dwe, dwep)
        for (S, V, W, PM) in ((PS, dvh, dwe, PROG_mean), (PSp, dvhp, dwep, PROG_mean_pl)):
            S[..., I_RHOGVX] = V[..., 0]
            S[..., I_RHOGVY] = V[..., 1]
            S[..., I_RHOGVZ] = V[..., 2]
            S[..., I_RHOG] = W[..., 0]
            S[..., I_RHOGW] = W[..., 1]
            S[..., I_RHOGE] = W[..., 2]
            PM += S[..., 0:5] * rweight
    PROG[..., 0:6] += PS[..., 0:6]
    PROG_pl[...] += PSp
    a, b, c = PROG[..., I_RHOGVX].copy(), PROG[..., I_RHOGVY].copy(), PROG[..., I_RHOGVZ].copy()
    horizontalize(g, a, b, c)
    PROG[..., I_RHOGVX], PROG[..., I_RHOGVY], PROG[..., I_RHOGVZ] = a, b, c
    a, b, c = PROG_pl[..., I_RHOGVX].copy(), PROG_pl[..., I_RHOGVY].copy(), PROG_pl[..., I_RHOGVZ].copy()
    horizontalize_pl(g, a, b, c)
    PROG_pl[..., I_RHOGVX], PROG_pl[..., I_RHOGVY], PROG_pl[..., I_RHOGVZ] = a, b, c
    comm(g, PROG_mean, PROG_mean_pl)
    return PROG_mean, PROG_mean_pl



# --------------------------------------------------------------------------
# tracer advection (mod_src_tracer.py, MIURA2004 + Thuburn limiters)
# --------------------------------------------------------------------------
def _tracer_vert_flux(g, rvx, rvy, rvz, rw, rhog_in, frhog, dt, pole):
    """kernels/tracervertflux.py:44-167 -> flx_v, ck(...,2), rhog (b1 = 0)."""
    sfx = "_pl" if pole else ""
    kmin, kmax = g.kmin, g.kmax
    C2WGz = getattr(g, "VMTR_C2WfactGz" + sfx)
    RGAMH = getattr(g, "VMTR_RGAMH" + sfx)
    RGSQRTH = getattr(g, "VMTR_RGSQRTH" + sfx)
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    kc, kcp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
    K = (lambda a, s: a[:, s]) if pole else (lambda a, s: a[:, :, s])
    c2w = K(C2WGz, ks)
    horiz = (c2w[..., 0] * K(rvx, ks) + c2w[..., 1] * K(rvx, km) + c2w[..., 2] * K(rvy, ks)
             + c2w[..., 3] * K(rvy, km) + c2w[..., 4] * K(rvz, ks) + c2w[..., 5] * K(rvz, km)) * K(RGAMH, ks)
    vert = K(rw, ks) * K(RGSQRTH, ks)
    flx = np.zeros_like(rhog_in)
    ck = np.zeros(rhog_in.shape + (2,))
    rhog = np.zeros_like(rhog_in)
    b1 = 0.0
    if pole:
        flx[:, ks] = (horiz + vert) * 0.5 * dt
        rdz = g.GRD_rdgz[kc][None, :, None]
        ck[:, kc, :, 0] = -flx[:, kc] / rhog_in[:, kc] * rdz
        ck[:, kc, :, 1] = flx[:, kcp] / rhog_in[:, kc] * rdz
        rhog[:, kc] = rhog_in[:, kc] - (flx[:, kcp] - flx[:, kc]) * rdz + b1 * frhog[:, kc] * dt
        rhog[:, kmin - 1] = rhog_in[:, kmin]
        rhog[:, kmax + 1] = rhog_in[:, kmax]
    else:
        flx[:, :, ks] = (horiz + vert) * 0.5 * dt
        rdz = g.GRD_rdgz[kc][None, None, :, None]
        ck[:, :, kc, :, 0] = -flx[:, :, kc] / rhog_in[:, :, kc] * rdz
        ck[:, :, kc, :, 1] = flx[:, :, kcp] / rhog_in[:, :, kc] * rdz
        rhog[:, :, kc] = rhog_in[:, :, kc] - (flx[:, :, kcp] - flx[:, :, kc]) * rdz + b1 * frhog[:, :, kc] * dt
        rhog[:, :, kmin - 1] = rhog_in[:, :, kmin]
        rhog[:, :, kmax + 1] = rhog_in[:, :, kmax]
    return flx, ck, rhog


def vertical_limiter(g, q_h, q, d, ck):
    """mod_src_tracer.py:1909-2074 (host loop; regional and pole alike):
    clips q_h on k = kmin+1..kmax, in place.  Works on (..., k, l) arrays whose
    level axis is -2 (regional (i,j,k,l) and pole (g,k,l))."""
    kmin, kmax = g.kmin, g.kmax
    BIG, EPS = g.HUGE, g.EPS
    ax = q.ndim - 2
    T = lambda a, k: np.take(a, k, axis=ax)
    ck0, ck1 = ck[..., 0], ck[..., 1]
    qmin_prev = qmax_prev = None
    for k in range(kmin, kmax + 1):
        inL = 0.5 - np.copysign(0.5, T(ck0, k))
        inU = 0.5 + np.copysign(0.5, T(ck0, k + 1))
        qc, qb, qa = T(q, k), T(q, k - 1), T(q, k + 1)
        QminL = np.where(inL == 1.0, np.minimum(qc, qb), BIG)
        QminU = np.where(inU == 1.0, np.minimum(qc, qa), BIG)
        QmaxL = np.where(inL == 1.0, np.maximum(qc, qb), -BIG)
        QmaxU = np.where(inU == 1.0, np.maximum(qc, qa), -BIG)
        qnmin = np.minimum(np.minimum(QminL, QminU), qc)
        qnmax = np.maximum(np.maximum(QmaxL, QmaxU), qc)
        c1, c2 = T(ck0, k), T(ck1, k)
        Cin = inL * c1 + inU * c2
        Cout = (1.0 - inL) * c1 + (1.0 - inU) * c2
        CQmin = inL * c1 * QminL + inU * c2 * QminU
        CQmax = inL * c1 * QmaxL + inU * c2 * QmaxU
        zsw = 0.5 - np.copysign(0.5, np.abs(Cout) - EPS)
        dk = T(d, k)
        qomin = ((qc - qnmax) + qnmax * (Cin + Cout - dk) - CQmax) / (Cout + zsw) * (1.0 - zsw) + qc * zsw
        qomax = ((qc - qnmin) + qnmin * (Cin + Cout - dk) - CQmin) / (Cout + zsw) * (1.0 - zsw) + qc * zsw
        if k > kmin:
            qh = T(q_h, k)
            new = (inL * np.minimum(np.maximum(qh, qmin_prev), qmax_prev)
                   + (1.0 - inL) * np.minimum(np.maximum(qh, qomin), qomax))
            if ax == 2:
                q_h[:, :, k] = new
            else:
                q_h[:, k] = new
        qmin_prev, qmax_prev = qomin, qomax


def _vertical_advection(g, rhogq, q_den, flx, ck, d, pole, clamp):
    """one vertical fractional step for one tracer (mod_src_tracer.py:389-533,
    1036-1204), in place on rhogq."""
    kmin, kmax = g.kmin, g.kmax
    af, bf = g.GRD_afact, g.GRD_bfact
    q = rhogq / q_den
    q_h = np.zeros_like(q)
    if pole:
        q_h[:, kmin:kmax + 2] = af[kmin:kmax + 2][None, :, None] * q[:, kmin:kmax + 2] \
            + bf[kmin:kmax + 2][None, :, None] * q[:, kmin - 1:kmax + 1]
    else:
        for k in range(kmin, kmax + 2):
            q_h[:, :, k] = af[k] * q[:, :, k] + bf[k] * q[:, :, k - 1]
    vertical_limiter(g, q_h, q, d, ck)
    _kset(q_h, kmin, 0.0)
    _kset(q_h, kmax + 1, 0.0)
    for k in range(kmin, kmax + 1):
        upd = (_kidx(flx, k + 1) * _kidx(q_h, k + 1) - _kidx(flx, k) * _kidx(q_h, k)) * g.GRD_rdgz[k]
        _kset(rhogq, k, _kidx(rhogq, k) - upd)
    _kset(rhogq, kmin - 1, 0.0)
    _kset(rhogq, kmax + 1, 0.0)
    if clamp:
        if pole:
            m = (rhogq > -1.0e-10) & (rhogq < 0.0)
            rhogq[m] = 0.0
        else:
            sub = rhogq[:, :, kmin:kmax + 1]
            m = (sub > -1.0e-10) & (sub < 0.0)
            sub[m] = 0.0


def horizontal_flux(g, rho, rvx, rvy, rvz, rho_pl, rvx_pl, rvy_pl, rvz_pl, dt):
    """mod_src_tracer.py:1376-1531 -> flx_h (i,j,k,l,6), grd_xc (i,j,k,l,3,3),
    flx_h_pl (g,k,l), grd_xc_pl (g,k,l,3)."""
    i, j, kall, lall = rho.shape
    EPS = g.EPS
    gt = g.GMTR_t[:, :, 0]                      # (i,j,l,2,5)
    ga = g.GMTR_a[:, :, 0]                      # (i,j,l,3,12)
    gp = g.GMTR_p[:, :, 0]                      # (i,j,l,8)
    xr = g.GRD_xr[:, :, 0]                      # (i,j,l,3,3)
    flx_h = np.zeros(rho.shape + (6,))
    grd_xc = np.zeros(rho.shape + (3, 3))
    isl, jsl = slice(0, i - 1), slice(0, j - 1)
    isp, jsp = slice(1, i), slice(1, j)
    W = lambda t, w: gt[isl, jsl, :, t, w][:, :, None, :]
    fields = [rho, rvx, rvy, rvz]
    TIv, TJv = [], []
    for f in fields:
        ti = f[isl, jsl] * W(TI, W1) + f[isp, jsl] * W(TI, W2)
        tj = f[isl, jsl] * W(TJ, W1)
        ti = ti + f[isp, jsp] * W(TI, W3)
        tj = tj + (f[isp, jsp] * W(TJ, W2) + f[isl, jsp] * W(TJ, W3))
        m0 = g.pntmask[0, :, 0][None, :]
        m1 = g.pntmask[0, :, 1][None, :]
        ti[0, 0] = ti[0, 0] * m0 + tj[1, 0] * m1
        TIv.append(ti)
        TJv.append(tj)
    rT, xT, yT, zT = TIv
    rJ, xJ, yJ, zJ = TJv
    PR = lambda a, b: gp[a, b, :, P_RAREA][:, :, None, :]

    def edge(a_sl, b_sl, rr, vx2, vy2, vz2, face):
        rr2 = 1.0 / np.maximum(rr, EPS)
        A = lambda c: ga[a_sl, b_sl, :, face, c][:, :, None, :]
        flux = 0.5 * (vx2 * A(HNX) + vy2 * A(HNY) + vz2 * A(HNZ))
        xc = [xr[a_sl, b_sl, :, face, d][:, :, None, :] - v2 * rr2 * dt * 0.5
              for d, v2 in ((XDIR, vx2), (YDIR, vy2), (ZDIR, vz2))]
        return flux, xc
    # AI face: isl, jsl = 0..i-2, 1..j-2
    a_, b_ = slice(0, i - 1), slice(1, j - 1)
    bm = slice(0, j - 2)
    flux, xc = edge(a_, b_, rJ[:, bm] + rT[:, b_], xJ[:, bm] + xT[:, b_], yJ[:, bm] + yT[:, b_],
                    zJ[:, bm] + zT[:, b_], AI)
    flx_h[a_, b_, :, :, 0] = flux * PR(a_, b_) * dt
    flx_h[1:i, b_, :, :, 3] = -flux * PR(slice(1, i), b_) * dt
    for d in range(3):
        grd_xc[a_, b_, :, :, AI, d] = xc[d]
    # AIJ face: 0..i-2, 0..j-2
    a_, b_ = slice(0, i - 1), slice(0, j - 1)
    flux, xc = edge(a_, b_, rT + rJ, xT + xJ, yT + yJ, zT + zJ, AIJ)
    flx_h[a_, b_, :, :, 1] = flux * PR(a_, b_) * dt
    flx_h[1:i, 1:j, :, :, 4] = -flux * PR(slice(1, i), slice(1, j)) * dt
    for d in range(3):
        grd_xc[a_, b_, :, :, AIJ, d] = xc[d]
    # AJ face: 1..i-2, 0..j-2
    a_, b_ = slice(1, i - 1), slice(0, j - 1)
    am = slice(0, i - 2)
    flux, xc = edge(a_, b_, rJ[a_] + rT[am], xJ[a_] + xT[am], yJ[a_] + yT[am], zJ[a_] + zT[am], AJ)
    flx_h[a_, b_, :, :, 2] = flux * PR(a_, b_) * dt
    flx_h[a_, 1:j, :, :, 5] = -flux * PR(a_, slice(1, j)) * dt
    for d in range(3):
        grd_xc[a_, b_, :, :, AJ, d] = xc[d]
    flx_h[1, 1, :, :, 5] *= g.pntmask[0, :, 0].astype(np.float64)[None, :]
    # pole
    gtp = g.GMTR_t_pl[:, 0]                     # (6, l, 5)
    gap = g.GMTR_a_pl[:, 0]                     # (6, l, 18)
    gpp = g.GMTR_p_pl[:, 0]
    flx_pl = np.zeros_like(rho_pl)
    xc_pl = np.zeros(rho_pl.shape + (3,))
    for l in range(rho_pl.shape[2]):
        tv = {}
        for v in range(1, 6):
            vp1 = 1 if v + 1 == 6 else v + 1
            tv[v] = [f[0, :, l] * gtp[v, l, W1] + f[v, :, l] * gtp[v, l, W2] + f[vp1, :, l] * gtp[v, l, W3]
                     for f in (rho_pl, rvx_pl, rvy_pl, rvz_pl)]
        for v in range(1, 6):
            vm1 = 5 if v - 1 == 0 else v - 1
            rr2 = 1.0 / np.maximum(tv[vm1][0] + tv[v][0], EPS)
            v2 = [tv[vm1][n] + tv[v][n] for n in (1, 2, 3)]
            flux = 0.5 * (v2[0] * gap[v, l, HNX] + v2[1] * gap[v, l, HNY] + v2[2] * gap[v, l, HNZ])
            flx_pl[v, :, l] = flux * gpp[0, l, P_RAREA] * dt
            for d in range(3):
                xc_pl[v, :, l, d] = g.GRD_xr_pl[v, 0, l, d] - v2[d] * rr2 * dt * 0.5
    return flx_h, grd_xc, flx_pl, xc_pl


def horizontal_remap(g, q, q_pl, cmask, cmask_pl, grd_xc, grd_xc_pl):
    """mod_src_tracer.py:1535-1847 (numpy loops) -> q_a (i,j,k,l,6), q_a_pl."""
    i, j = q.shape[:2]
    gq = gradient(g, q)
    gq_pl = gradient_pl(g, q_pl)
    comm(g, gq, gq_pl)
    X = g.GRD_x[:, :, 0]                        # (i,j,l,3)

    def rec(qs, gqs, xcs, xs):
        out = qs
        for d in (XDIR, YDIR, ZDIR):
            out = out + gqs[..., d] * (xcs[..., d] - xs[..., d][:, :, None, :])
        return out
    isl, jsl, isp, jsp = slice(0, i - 1), slice(0, j - 1), slice(1, i), slice(1, j)
    ins, jns, inm, jnm = slice(1, i - 1), slice(1, j - 1), slice(0, i - 2), slice(0, j - 2)
    qap = [np.zeros(q.shape) for _ in range(6)]
    qam = [np.zeros(q.shape) for _ in range(6)]
    xc = lambda a, b, f: grd_xc[a, b, :, :, f, :]
    qap[0][isl, jsl] = rec(q[isl, jsl], gq[isl, jsl], xc(isl, jsl, AI), X[isl, jsl])
    qam[0][isl, jsl] = rec(q[isp, jsl], gq[isp, jsl], xc(isl, jsl, AI), X[isp, jsl])
    qap[1][isl, jsl] = rec(q[isl, jsl], gq[isl, jsl], xc(isl, jsl, AIJ), X[isl, jsl])
    qam[1][isl, jsl] = rec(q[isp, jsp], gq[isp, jsp], xc(isl, jsl, AIJ), X[isp, jsp])
    qap[2][isl, jsl] = rec(q[isl, jsl], gq[isl, jsl], xc(isl, jsl, AJ), X[isl, jsl])
    qam[2][isl, jsl] = rec(q[isl, jsp], gq[isl, jsp], xc(isl, jsl, AJ), X[isl, jsp])
    qap[3][ins, jns] = rec(q[inm, jns], gq[inm, jns], xc(inm, jns, AI), X[inm, jns])
    qam[3][ins, jns] = rec(q[ins, jns], gq[ins, jns], xc(inm, jns, AI), X[ins, jns])
    qap[4][ins, jns] = rec(q[inm, jnm], gq[inm, jnm], xc(inm, jnm, AIJ), X[inm, jnm])
    qam[4][ins, jns] = rec(q[ins, jns], gq[ins, jns], xc(inm, jnm, AIJ), X[ins, jns])
    qap[5][ins, jns] = rec(q[ins, jnm], gq[ins, jnm], xc(ins, jnm, AJ), X[ins, jnm])
    qam[5][ins, jns] = rec(q[ins, jns], gq[ins, jns], xc(ins, jnm, AJ), X[ins, jns])
    q_a = np.full(q.shape + (6,), np.nan)
    for f in range(6):
        q_a[isl, jsl, :, :, f] = cmask[isl, jsl, :, :, f] * qam[f][isl, jsl] \
            + (1.0 - cmask[isl, jsl, :, :, f]) * qap[f][isl, jsl]
    q_a_pl = np.full(q_pl.shape, np.nan)
    Xp = g.GRD_x_pl[:, 0]                       # (6,l,3)
    for v in range(1, 6):
        ap = q_pl[0]
        am = q_pl[v]
        for d in (XDIR, YDIR, ZDIR):
            ap = ap + gq_pl[0, :, :, d] * (grd_xc_pl[v, :, :, d] - Xp[0, :, d][None, :])
        for d in (XDIR, YDIR, ZDIR):
            am = am + gq_pl[v, :, :, d] * (grd_xc_pl[v, :, :, d] - Xp[v, :, d][None, :])
        q_a_pl[v] = cmask_pl[v] * am + (1.0 - cmask_pl[v]) * ap
    return q_a, q_a_pl


def horizontal_limiter(g, q_a, q_a_pl, q, q_pl, d, d_pl, ch, ch_pl, cmask, cmask_pl):
    """mod_src_tracer.py:2115-2664 (numpy branch), in place on q_a / q_a_pl."""
    i, j = q.shape[:2]
    BIG, EPS = g.HUGE, g.EPS
    Qin = np.full(q.shape + (2, 6), np.nan)
    mn = lambda *a: _reduce(np.minimum, a)
    mx = lambda *a: _reduce(np.maximum, a)
    I0, J0 = slice(0, i - 1), slice(0, j - 1)
    q0 = q[I0, J0]
    q1 = np.empty_like(q0)
    q1[:, 1:] = q[I0, 0:j - 2]
    q1[:, 0] = q[0, 0]
    q2 = q[1:i, J0]
    q3 = q[1:i, 1:j]
    qjp = q[I0, 1:j]
    q4 = np.empty_like(q0)
    q4[1:, :] = q[0:i - 2, J0]
    q4[0, :] = q[0, 0]
    qmin = [mn(q0, q1, q2, q3), mn(q0, q2, q3, qjp), mn(q0, q3, qjp, q4)]
    qmax = [mx(q0, q1, q2, q3), mx(q0, q2, q3, qjp), mx(q0, q3, qjp, q4)]
    cm = cmask[I0, J0]
    for m in range(3):
        Qin[I0, J0, :, :, 0, m] = cm[..., m] * qmin[m] + (1.0 - cm[..., m]) * BIG
        Qin[I0, J0, :, :, 1, m] = cm[..., m] * qmax[m] + (1.0 - cm[..., m]) * (-BIG)
    Qin[1:i, J0, :, :, 0, 3] = cm[..., 0] * BIG + (1.0 - cm[..., 0]) * qmin[0]
    Qin[1:i, J0, :, :, 1, 3] = cm[..., 0] * (-BIG) + (1.0 - cm[..., 0]) * qmax[0]
    Qin[1:i, 1:j, :, :, 0, 4] = cm[..., 1] * BIG + (1.0 - cm[..., 1]) * qmin[1]
    Qin[1:i, 1:j, :, :, 1, 4] = cm[..., 1] * (-BIG) + (1.0 - cm[..., 1]) * qmax[1]
    Qin[I0, 1:j, :, :, 0, 5] = cm[..., 2] * BIG + (1.0 - cm[..., 2]) * qmin[2]
    Qin[I0, 1:j, :, :, 1, 5] = cm[..., 2] * (-BIG) + (1.0 - cm[..., 2]) * qmax[2]
    for l in range(q.shape[3]):
        if g.have_sgp[l]:
            vals = np.stack([q[0, 0, :, l], q[1, 1, :, l], q[2, 1, :, l], q[0, 1, :, l]])
            qn, qx = vals.min(axis=0), vals.max(axis=0)
            c1 = cmask[0, 0, :, l, 1]
            Qin[0, 0, :, l, 0, 1] = np.where(c1 == 1.0, qn, BIG)
            Qin[1, 1, :, l, 0, 4] = np.where(c1 == 1.0, BIG, qn)
            Qin[0, 0, :, l, 1, 1] = np.where(c1 == 1.0, qx, -BIG)
            Qin[1, 1, :, l, 1, 4] = np.where(c1 == 1.0, -BIG, qx)
    Qout = np.full(q.shape + (2,), np.nan)
    In, Jn = slice(1, i - 1), slice(1, j - 1)
    qi = q[In, Jn]
    Qi = Qin[In, Jn]
    qnmin = mn(qi, *[Qi[..., 0, m] for m in range(6)])
    qnmax = mx(qi, *[Qi[..., 1, m] for m in range(6)])
    chi = ch[In, Jn]
    chm = np.minimum(chi, 0.0)
    Cin = np.sum(chm, axis=-1)
    Cout = np.sum(chi - chm, axis=-1)
    CQmin = np.sum(chm * Qi[..., 0, :], axis=-1)
    CQmax = np.sum(chm * Qi[..., 1, :], axis=-1)
    zsw = 0.5 - np.copysign(0.5, np.abs(Cout) - EPS)
    di = d[In, Jn]
    Qout[In, Jn, :, :, 0] = (qi - CQmax - qnmax * (1.0 - Cin - Cout + di)) / (Cout + zsw) * (1.0 - zsw) + qi * zsw
    Qout[In, Jn, :, :, 1] = (qi - CQmin - qnmin * (1.0 - Cin - Cout + di)) / (Cout + zsw) * (1.0 - zsw) + qi * zsw
    for b in (0, 1):
        Qout[:, 0, :, :, b] = q[:, 0]
        Qout[:, j - 1, :, :, b] = q[:, j - 1]
        Qout[0, 1:j - 1, :, :, b] = q[0, 1:j - 1]
        Qout[i - 1, 1:j - 1, :, :, b] = q[i - 1, 1:j - 1]
    # pole Qin / Qout (mod_src_tracer.py:2437-2495)
    Qin_pl = np.full(q_pl.shape + (2, 2), np.nan)
    Qout_pl = np.full(q_pl.shape + (2,), np.nan)
    for v in range(1, 6):
        vp1 = 1 if v + 1 > 5 else v + 1
        vm1 = 5 if v - 1 < 1 else v - 1
        # Python builtin min/max (mod_src_tracer.py:2446-2447): ties keep the first
        qn = _reduce(_pymin, (q_pl[0], q_pl[v], q_pl[vm1], q_pl[vp1]))
        qx = _reduce(_pymax, (q_pl[0], q_pl[v], q_pl[vm1], q_pl[vp1]))
        c = cmask_pl[v]
        Qin_pl[v, ..., 0, 0] = np.where(c == 1.0, qn, BIG)
        Qin_pl[v, ..., 0, 1] = np.where(c == 1.0, BIG, qn)
        Qin_pl[v, ..., 1, 0] = np.where(c == 1.0, qx, -BIG)
        Qin_pl[v, ..., 1, 1] = np.where(c == 1.0, -BIG, qx)
    qnm = q_pl[0].copy()
    qnx = q_pl[0].copy()
    for v in range(1, 6):
        qnm = _pymin(qnm, Qin_pl[v, ..., 0, 0])
        qnx = _pymax(qnx, Qin_pl[v, ..., 1, 0])
    Ci = np.zeros_like(q_pl[0]); Co = np.zeros_like(q_pl[0])
    CQn = np.zeros_like(q_pl[0]); CQx = np.zeros_like(q_pl[0])
    for v in range(1, 6):
        chm_ = cmask_pl[v] * ch_pl[v]
        Ci = Ci + chm_
        Co = Co + (ch_pl[v] - chm_)
        CQn = CQn + chm_ * Qin_pl[v, ..., 0, 0]
        CQx = CQx + chm_ * Qin_pl[v, ..., 1, 0]
    zs = 0.5 - np.copysign(0.5, np.abs(Co) - EPS)
    den = Co + zs
    fac = 1.0 - zs
    q0p = q_pl[0]
    dv = d_pl[0]
    Qout_pl[0, ..., 0] = (q0p - CQx - qnx * (1.0 - Ci - Co + dv)) / den * fac + q0p * zs
    Qout_pl[0, ..., 1] = (q0p - CQn - qnm * (1.0 - Ci - Co + dv)) / den * fac + q0p * zs
    comm(g, Qout, Qout_pl)
    # apply (mod_src_tracer.py:2536-2605)
    Ip, Jp = slice(1, i), slice(1, j)
    c = cmask[I0, J0]

    def clampin(x, lo, hi):
        return np.minimum(np.maximum(x, lo), hi)

    def clampout(x, hi, lo):
        return np.maximum(np.minimum(x, hi), lo)
    for f, (A, B), m2 in ((0, (Ip, J0), 3), (1, (Ip, Jp), 4), (2, (I0, Jp), 5)):
        cf = c[..., f]
        qa = q_a[I0, J0, :, :, f]
        qa = cf * clampin(qa, Qin[I0, J0, :, :, 0, f], Qin[I0, J0, :, :, 1, f]) \
            + (1.0 - cf) * clampin(qa, Qin[A, B, :, :, 0, m2], Qin[A, B, :, :, 1, m2])
        qa = cf * clampout(qa, Qout[A, B, :, :, 1], Qout[A, B, :, :, 0]) \
            + (1.0 - cf) * clampout(qa, Qout[I0, J0, :, :, 1], Qout[I0, J0, :, :, 0])
        q_a[I0, J0, :, :, f] = qa
        q_a[A, B, :, :, m2] = qa
    for v in range(1, 6):
        cmv = cmask_pl[v]
        a0 = clampin(q_a_pl[v], Qin_pl[v, ..., 0, 0], Qin_pl[v, ..., 1, 0])
        a1 = clampin(q_a_pl[v], Qin_pl[v, ..., 0, 1], Qin_pl[v, ..., 1, 1])
        q_a_pl[v] = cmv * a0 + (1.0 - cmv) * a1
        a2 = clampout(q_a_pl[v], Qout_pl[v, ..., 1], Qout_pl[v, ..., 0])
        a3 = clampout(q_a_pl[v], Qout_pl[0, ..., 1], Qout_pl[0, ..., 0])
        q_a_pl[v] = cmv * a2 + (1.0 - cmv) * a3


def _pymin(a, b):
    return np.where(b < a, b, a)


def _pymax(a, b):
    return np.where(b > a, b, a)


def _reduce(fn, arrs):
    out = arrs[0]
    for a in arrs[1:]:
        out = fn(out, a)
    return out


def tracer_advection(g, rhogq, rhogq_pl, rhog_in, rhog_in_pl, PM, PM_pl, frhog, frhog_pl, dt):
    """mod_src_tracer.py:83-1228 numpy path (Strang V/H/V, b1=0, b2=1, b3=0);
    updates rhogq (i,j,k,l,nq) / rhogq_pl in place."""
    kmin, kmax = g.kmin, g.kmax
    rvx_m, rvy_m, rvz_m, rw_m = (PM[..., I_RHOGVX], PM[..., I_RHOGVY], PM[..., I_RHOGVZ], PM[..., I_RHOGW])
    rvx_mp, rvy_mp, rvz_mp, rw_mp = (PM_pl[..., I_RHOGVX], PM_pl[..., I_RHOGVY], PM_pl[..., I_RHOGVZ],
                                     PM_pl[..., I_RHOGW])
    flx, ck, rhog = _tracer_vert_flux(g, rvx_m, rvy_m, rvz_m, rw_m, rhog_in, frhog, dt, False)
    flxp, ckp, rhogp = _tracer_vert_flux(g, rvx_mp, rvy_mp, rvz_mp, rw_mp, rhog_in_pl, frhog_pl, dt, True)
    b1, b2, b3 = 0.0, 1.0, 1.0 - (0.0 + 1.0)
    d = b1 * frhog / rhog_in * dt
    dp = b1 * frhog_pl / rhog_in_pl * dt
    for iq in range(rhogq.shape[-1]):
        _vertical_advection(g, rhogq[..., iq], rhog_in, flx, ck, d, False, False)
        _vertical_advection(g, rhogq_pl[..., iq], rhog_in_pl, flxp, ckp, dp, True, False)
    # horizontal step
    d = b2 * frhog / rhog * dt
    rvx = rvx_m * g.VMTR_RGAM
    rvy = rvy_m * g.VMTR_RGAM
    rvz = rvz_m * g.VMTR_RGAM
    rvxp = rvx_mp * g.VMTR_RGAM_pl
    rvyp = rvy_mp * g.VMTR_RGAM_pl
    rvzp = rvz_mp * g.VMTR_RGAM_pl
    flx_h, grd_xc, flx_hp, grd_xcp = horizontal_flux(g, PM[..., I_RHOG], rvx, rvy, rvz,
                                                      PM_pl[..., I_RHOG], rvxp, rvyp, rvzp, dt)
    ch = flx_h / rhog[..., None]
    cmask = 0.5 - np.copysign(0.5, ch - g.EPS)
    ch_pl = np.full_like(flx_hp, np.nan)
    cmask_pl = np.full_like(flx_hp, np.nan)
    ch_pl[1:6] = flx_hp[1:6] / rhogp[0]
    cmask_pl[1:6] = 0.5 - np.copysign(0.5, ch_pl[1:6] - g.EPS)
    dp = b2 * frhog_pl / rhogp * dt
    i, j = rhog.shape[:2]
    isl, jsl = slice(1, i - 1), slice(1, j - 1)
    for iq in range(rhogq.shape[-1]):
        q = rhogq[..., iq] / rhog
        q_pl = rhogq_pl[..., iq] / rhogp
        q_a, q_a_pl = horizontal_remap(g, q, q_pl, cmask, cmask_pl, grd_xc, grd_xcp)
        horizontal_limiter(g, q_a, q_a_pl, q, q_pl, d, dp, ch, ch_pl, cmask, cmask_pl)
        rhogq[isl, jsl, :, :, iq] -= (flx_h[isl, jsl, :, :, 0] * q_a[isl, jsl, :, :, 0]
                                      + flx_h[isl, jsl, :, :, 1] * q_a[isl, jsl, :, :, 1]
                                      + flx_h[isl, jsl, :, :, 2] * q_a[isl, jsl, :, :, 2]
                                      + flx_h[isl, jsl, :, :, 3] * q_a[isl, jsl, :, :, 3]
                                      + flx_h[isl, jsl, :, :, 4] * q_a[isl, jsl, :, :, 4]
                                      + flx_h[isl, jsl, :, :, 5] * q_a[isl, jsl, :, :, 5])
        for v in range(1, 6):
            rhogq_pl[0, :, :, iq] -= flx_hp[v] * q_a_pl[v]
    rhog[isl, jsl] -= (flx_h[isl, jsl, :, :, 0] + flx_h[isl, jsl, :, :, 1] + flx_h[isl, jsl, :, :, 2]
                       + flx_h[isl, jsl, :, :, 3] + flx_h[isl, jsl, :, :, 4]
                       + flx_h[isl, jsl, :, :, 5]) - (b2 * frhog[isl, jsl] * dt)
    for v in range(1, 6):
        rhogp[0] -= flx_hp[v]
    rhogp[0] += b2 * frhog_pl[0] * dt
    # second vertical step
    d = b3 * frhog / rhog * dt
    ck = np.zeros_like(ck)
    kc = slice(kmin, kmax + 1)
    rdz = g.GRD_rdgz[kc][:, None]
    ck[:, :, kc, :, 0] = -flx[:, :, kc] / rhog[:, :, kc] * rdz
    ck[:, :, kc, :, 1] = flx[:, :, kmin + 1:kmax + 2] / rhog[:, :, kc] * rdz
    dp = b3 * frhog_pl / rhogp * dt
    ckp = np.zeros_like(ckp)
    for k in range(kmin, kmax + 1):
        ckp[:, k, :, 0] = -flxp[:, k] / rhogp[:, k] * g.GRD_rdgz[k]
        ckp[:, k, :, 1] = flxp[:, k + 1] / rhogp[:, k] * g.GRD_rdgz[k]
    for iq in range(rhogq.shape[-1]):
        _vertical_advection(g, rhogq[..., iq], rhog, flx, ck, d, False, True)
        _vertical_advection(g, rhogq_pl[..., iq], rhogp, flxp, ckp, dp, True, True)


# --------------------------------------------------------------------------
# the large step
# --------------------------------------------------------------------------
def dynamics_step(g, prg, prg_pl, keep=None):
    """mod_dynamics.py:1725-2741 numpy path: one RK3-HEVI large step.
    ``prg (i,j,k,l,6+nq)`` / ``prg_pl (g,k,l,6+nq)`` are not modified; the new
    state is returned (after the final halo exchange).  With a dict ``keep``,
    ``keep["w"]`` receives the diagnostic w of the last RK stage (boundary rows
    as BNDCND left them), the buffer the history diagnostics read."""
    PROG = prg[..., 0:6].copy()
    PROG_pl = prg_pl[..., 0:6].copy()
    PROGq = prg[..., 6:].copy()
    PROGq_pl = prg_pl[..., 6:].copy()
    PROG0 = PROG.copy()
    PROG0_pl = PROG_pl.copy()
    PROG00_rhog = PROG[..., I_RHOG].copy()
    PROG00_rhog_pl = PROG_pl[..., I_RHOG].copy()
    DIAG = np.zeros(PROG.shape)
    DIAG_pl = np.zeros(PROG_pl.shape)
    nstage = len(g.sstep)
    large_dt = g.dtl
    for nl in range(nstage):
        rho, ein, q, rho_pl, ein_pl, q_pl = diagnostics(g, PROG, PROGq, DIAG, PROG_pl, PROGq_pl, DIAG_pl)
        bndcnd_all(g, DIAG, PROG, rho, ein)
        bndcnd_all(g, DIAG_pl, PROG_pl, rho_pl, ein_pl, pole=True)
        eth = ein + DIAG[..., I_pre] / rho
        eth_pl = ein_pl + DIAG_pl[..., I_pre] / rho_pl
        pregd = (DIAG[..., I_pre] - g.pre_bs) * g.VMTR_GSGAM2
        rhogd = (rho - g.rho_bs) * g.VMTR_GSGAM2
        pregd_pl = (DIAG_pl[..., I_pre] - g.pre_bs_pl) * g.VMTR_GSGAM2_pl
        rhogd_pl = (rho_pl - g.rho_bs_pl) * g.VMTR_GSGAM2_pl
        adv, adv_pl = advection_momentum(g, DIAG, PROG, DIAG_pl, PROG_pl)
        g_TEND = np.zeros(PROG.shape)
        g_TEND_pl = np.zeros(PROG_pl.shape)
        for n, iv in enumerate((I_RHOGVX, I_RHOGVY, I_RHOGVZ, I_RHOGW)):
            g_TEND[..., iv] = adv[n]
            g_TEND_pl[..., iv] = adv_pl[n]
        f_TEND, f_TEND_pl = hdiffusion(g, PROG[..., I_RHOG], rho, DIAG, PROG_pl[..., I_RHOG], rho_pl, DIAG_pl)
        if "rayleigh_coef" in g.d:
            rayleigh_damping(g, f_TEND, f_TEND_pl, PROG[..., I_RHOG], PROG_pl[..., I_RHOG], DIAG, DIAG_pl)
        g_TEND = g_TEND + f_TEND
        g_TEND_pl = g_TEND_pl + f_TEND_pl
        if nl == 0:
            PROG_split = np.zeros(PROG.shape)
            PROG_split_pl = np.zeros(PROG_pl.shape)
        else:
            PROG_split = PROG0 - PROG
            PROG_split_pl = PROG0_pl - PROG_pl
        PM, PM_pl = vi_small_step(g, PROG, PROG_pl, DIAG, DIAG_pl, eth, eth_pl, rhogd, rhogd_pl,
                                  pregd, pregd_pl, g_TEND, g_TEND_pl, PROG_split, PROG_split_pl,
                                  g.sstep[nl], g.dts)
        if nl != nstage - 1:
            comm(g, PROG, PROG_pl)
        else:
            tracer_advection(g, PROGq, PROGq_pl, PROG00_rhog, PROG00_rhog_pl, PM, PM_pl,
                             f_TEND[..., I_RHOG], f_TEND_pl[..., I_RHOG], large_dt)
            PROGq += large_dt * np.zeros_like(PROGq)
            PROGq_pl += large_dt * np.zeros_like(PROGq_pl)
    out = np.concatenate([PROG, PROGq], axis=-1)
    out_pl = np.concatenate([PROG_pl, PROGq_pl], axis=-1)
    comm(g, out, out_pl)
    if keep is not None:
        keep["w"] = DIAG[..., I_w].copy()
    return out, out_pl


# --------------------------------------------------------------------------
# Held-Suarez artificial forcing  (Dyn.forcing_step, AF_TYPE 'HELD-SUAREZ')
# --------------------------------------------------------------------------
HS_SIGMA_B = 0.7                        # forcing/mod_af_heldsuarez.py:19-24 (dry case, :31-36)
HS_KF = 1.0 / (1.0 * 86400.0)
HS_DTH_Z = 10.0
HS_KA = 1.0 / (40.0 * 86400.0)
HS_KS = 1.0 / (4.0 * 86400.0)
HS_T_EQ0 = 315.0
HS_DT_Y = 60.0


def hs_latitude_terms(lat):
    """|sin(lat)|**2, |cos(lat)|**2 and |cos(lat)|**4 of the column latitudes,
    with the reference's numpy expressions (mod_af_heldsuarez.py:61-63)."""
    sinlat = np.abs(np.sin(lat))
    coslat = np.abs(np.cos(lat))
    return sinlat ** 2, coslat ** 2, coslat ** 4


def held_suarez(g, lat, pre, tem, vx, vy, vz, moist=False):
    """forcing/mod_af_heldsuarez.py:38-88 AF_heldsuarez: tendencies
    (fvx, fvy, fvz, fe) on regional (i,j,k,l) fields, zero outside kmin..kmax;
    ``moist`` takes the moist case's equilibrium profile (T_eq0 294 K,
    DT_y 65 K; AF_heldsuarez_init :31-39)."""
    T_eq0, DT_y = (294.0, 65.0) if moist else (HS_T_EQ0, HS_DT_Y)
    kmin, kmax = g.kmin, g.kmax
    sin2, cos2, cos4 = (t[:, :, None, :] for t in hs_latitude_terms(lat))
    psref = (0.5 * (pre[:, :, kmin, :] + pre[:, :, kmin - 1, :]))[:, :, None, :]
    sigma = pre / psref
    factor = np.maximum((sigma - HS_SIGMA_B) / (1.0 - HS_SIGMA_B), 0.0)
    fvx = -HS_KF * factor * vx
    fvy = -HS_KF * factor * vy
    fvz = -HS_KF * factor * vz
    ap0 = np.abs(pre / g.PRE00)
    Kt = HS_KA + (HS_KS - HS_KA) * factor * cos4
    T_eq = np.maximum(200.0, (T_eq0 - DT_y * sin2
                              - HS_DTH_Z * np.log(np.maximum(ap0, 1e-30)) * cos2) * ap0 ** (g.Rdry / g.CPdry))
    fe = -Kt * (tem - T_eq) * g.CVdry
    kk = np.arange(pre.shape[2]).reshape(1, 1, -1, 1)
    valid = (kk >= kmin) & (kk <= kmax)
    return tuple(np.where(valid, f, 0.0) for f in (fvx, fvy, fvz, fe))


def forcing_step_hs(g, prg, prg_pl, lat):
    """Dyn.forcing_step for AF_TYPE 'HELD-SUAREZ' on the host path
    (nhm/dynamics/mod_dynamics.py:597-735): diagnostics of the regional
    prognostic, the Held-Suarez tendencies applied as
    PROG + dt * f * rho * GSGAM2 (nhm/forcing/mod_forcing.py:14-28
    hs_apply_core, :323-349 forcing_step_hs; no forcing of RHOG, RHOGW, the
    tracers or the poles), then the halo exchange of the whole PRG_var.
    ``lat`` is GRD_LAT[:, :, K0, :] (i, j, l).  Returns new arrays."""
    out = prg.copy()
    out_pl = prg_pl.copy()
    PROG = out[..., 0:6]
    PROGq = out[..., 6:]
    DIAG = np.zeros(PROG.shape)
    rho, _ein, _q, _, _, _ = diagnostics(g, PROG, PROGq, DIAG, prg_pl[..., 0:6].copy(), prg_pl[..., 6:].copy(),
                                          np.zeros(prg_pl[..., 0:6].shape))
    fvx, fvy, fvz, fe = held_suarez(g, lat, DIAG[..., I_pre], DIAG[..., I_tem], DIAG[..., I_vx], DIAG[..., I_vy],
                                    DIAG[..., I_vz])
    dt = g.dtl
    z = np.zeros_like(fvx)
    comps = [z] * 6
    comps[I_RHOGVX] = dt * fvx * rho * g.VMTR_GSGAM2
    comps[I_RHOGVY] = dt * fvy * rho * g.VMTR_GSGAM2
    comps[I_RHOGVZ] = dt * fvz * rho * g.VMTR_GSGAM2
    comps[I_RHOGE] = dt * fe * rho * g.VMTR_GSGAM2
    out[..., 0:6] = PROG + np.stack(comps, axis=-1)
    comm(g, out, out_pl)
    return out, out_pl


# --------------------------------------------------------------------------
# DCMIP forcing with Kessler warm-rain microphysics only (AF_TYPE 'DCMIP',
# USE_Kessler; the scheme set of DCMIP2016 case 1-3)
# --------------------------------------------------------------------------
def kessler(theta, qv, qc, qr, rho, pk, dt, z):
    """nhm/forcing/kessler.py:9-179 on (ncol, nz) columns ordered surface to
    top: potential temperature, dry mixing ratios, dry density, Exner
    function, heights.  Returns the updated theta, qv, qc, qr and the
    precipitation rate per column.  Rain sedimentation is sub-cycled per
    column (CFL 0.8); columns with fewer sub-cycles are left unchanged in the
    later ones."""
    f2x = 17.27
    f5 = 237.3 * f2x * 2500000.0 / 1003.0
    xk = 0.2875
    psl = 1000.0
    rhoqr = 1000.0
    theta, qv, qc, qr = theta.copy(), qv.copy(), qc.copy(), qr.copy()
    r = 0.001 * rho
    rhalf = np.sqrt(rho[:, 0:1] / rho)
    pc = 3.8 / (pk ** (1.0 / xk) * psl)
    velqr = 36.34 * (qr * r) ** 0.1364 * rhalf
    dz = z[:, 1:] - z[:, :-1]
    vk = velqr[:, :-1]
    vk_safe = np.where(vk != 0.0, vk, 1.0)
    cfl = np.where(vk != 0.0, 0.8 * dz / vk_safe, dt)
    dt_max = np.minimum(dt, cfl.min(axis=1))
    rainsplit = np.ceil(dt / dt_max).astype(np.int32)
    dt0 = dt / rainsplit.astype(np.float64)
    dt0c = dt0[:, None]
    precl = np.zeros(theta.shape[0])
    for nt in range(1, int(rainsplit.max()) + 1):
        active = nt <= rainsplit
        am = active[:, None]
        precl = precl + np.where(active, rho[:, 0] * qr[:, 0] * velqr[:, 0] / rhoqr, 0.0)
        num = r[:, 1:] * qr[:, 1:] * velqr[:, 1:] - r[:, :-1] * qr[:, :-1] * velqr[:, :-1]
        sed_int = dt0c * num / (r[:, :-1] * dz)
        sed_top = -dt0 * qr[:, -1] * velqr[:, -1] / (0.5 * (z[:, -1] - z[:, -2]))
        sed = np.concatenate([sed_int, sed_top[:, None]], axis=1)
        qc0, qr0, qv0, th0 = qc, qr, qv, theta
        qrprod = qc0 - (qc0 - dt0c * np.maximum(0.001 * (qc0 - 0.001), 0.0)) / (1.0 + dt0c * 2.2 * qr0 ** 0.875)
        qc1 = np.maximum(qc0 - qrprod, 0.0)
        qr1 = np.maximum(qr0 + qrprod + sed, 0.0)
        pkt = pk * th0
        qvs = pc * np.exp(f2x * (pkt - 273.0) / (pkt - 36.0))
        prod = (qv0 - qvs) / (1.0 + qvs * f5 / (pkt - 36.0) ** 2)
        rqr = r * qr1
        ern = np.minimum(np.minimum(
            dt0c * (((1.6 + 124.9 * rqr ** 0.2046) * rqr ** 0.525) / (2550000.0 * pc / (3.8 * qvs) + 540000.0))
            * (np.maximum(qvs - qv0, 0.0) / (r * qvs)),
            np.maximum(-prod - qc1, 0.0)), qr1)
        mpc = np.maximum(prod, -qc1)
        th_new = th0 + 2500000.0 / (1003.0 * pk) * (mpc - ern)
        qv_new = np.maximum(qv0 - mpc + ern, 0.0)
        qc_new = qc1 + mpc
        qr_new = qr1 - ern
        theta = np.where(am, th_new, th0)
        qv = np.where(am, qv_new, qv0)
        qc = np.where(am, qc_new, qc0)
        qr = np.where(am, qr_new, qr0)
        velqr = np.where((nt < rainsplit)[:, None], 36.34 * (qr * r) ** 0.1364 * rhalf, velqr)
    return theta, qv, qc, qr, precl / rainsplit.astype(np.float64)


def terminator_tendency(lat_deg, lon_deg, cl, cl2, dt):
    """nhm/forcing/terminator.py:20-70 tendency_terminator: the Cl / Cl2
    photolysis-recombination rates (k1 from the solar zenith projection
    toward 20 N, 300 E, k2 = 1) integrated analytically over dt; returns
    (cl_f, cl2_f) per second, cl2_f = -cl_f / 2"""
    d2r = np.pi / 180.0
    lat_c, lon_c = 20.0 * d2r, 300.0 * d2r
    la, lo = lat_deg * d2r, lon_deg * d2r
    k1 = np.maximum(0.0, np.sin(la) * np.sin(lat_c) + np.cos(la) * np.cos(lat_c) * np.cos(lo - lon_c))
    k2 = 1.0
    r = k1 / (4.0 * k2)
    cly = cl + 2.0 * cl2
    det = np.sqrt(r * r + 2.0 * r * cly)
    expdt = np.exp(-4.0 * k2 * det * dt)
    mask = np.abs(det * k2 * dt) > 1.0e-16
    det_safe = np.where(mask, det, np.ones_like(det))
    el = np.where(mask, (1.0 - expdt) / det_safe / dt, np.full_like(det, 4.0 * k2))
    cl_f = -el * (cl - det + r) * (cl + det + r) / (1.0 + expdt + dt * el * (cl + r))
    return cl_f, -cl_f / 2.0


# DCMIP simple physics (nhm/forcing/simple_physics.py; DCMIP2016 v6 scheme):
# constants of simple_physics.py:25-46 (use_HS off)
SP_RAIR, SP_RH2O, SP_GRAV, SP_CPAIR, SP_LATVAP = 287.0, 461.5, 9.80616, 1.0045e3, 2.5e6
SP_EPSILO, SP_ZVIR = SP_RAIR / SP_RH2O, (SP_RH2O / SP_RAIR) - 1.0
SP_C, SP_T0, SP_E0, SP_RHOW = 0.0011, 273.16, 610.78, 1000.0
SP_CD0, SP_CD1, SP_CM, SP_V20 = 0.0007, 0.000065, 0.002, 20.0
SP_P0, SP_PBLTOP, SP_PBLCONST = 100000.0, 85000.0, 10000.0


def dcmip_sst(lat, latdepend, held_suarez=False, mitc_type=1):
    """simple_physics.py:152-197 _sst_tsurf: for moist Held-Suarez the
    Gaussian-in-latitude SST of MITC type 1-3; otherwise the latitude-dependent
    sea-surface temperature of the moist baroclinic wave (test 1) or the
    constant 302.15 K of the tropical cyclone (test 0)"""
    import math
    pi = math.pi
    if held_suarez:
        if mitc_type == 1:
            return 29.0 * np.exp(-0.5 * lat * lat / (26.0 / 180.0 * pi) ** 2) + 271.0
        amp, w, c0 = (29.0, 20.0, 17.0) if mitc_type == 2 else (32.0, 23.0, 12.0)
        return amp * np.exp(-0.5 * np.maximum(np.abs(lat) - (c0 / 180.0 * pi), 0.0) ** 2 / (w / 180.0 * pi) ** 2) + 271.0
    if not latdepend:
        return np.full_like(lat, 302.15)
    T00, u0, a, omega, q0, eta0 = 288.0, 35.0, 6371220.0, 7.29212e-5, 0.021, 0.252
    etav, latw = (1.0 - eta0) * 0.5 * pi, 2.0 * pi / 9.0
    sinl, cosl = np.sin(lat), np.cos(lat)
    termA = (-2.0 * sinl ** 6 * (cosl ** 2 + 1.0 / 3.0) + 10.0 / 63.0) * u0 * (math.cos(etav)) ** 1.5
    termB = (8.0 / 5.0 * cosl ** 3 * (sinl ** 2 + 2.0 / 3.0) - pi / 4.0) * a * omega * 0.5
    pref = pi * u0 / SP_RAIR * 1.5 * math.sin(etav) * (math.cos(etav)) ** 0.5
    return (T00 + pref * (termA + termB)) / (1.0 + SP_ZVIR * q0 * np.exp(-(lat / latw) ** 4))


def simple_physics(t, q, u, v, pmid, pint, pdel, rpdel, ps, tsurf, dtime, lsc, Cexch=SP_C, bryan=False):
    """simple_physics.py:310-366 (RJ2012 boundary layer, no Held-Suarez) on
    (ncol, nz) columns ordered top to bottom: the lowest full level's
    hydrostatic height, the large-scale condensation (lsc, :48-91), the
    drag / diffusivities from the lowest-level wind (:118-149), the implicit
    bulk surface fluxes of the lowest level (:200-225) and the implicit
    boundary-layer diffusion of u, v, potential temperature and q
    (:228-307).  ``Cexch`` is the heat / moisture exchange coefficient
    (four times 0.0011 for moist Held-Suarez); ``bryan`` takes the
    height-based boundary layer of the tropical-cyclone test (TC_PBL_mod).
    Returns t, q, u, v and the condensation's precipitation."""
    ncol, nz = t.shape
    dlnpint = np.log(ps) - np.log(pint[:, nz - 1])
    za = SP_RAIR / SP_GRAV * t[:, -1] * (1.0 + SP_ZVIR * q[:, -1]) * 0.5 * dlnpint
    if lsc:
        qsat = SP_EPSILO * SP_E0 / pmid * np.exp(-SP_LATVAP / SP_RH2O * ((1.0 / t) - 1.0 / SP_T0))
        denom = 1.0 + (SP_LATVAP / SP_CPAIR) * (SP_EPSILO * SP_LATVAP * qsat / (SP_RAIR * t * t))
        cond = np.where(q > qsat, (1.0 / dtime) * (q - qsat) / denom, 0.0)
        t = t + (SP_LATVAP / SP_CPAIR) * cond * dtime
        q = q - cond * dtime
        precl = np.sum(cond * pdel / (SP_GRAV * SP_RHOW), axis=1)
    else:
        precl = np.zeros(ncol)
    wind = np.sqrt(u[:, -1] ** 2 + v[:, -1] ** 2)
    Cd = np.where(wind < SP_V20, SP_CD0 + SP_CD1 * wind, SP_CM)
    if bryan:   # :128-141, the height-based boundary layer of the tropical-cyclone test
        Km, Ke = np.zeros((ncol, nz)), np.zeros((ncol, nz))
        zi = np.zeros(ncol)
        with np.errstate(divide="ignore", invalid="ignore"):
            for c in range(nz - 1, -1, -1):
                dlnpint = np.log(pint[:, c + 1]) - np.log(pint[:, c])
                zi = zi + SP_RAIR / SP_GRAV * t[:, c] * (1.0 + SP_ZVIR * q[:, c]) * dlnpint
                below = zi <= 1000.0
                fac = 1.0 - zi / 1000.0
                base = wind * zi * fac * fac
                Km[:, c] = np.where(below, 0.4 * np.sqrt(Cd) * base, 0.0)
                Ke[:, c] = np.where(below, 0.4 * np.sqrt(Cexch) * base, 0.0)
    else:
        decay = np.where(pint[:, 0:nz] >= SP_PBLTOP, 1.0, np.exp(-(SP_PBLTOP - pint[:, 0:nz]) ** 2 / SP_PBLCONST ** 2))
        Km = (Cd * wind * za)[:, None] * decay
        Ke = (Cexch * wind * za)[:, None] * decay
    # surface fluxes, lowest level only
    qsats = SP_EPSILO * SP_E0 / ps * np.exp(-SP_LATVAP / SP_RH2O * ((1.0 / tsurf) - 1.0 / SP_T0))
    dm = 1.0 + Cd * wind * dtime / za
    dh = 1.0 + Cexch * wind * dtime / za
    u, v, t, q = u.copy(), v.copy(), t.copy(), q.copy()
    u[:, -1] = u[:, -1] / dm
    v[:, -1] = v[:, -1] / dm
    t[:, -1] = (t[:, -1] + Cexch * wind * tsurf * dtime / za) / dh
    q[:, -1] = (q[:, -1] + Cexch * wind * qsats * dtime / za) / dh
    # implicit vertical diffusion: coefficients at the interfaces between levels c and c+1
    kap = SP_RAIR / SP_CPAIR
    g2dt = dtime * SP_GRAV * SP_GRAV
    rho = pint[:, 1:nz] / (SP_RAIR * (t[:, 1:nz] * (1.0 + SP_ZVIR * q[:, 1:nz])
                                      + t[:, 0:nz - 1] * (1.0 + SP_ZVIR * q[:, 0:nz - 1])) / 2.0)
    dpm = pmid[:, 1:nz] - pmid[:, 0:nz - 1]
    fm = g2dt * Km[:, 1:nz] * rho * rho / dpm
    fe = g2dt * Ke[:, 1:nz] * rho * rho / dpm
    CAm, CCm, CA, CC = (np.zeros((ncol, nz)) for _ in range(4))
    CAm[:, 0:nz - 1] = rpdel[:, 0:nz - 1] * fm
    CCm[:, 1:nz] = rpdel[:, 1:nz] * fm
    CA[:, 0:nz - 1] = rpdel[:, 0:nz - 1] * fe
    CC[:, 1:nz] = rpdel[:, 1:nz] * fe
    CE, CEm, CFu, CFv, CFt, CFq = (np.zeros((ncol, nz)) for _ in range(6))
    ce = cem = cfu = cfv = cft = cfq = np.zeros(ncol)
    for c in range(nz - 1, -1, -1):   # upward elimination
        de = 1.0 + CA[:, c] + CC[:, c] - CA[:, c] * ce
        dmm = 1.0 + CAm[:, c] + CCm[:, c] - CAm[:, c] * cem
        ce, cem = CC[:, c] / de, CCm[:, c] / dmm
        cfu = (u[:, c] + CAm[:, c] * cfu) / dmm
        cfv = (v[:, c] + CAm[:, c] * cfv) / dmm
        cft = ((SP_P0 / pmid[:, c]) ** kap * t[:, c] + CA[:, c] * cft) / de
        cfq = (q[:, c] + CA[:, c] * cfq) / de
        CE[:, c], CEm[:, c], CFu[:, c], CFv[:, c], CFt[:, c], CFq[:, c] = ce, cem, cfu, cfv, cft, cfq
    uo, vo, to, qo = (np.zeros((ncol, nz)) for _ in range(4))
    uo[:, 0], vo[:, 0] = CFu[:, 0], CFv[:, 0]
    to[:, 0] = CFt[:, 0] * (pmid[:, 0] / SP_P0) ** kap
    qo[:, 0] = CFq[:, 0]
    for c in range(1, nz):            # downward substitution
        uo[:, c] = CEm[:, c] * uo[:, c - 1] + CFu[:, c]
        vo[:, c] = CEm[:, c] * vo[:, c - 1] + CFv[:, c]
        to[:, c] = (CE[:, c] * to[:, c - 1] * (SP_P0 / pmid[:, c - 1]) ** kap + CFt[:, c]) * (pmid[:, c] / SP_P0) ** kap
        qo[:, c] = CE[:, c] * qo[:, c - 1] + CFq[:, c]
    return to, qo, uo, vo, precl


def forcing_step_kessler(g, prg, prg_pl, zf, negative_fixer=False, update_tot_dens=True, chem=None,
                         kessler_on=True, sm=None):
    """Dyn.forcing_step for AF_TYPE 'DCMIP' with Kessler microphysics only
    (nhm/dynamics/mod_dynamics.py:597-735 -> nhm/forcing/mod_forcing.py:207-321
    forcing_step -> mod_af_dcmip.py:129-230 AF_dcmip, Kessler branch):
    diagnostics of the regional prognostic (water tracers 0, 1, 2 = vapour,
    cloud, rain), dry mixing ratios and density, Exner function and
    potential temperature on kmin..kmax, the microphysics, the tracer and
    energy tendencies (the energy one from increments), applied as
    PROG + dt * f * rho * GSGAM2 with the water tendencies also added to
    RHOG (update_tot_dens), then the halo exchange of PRG_var.  ``zf`` is
    GRD_vz[..., GRD_Z] (i, j, k, l).  ``chem`` = (lat, lon, nchem_str,
    nchem_end) adds the terminator toy chemistry (mod_af_dcmip.py:171-187;
    lat, lon of the columns in radians (i, j, l)) on the Cl / Cl2 tracers.
    ``sm`` = dict(zh, zsfc, lat, ij, latdepend, lsc) adds the simple physics
    (mod_af_dcmip.py:230-317) from the same (old) state: half-level heights
    GRD_vz[..., GRD_ZH], the surface height and latitude (i, j, l), the
    column unit vectors GMTR_p IX..JZ (i, j, l, 6), the sea-surface
    temperature form and the large-scale condensation switch; its momentum,
    vapour and energy tendencies add to Kessler's (``kessler_on`` False
    leaves the simple physics alone).  With sm["held_suarez"] (and
    sm["mitc"], the SST type) the moist Held-Suarez case: the simple physics
    with the exchange coefficient x4 and the Held-Suarez SST, and the
    Held-Suarez relaxation on top, its momentum tendency replacing the
    others', its energy tendency added (mod_forcing.py:278-287).  Returns
    (prg, prg_pl, precip (i, j, l))."""
    out = prg.copy()
    out_pl = prg_pl.copy()
    PROG = out[..., 0:6]
    PROGq = out[..., 6:]
    DIAG = np.zeros(PROG.shape)
    rho, ein, q, _, _, _ = diagnostics(g, PROG, PROGq, DIAG, prg_pl[..., 0:6].copy(), prg_pl[..., 6:].copy(),
                                       np.zeros(prg_pl[..., 0:6].shape))
    pre, tem = DIAG[..., I_pre], DIAG[..., I_tem]
    if negative_fixer:
        q = np.maximum(q, 0.0)
    kmin, kmax = g.kmin, g.kmax
    I, J, K, L = rho.shape
    sl = slice(kmin, kmax + 1)
    dt = g.dtl
    col = lambda a: a.transpose(0, 1, 3, 2).reshape(I * J * L, K)[:, sl]      # (ncol, levels kmin..kmax)
    warm = g.nqw == 3   # RAIN_TYPE WARM (vapour, cloud, rain) or DRY (vapour only)
    qv_m = col(q[..., 0])
    if warm:
        qc_m, qr_m = col(q[..., 1]), col(q[..., 2])

    def grid(c):   # (ncol, levels kmin..kmax) -> (i, j, k, l), zero outside kmin..kmax
        full = np.zeros((I * J * L, K))
        full[:, sl] = c
        return full.reshape(I, J, L, K).transpose(0, 1, 3, 2)
    zero = np.zeros(rho.shape)
    fe, fv = zero, [zero, zero, zero]
    nwq = 3 if warm else 1
    fq = [zero] * nwq + [None] * (PROGq.shape[-1] - nwq)
    precl = np.zeros(I * J * L)
    if kessler_on:
        qd = 1.0 - qv_m - qc_m - qr_m
        qvk, qck, qrk = qv_m / qd, qc_m / qd, qr_m / qd
        rhod = col(rho) * qd
        pk = (col(pre) / g.PRE00) ** (g.Rdry / g.CPdry)
        theta_k = col(tem) / pk
        theta_k, qvk, qck, qrk, prk = kessler(theta_k, qvk, qck, qrk, rhod, pk, dt, col(zf))
        qd2 = 1.0 / (1.0 + qvk + qck + qrk)
        qvk, qck, qrk = qvk * qd2, qck * qd2, qrk * qd2
        cvk = qd2 * g.CVdry + qvk * g.CVW[0] + qck * g.CVW[1] + qrk * g.CVW[2]
        tem_new = theta_k * pk
        tem_old = col(tem)
        cv_old = col(ein) / tem_old
        dtem = tem_new - tem_old
        dcv = cvk - cv_old
        fe = fe + grid((cv_old * dtem + tem_old * dcv + dcv * dtem) / dt)
        fq = [fq[0] + grid((qvk - qv_m) / dt), fq[1] + grid((qck - qc_m) / dt),
              fq[2] + grid((qrk - qr_m) / dt)] + fq[3:]
        precl = precl + prk
    if sm is not None:
        td = lambda a: col(a)[:, ::-1]            # levels kmax..kmin (top down)
        flat = lambda a: a.reshape(I * J * L)
        ij = [flat(sm["ij"][..., n]) for n in range(6)]
        tem_td, pre_td, alt_td, alth_td = td(tem), td(pre), td(zf), td(sm["zh"])
        vx_td, vy_td, vz_td, ein_td = td(DIAG[..., I_vx]), td(DIAG[..., I_vy]), td(DIAG[..., I_vz]), td(ein)
        qv_old = td(q[..., 0])
        u = vx_td * ij[0][:, None] + vy_td * ij[1][:, None] + vz_td * ij[2][:, None]
        v = vx_td * ij[3][:, None] + vy_td * ij[4][:, None] + vz_td * ij[5][:, None]
        nz = kmax - kmin + 1
        pre_sfc = flat(pre[:, :, kmin, :] + rho[:, :, kmin, :] * g.GRAV * (zf[:, :, kmin, :] - sm["zsfc"]))
        pint = np.zeros((I * J * L, nz + 1))
        pint[:, 1:nz] = pre_td[:, 1:nz] * np.exp(np.log(pre_td[:, 0:nz - 1] / pre_td[:, 1:nz])
                                                 * (alth_td[:, 0:nz - 1] - alt_td[:, 1:nz])
                                                 / (alt_td[:, 0:nz - 1] - alt_td[:, 1:nz]))
        pint[:, nz] = pre_sfc
        pdel = pint[:, 1:nz + 1] - pint[:, 0:nz]
        hs = bool(sm.get("held_suarez", False))
        tsurf = dcmip_sst(flat(sm["lat"]), sm["latdepend"], hs, sm.get("mitc", 1))
        t_n, qv_n, u_n, v_n, pr2 = simple_physics(tem_td, qv_old, u, v, pre_td, pint, pdel, 1.0 / pdel, pre_sfc,
                                                  tsurf, dt, sm["lsc"], SP_C * (4.0 if hs else 1.0),
                                                  bryan=bool(sm.get("bryan", False)))
        for d, (a, b, vd) in enumerate(((0, 3, vx_td), (1, 4, vy_td), (2, 5, vz_td))):
            fv[d] = grid(((u_n * ij[a][:, None] + v_n * ij[b][:, None] - vd) / dt)[:, ::-1])
        if warm:   # mod_af_dcmip.py:486-499
            qc, qr = td(q[..., 1]), td(q[..., 2])
            qd = 1.0 - qv_n - qc - qr
            cv = qd * g.CVdry + qv_n * g.CVW[0] + qc * g.CVW[1] + qr * g.CVW[2]
        else:
            qd = 1.0 - qv_n
            cv = qd * g.CVdry + qv_n * g.CVW[0]
        cv_old = ein_td / tem_td
        dtem = t_n - tem_td
        dcv = cv - cv_old
        fq[0] = fq[0] + grid(((qv_n - qv_old) / dt)[:, ::-1])
        fe = fe + grid(((cv_old * dtem + tem_td * dcv + dcv * dtem) / dt)[:, ::-1])
        precl = precl + pr2
        if hs:
            hfvx, hfvy, hfvz, hfe = held_suarez(g, sm["lat"], pre, tem, DIAG[..., I_vx], DIAG[..., I_vy],
                                                DIAG[..., I_vz], moist=True)
            fv = [hfvx, hfvy, hfvz]
            fe = fe + hfe
    if chem is not None:
        lat, lon, n_cl, n_cl2 = chem
        d2r = np.pi / 180.0
        lat_deg = (lat.reshape(I * J * L) / d2r)[:, None]
        lon_deg = (lon.reshape(I * J * L) / d2r)[:, None]
        qvd = 1.0 - qv_m
        cl_f, cl2_f = terminator_tendency(lat_deg, lon_deg, col(q[..., n_cl]) / qvd, col(q[..., n_cl2]) / qvd, dt)
        fq[n_cl] = grid(cl_f * qvd)
        fq[n_cl2] = grid(cl2_f * qvd)
    GS = g.VMTR_GSGAM2
    new = PROG.copy()
    for d, v in enumerate((I_RHOGVX, I_RHOGVY, I_RHOGVZ)):
        new[..., v] = PROG[..., v] + dt * fv[d] * rho * GS
    new[..., I_RHOGE] = PROG[..., I_RHOGE] + dt * fe * rho * GS
    rhog = PROG[..., I_RHOG]
    for n in range(PROGq.shape[-1]):
        f = fq[n] if fq[n] is not None else zero
        frhogq = f * rho * GS
        if negative_fixer:
            tmp = np.maximum(PROGq[..., n] + dt * frhogq, 0.0)
            frhogq = (tmp - PROGq[..., n]) / dt
            PROGq[..., n] = tmp
        else:
            PROGq[..., n] = PROGq[..., n] + dt * frhogq
        if update_tot_dens and n < g.nqw:
            rhog = rhog + dt * frhogq
    new[..., I_RHOG] = rhog
    out[..., 0:6] = new
    comm(g, out, out_pl)
    return out, out_pl, precl.reshape(I, J, L)


# --------------------------------------------------------------------------
# offline tracer advection  (integ_type TRCADV, DCMIP2012 test 1-1)
# --------------------------------------------------------------------------
TRC_A, TRC_RD, TRC_G, TRC_PI = 6371220.0, 287.0, 9.80616, 3.141592653589793238   # mod_af_trcadv.py:14-19


def trcadv_winds12(time, lon, lat, zf, zh):
    """nhm/forcing/mod_af_trcadv.py:100-149 test12_velocity (DCMIP2012 test
    1-2, Hadley-like meridional circulation) with Sp_Unit_East /
    Sp_Unit_North: winds (vx, vy, vz) at full levels and w at half levels"""
    tau, u0, w0, T0 = 1.0 * 86400.0, 40.0, 0.15, 300.0
    H = TRC_RD * T0 / TRC_G
    K, ztop, p0, pi = 5.0, 12.0e3, 1000.e2, TRC_PI
    rho0 = p0 / (TRC_RD * T0)
    rho = p0 * np.exp(-zf / H) / (TRC_RD * T0)
    u = u0 * np.cos(lat)
    v = (-(rho0 / rho) * TRC_A * w0 * pi / (K * ztop) * np.cos(lat) * np.sin(K * lat)
         * np.cos(pi * zf / ztop) * np.cos(pi * time / tau))
    e0, e1, e2 = -np.sin(lon), np.cos(lon), np.zeros_like(lon)
    n0, n1, n2 = -np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)
    vx = e0 * u + n0 * v
    vy = e1 * u + n1 * v
    vz = e2 * u + n2 * v
    rho = p0 * np.exp(-zh / H) / (TRC_RD * T0)
    w = ((rho0 / rho) * (w0 / K) * (-2.0 * np.sin(K * lat) * np.sin(lat) + K * np.cos(lat) * np.cos(K * lat))
         * np.sin(pi * zh / ztop) * np.cos(pi * time / tau))
    return vx, vy, vz, w


def trcadv_winds(time, lon, lat, zf, zh, case="1-1"):
    """nhm/forcing/mod_af_trcadv.py:22-97 test11_velocity with
    Sp_Unit_East / Sp_Unit_North (:151-171): winds (vx, vy, vz) at full levels
    and w at half levels at model time ``time``; ``lon``/``lat`` broadcast
    against the heights.  ``case`` "1-2" takes test12_velocity instead."""
    if case == "1-2":
        return trcadv_winds12(time, lon, lat, zf, zh)
    tau = 12.0 * 86400.0
    u0 = 2.0 * TRC_PI * TRC_A / tau
    k0 = 10.0 * TRC_A / tau
    omega0 = 23000.0 * TRC_PI / tau
    T0 = 300.0
    H = TRC_RD * T0 / TRC_G
    p0 = 1000.E2
    dlon = 2.0 * TRC_PI * time / tau
    lonp = lon - dlon
    bs = 0.2
    p = p0 * np.exp(-zf / H)
    ptop = p0 * np.exp(-12000.0 / H)
    ud = (omega0 * TRC_A) / (bs * ptop) * np.cos(lonp) * np.cos(lat) ** 2 * np.cos(dlon) * (
        -np.exp((p - p0) / (bs * ptop)) + np.exp((ptop - p) / (bs * ptop)))
    u = k0 * np.sin(2.0 * lat) * np.sin(lonp) ** 2 * np.cos(0.5 * dlon) + u0 * np.cos(lat) + ud
    v = k0 * np.sin(2.0 * lonp) * np.cos(lat) * np.cos(0.5 * dlon)
    e0, e1, e2 = -np.sin(lon), np.cos(lon), np.zeros_like(lon)
    n0, n1, n2 = -np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)
    vx = e0 * u + n0 * v
    vy = e1 * u + n1 * v
    vz = e2 * u + n2 * v
    p = p0 * np.exp(-zh / H)
    s = (1.0 + np.exp((ptop - p0) / (bs * ptop)) - np.exp((p - p0) / (bs * ptop)) - np.exp((ptop - p) / (bs * ptop)))
    w = -(TRC_RD * T0) / (TRC_G * p) * omega0 * np.sin(lonp) * np.cos(lat) * np.cos(dlon) * s
    return vx, vy, vz, w


def trcadv_step(g, prg, prg_pl, time, lon, lat, zf, zh, lon_pl, lat_pl, zf_pl, zh_pl, case="1-1"):
    """Dyn.dynamics_step for integ_type TRCADV (mod_dynamics.py:2030-2085 and
    the marshal-out :2690-2727): the tracers are advected with the current
    PROG as the mean state (rhog_in = PROG0 rhog, no density tendency), then
    the prescribed winds of model time ``time`` are set as wind * RHOG
    (nhm/forcing/mod_forcing.py:113-210 forcing_update), then PRG_var is
    exchanged.  ``lon``/``lat`` are GRD_LON/GRD_LAT[:, :, K0, :] (i,j,l),
    ``zf``/``zh`` the full/half-level heights (i,j,k,l); the pole arrays are
    (g,l) and (g,k,l).  Returns new arrays."""
    out = prg.copy()
    out_pl = prg_pl.copy()
    PROG, PROGq = out[..., 0:6], out[..., 6:]
    PROG_pl, PROGq_pl = out_pl[..., 0:6], out_pl[..., 6:]
    rhog_in = PROG[..., I_RHOG].copy()
    rhog_in_pl = PROG_pl[..., I_RHOG].copy()
    tracer_advection(g, PROGq, PROGq_pl, rhog_in, rhog_in_pl, PROG[..., 0:5].copy(), PROG_pl[..., 0:5].copy(),
                     np.zeros_like(rhog_in), np.zeros_like(rhog_in_pl), g.dtl)
    for P, lo, la, z, zhh in ((PROG, lon[:, :, None, :], lat[:, :, None, :], zf, zh),
                              (PROG_pl, lon_pl[:, None, :], lat_pl[:, None, :], zf_pl, zh_pl)):
        vx, vy, vz, w = trcadv_winds(time, lo, la, z, zhh, case)
        P[..., I_RHOGVX] = vx * P[..., I_RHOG]
        P[..., I_RHOGVY] = vy * P[..., I_RHOG]
        P[..., I_RHOGVZ] = vz * P[..., I_RHOG]
        P[..., I_RHOGW] = w * P[..., I_RHOG]
    comm(g, out, out_pl)
    return out, out_pl

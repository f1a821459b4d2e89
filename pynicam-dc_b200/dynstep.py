"""The dynamics step as a differentiable function of the prognostic state.

One RK3-HEVI large step (mod_dynamics.py:1725-2741 with the numpy-path
operators: Pre_Post diagnostics and boundary conditions, momentum advection,
hyperdiffusion (DIRECT or NONLINEAR1 Kh), the Rayleigh sponge, the HEVI small steps of mod_vi.py:104-1590 with the 3-D and
2-D divergence damping, path 1 and vi_main) restated as torch expressions in
the reference's operation order, on CUDA tensors in the library's device
layout (regional (lall, kall, g, g), pole (6, kall, 2): the level axis is
axis 1 in both).  Every horizontal stencil and every halo exchange is one of
the library's hand-written float64 kernels wrapped as a
``torch.autograd.Function`` (``adjoint.Divergence``, ``Gradient``,
``Laplacian``, ``Diffusion``, ``divdamp3d`` / ``divdamp2d``, ``Exchange``;
the Thomas solve ``VerticalSolve``), whose adjoints are hand-written
transposed kernels; the pointwise and per-column algebra between them is
differentiated by torch.  The reverse pass of a step is therefore the
discrete adjoint of the step, and ``run`` checkpoints every large step.
The Held-Suarez forcing step (``held_suarez``) can follow each step.

The tracer masses are carried through unchanged: the tracer advection of the
step's last stage (mod_src_tracer.py) is not part of this restatement, and
the tracers enter the dynamics only through the water terms of the
diagnostics (kernels/diag.py:97-115), which vanish for a dry state (zero
water tracers), the adjoint configuration's case.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.utils.checkpoint

from . import adjoint as A
from .runtime import _scalar

I_RHOG, I_RHOGVX, I_RHOGVY, I_RHOGVZ, I_RHOGW, I_RHOGE = range(6)


class F:
    """a regional field and its pole rows, with elementwise arithmetic on both"""
    __slots__ = ("r", "p")

    def __init__(self, r, p):
        self.r, self.p = r, p

    def _op(self, o, f):
        if isinstance(o, F):
            return F(f(self.r, o.r), f(self.p, o.p))
        return F(f(self.r, o), f(self.p, o))

    def __add__(self, o): return self._op(o, lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, lambda a, b: b * a)
    def __truediv__(self, o): return self._op(o, lambda a, b: a / b)
    def __rtruediv__(self, o): return self._op(o, lambda a, b: b / a)
    def __neg__(self): return F(-self.r, -self.p)
    def __pow__(self, e): return F(self.r ** e, self.p ** e)

    def k(self, sl):
        """levels ``sl`` (a slice or an index, kept as a length-1 axis)"""
        if isinstance(sl, int):
            sl = slice(sl, sl + 1)
        return F(self.r[:, sl], self.p[:, sl])

    def setk(self, sl, v):
        """a copy with levels ``sl`` replaced by ``v`` (a field or a number)"""
        if isinstance(sl, int):
            sl = slice(sl, sl + 1)
        r, p = self.r.clone(), self.p.clone()
        if isinstance(v, F):
            r[:, sl], p[:, sl] = v.r, v.p
        else:
            r[:, sl], p[:, sl] = v, v
        return F(r, p)

    def zeros(self):
        return F(torch.zeros_like(self.r), torch.zeros_like(self.p))


def cat_k(parts):
    """concatenate fields along the level axis"""
    return F(torch.cat([a.r for a in parts], 1), torch.cat([a.p for a in parts], 1))


def stack(fs):
    return torch.stack([f.r for f in fs]), torch.stack([f.p for f in fs])


def unstack(r, p):
    return [F(r[n], p[n]) for n in range(r.shape[0])]


class Metrics(dict):
    """the metrics, vertical factors and run constants of one grid from a
    setup dict, as device tensors in the device layout"""

    def __init__(self, geo: dict, device="cuda"):
        super().__init__()
        sc = lambda k: float(_scalar(geo[k]))
        dl = lambda a: A.to_device_layout(np.asarray(a, np.float64), device)
        pl = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, np.float64))).to(device)
        for k in ("GSGAM2", "PHI", "RGAM", "RGAMH", "RGSQRTH", "GAM2H", "RGSGAM2", "RGSGAM2H", "GSGAM2H"):
            self[k] = F(dl(geo["VMTR_" + k]), pl(geo["VMTR_" + k + "_pl"]))
        for k, n in (("C2Wfact", 2), ("W2Cfact", 2), ("C2WfactGz", 6)):
            r, p = np.asarray(geo["VMTR_" + k]), np.asarray(geo["VMTR_" + k + "_pl"])
            self[k] = [F(dl(r[..., c]), pl(p[..., c])) for c in range(n)]
        for k in ("rho_bs", "pre_bs", "tem_bs"):
            self[k] = F(dl(geo[k]), pl(geo[k + "_pl"]))
        gx, gxp = np.asarray(geo["GRD_x"], np.float64), np.asarray(geo["GRD_x_pl"], np.float64)
        # position vectors broadcast along the levels: (lall, 1, g, g) and (6, 1, 2)
        self["GRD_x"] = [F(dl(gx[:, :, 0:1, :, d]), pl(gxp[:, 0:1, :, d])) for d in range(3)]
        for k in ("rdgz", "rdgzh", "afact", "bfact", "cfact", "dfact"):
            self[k] = torch.as_tensor(np.asarray(geo["GRD_" + k], np.float64)).to(device)
        for k in ("GRAV", "Rdry", "CVdry", "CPdry", "Rvap", "OHM", "PRE00", "rscale", "alpha", "dtl", "dts", "Kh_coef",
                  "divdamp_coef", "hdiff_fact_rho"):
            self[k] = sc(k)
        self["CVW"] = [float(x) for x in np.asarray(geo["CVW"], np.float64).reshape(-1)]
        self["nqw"] = int(_scalar(geo["NQW_END"])) + 1 if "NQW_END" in geo else 1
        self["kmin"], self["kmax"] = int(_scalar(geo["kmin"])), int(_scalar(geo["kmax"]))
        self["sstep"] = [int(x) for x in np.asarray(geo["sstep"]).reshape(-1)]
        self["hevi"] = A.hevi_metrics(geo, device)
        vec = lambda k: torch.as_tensor(np.asarray(geo[k], np.float64).reshape(-1)).to(device)
        self["nl"] = "hdiff_nl_kh_max" in geo           # NONLINEAR1 hyperdiffusion
        if self["nl"]:
            self["nl_khmax"] = vec("hdiff_nl_kh_max")
            self["nl_minlim"], self["nl_area"] = sc("hdiff_nl_minlim"), sc("hdiff_nl_area")
        self["ray"] = "rayleigh_coef" in geo            # the Rayleigh sponge
        if self["ray"]:
            self["ray_c"], self["ray_ch"] = vec("rayleigh_coef"), vec("rayleigh_coef_h")
            self["ray_only_w"] = bool(int(_scalar(geo["rayleigh_only_w"])))

    def lv(self, name, sl):
        """a 1-D level vector sliced and shaped to broadcast along axis 1"""
        v = self[name][sl]
        return F(v.view(1, -1, 1, 1), v.view(1, -1, 1))


# ---------------------------------------------------------------------------
# Pre_Post: diagnostics (kernels/diag.py:53-143, mod_dynamics.py:1163-1196)
# and boundary conditions (share/mod_bndcnd.py:182-264, kernels/bndcnd.py)
# ---------------------------------------------------------------------------
def diagnostics(m, P, Q, w_prev):
    """rho, pre, tem, vx, vy, vz, w, ein of the prognostics P (6 fields) and
    tracer masses Q; w outside kmin+1..kmax is taken from ``w_prev``"""
    kmin, kmax = m["kmin"], m["kmax"]
    rhog = P[I_RHOG]
    rho = rhog / m["GSGAM2"]
    vx, vy, vz = P[I_RHOGVX] / rhog, P[I_RHOGVY] / rhog, P[I_RHOGVZ] / rhog
    ein = P[I_RHOGE] / rhog
    q = [t / rhog for t in Q]
    nqw = min(m["nqw"], len(q))
    if nqw:
        qsum = q[0]
        for n in range(1, nqw):
            qsum = qsum + q[n]
        qd = 1.0 - qsum
        cv = q[0] * m["CVW"][0]
        for n in range(1, nqw):
            cv = cv + q[n] * m["CVW"][n]
        cv = cv + qd * m["CVdry"]
        tem = ein / cv
        pre = rho * tem * (qd * m["Rdry"] + q[0] * m["Rvap"])
    else:
        tem = ein / m["CVdry"]
        pre = rho * tem * m["Rdry"]
    c2w = m["C2Wfact"]
    kin, kdn = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    w = w_prev.setk(kin, P[I_RHOGW].k(kin) / (c2w[0].k(kin) * rhog.k(kin) + c2w[1].k(kin) * rhog.k(kdn)))
    return dict(rho=rho, pre=pre, tem=tem, vx=vx, vy=vy, vz=vz, w=w, ein=ein)


def bndcnd(m, D, P):
    """the ghost levels kmin-1 / kmax+1 of the diagnostics and prognostics
    (TEM / TEM, FREE top, RIGID bottom), returned as new fields"""
    kmin, kmax = m["kmin"], m["kmax"]
    GS, C2W, C2WGz, PHI = m["GSGAM2"], m["C2Wfact"], m["C2WfactGz"], m["PHI"]
    tem, pre, rho, ein = D["tem"], D["pre"], D["rho"], D["ein"]
    tem_top, tem_btm = tem.k(kmax), tem.k(kmin)
    pre_top = pre.k(kmax - 1) - rho.k(kmax) * (PHI.k(kmax + 1) - PHI.k(kmax - 1))
    pre_btm = pre.k(kmin + 1) - rho.k(kmin) * (PHI.k(kmin - 1) - PHI.k(kmin + 1))
    rho_top = pre_top / (m["Rdry"] * tem_top)
    rho_btm = pre_btm / (m["Rdry"] * tem_btm)
    tem = tem.setk(kmax + 1, tem_top).setk(kmin - 1, tem_btm)
    pre = pre.setk(kmax + 1, pre_top).setk(kmin - 1, pre_btm)
    rho = rho.setk(kmax + 1, rho_top).setk(kmin - 1, rho_btm)
    rhog = P[I_RHOG]
    rhog = rhog.setk(kmax + 1, rho.k(kmax + 1) * GS.k(kmax + 1)).setk(kmin - 1, rho.k(kmin - 1) * GS.k(kmin - 1))
    ein = ein.setk(kmax + 1, m["CVdry"] * tem.k(kmax + 1)).setk(kmin - 1, m["CVdry"] * tem.k(kmin - 1))
    rhoge = P[I_RHOGE].setk(kmax + 1, rhog.k(kmax + 1) * ein.k(kmax + 1))
    rhoge = rhoge.setk(kmin - 1, rhog.k(kmin - 1) * ein.k(kmin - 1))
    mom = []
    for iv in (I_RHOGVX, I_RHOGVY, I_RHOGVZ):
        v = P[iv]
        top = 1.0 * (v.k(kmax) / rhog.k(kmax)) * rhog.k(kmax + 1)
        btm = -1.0 * (v.k(kmin) / rhog.k(kmin)) * rhog.k(kmin - 1)
        mom.append(v.setk(kmax + 1, top).setk(kmin - 1, btm))
    vel = []
    for iv, name in zip(range(3), ("vx", "vy", "vz")):
        v = D[name]
        for kk in (kmax + 1, kmin - 1):
            v = v.setk(kk, mom[iv].k(kk) / rhog.k(kk))
        vel.append(v)
    vx, vy, vz = mom
    cz = lambda k, c: C2WGz[c].k(k)
    rw_top = -(cz(kmax + 1, 0) * vx.k(kmax + 1) + cz(kmax + 1, 1) * vx.k(kmax)
               + cz(kmax + 1, 2) * vy.k(kmax + 1) + cz(kmax + 1, 3) * vy.k(kmax)
               + cz(kmax + 1, 4) * vz.k(kmax + 1) + cz(kmax + 1, 5) * vz.k(kmax))
    rw = P[I_RHOGW].setk(kmax + 1, rw_top).setk(kmin, 0.0).setk(kmin - 1, 0.0)
    w = D["w"]
    w = w.setk(kmax + 1, rw.k(kmax + 1) / (C2W[0].k(kmax + 1) * rhog.k(kmax + 1) + C2W[1].k(kmax + 1) * rhog.k(kmax)))
    w = w.setk(kmin, rw.k(kmin) / (C2W[0].k(kmin) * rhog.k(kmin) + C2W[1].k(kmin) * rhog.k(kmin - 1)))
    w = w.setk(kmin - 1, 0.0)
    D = dict(D, tem=tem, pre=pre, rho=rho, ein=ein, vx=vel[0], vy=vel[1], vz=vel[2], w=w)
    return D, [rhog, vx, vy, vz, rw, rhoge]


# ---------------------------------------------------------------------------
# horizontal operators: the library's kernels through their autograd wrappers
# ---------------------------------------------------------------------------
def div(core, vx, vy, vz):
    return F(*A.divergence(core, *stack([vx, vy, vz])))


def grad(core, s):
    return unstack(*A.gradient(core, s.r, s.p))


def lap(core, s):
    return F(*A.laplacian(core, s.r, s.p))


def xch(core, fs):
    """the halo exchange of a list of fields"""
    return unstack(*A.exchange(core, *stack(fs)))


def horizontalize(m, vx, vy, vz):
    """kernels/horizontalizevec.py:34-71: the radial component removed; the
    regional form on interior cells only (the border kept), the pole form on
    every pole row, each with its own division order"""
    gx, r = m["GRD_x"], m["rscale"]
    out = []
    prd_r = (vx.r * gx[0].r + vy.r * gx[1].r + vz.r * gx[2].r) / r
    prd_p = vx.p * gx[0].p / r + vy.p * gx[1].p / r + vz.p * gx[2].p / r
    for v, g in zip((vx, vy, vz), gx):
        nr = v.r.clone()
        nr[..., 1:-1, 1:-1] = (v.r - prd_r * g.r / r)[..., 1:-1, 1:-1]
        out.append(F(nr, v.p - prd_p * g.p / r))
    return out


# ---------------------------------------------------------------------------
# sources (mod_src.py): flux and advection convergence, pressure gradient,
# buoyancy, momentum advection
# ---------------------------------------------------------------------------
def flux_convergence(m, core, rvx, rvy, rvz, rw, vertical=True):
    """kernels/fluxconv.py:111-208"""
    kmin, kmax = m["kmin"], m["kmax"]
    RGAM, RGAMH, RGSQRTH, cz = m["RGAM"], m["RGAMH"], m["RGSQRTH"], m["C2WfactGz"]
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    vxm, vym, vzm = rvx * RGAM, rvy * RGAM, rvz * RGAM
    horiz = (cz[0].k(ks) * rvx.k(ks) + cz[1].k(ks) * rvx.k(km) + cz[2].k(ks) * rvy.k(ks)
             + cz[3].k(ks) * rvy.k(km) + cz[4].k(ks) * rvz.k(ks) + cz[5].k(ks) * rvz.k(km))
    horiz = horiz * RGAMH.k(ks)
    vflag = 1.0 if vertical else 0.0
    vmh = rw.zeros().setk(ks, horiz + vflag * rw.k(ks) * RGSQRTH.k(ks))
    d = div(core, vxm, vym, vzm)
    kc, kcp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
    return rw.zeros().setk(kc, -d.k(kc) - (vmh.k(kcp) - vmh.k(kc)) * m.lv("rdgz", kc))


def scaled_fluxes(m, rvx, rvy, rvz, rw, scl, vertical=True):
    """kernels/advconv.py:42-108"""
    kmin, kmax = m["kmin"], m["kmax"]
    sw = rw.zeros()
    if vertical:
        kk, kd = slice(kmin, kmax + 2), slice(kmin - 1, kmax + 1)
        sw = sw.setk(kk, rw.k(kk) * (m.lv("afact", kk) * scl.k(kk) + m.lv("bfact", kk) * scl.k(kd)))
    return rvx * scl, rvy * scl, rvz * scl, sw


def advection_convergence(m, core, rvx, rvy, rvz, rw, scl, vertical=True):
    """mod_src.py:499-623: scaled fluxes then flux convergence"""
    return flux_convergence(m, core, *scaled_fluxes(m, rvx, rvy, rvz, rw, scl, vertical), vertical)


def pres_gradient(m, core, P, vertical=True):
    """kernels/presgrad.py:126-265 (first-layer remedy, horizontalize)"""
    kmin, kmax = m["kmin"], m["kmax"]
    gh = grad(core, P * m["RGAM"])
    cz, rgh = m["C2WfactGz"], m["RGAMH"].k(slice(kmin, kmax + 2))
    Pk, Pkm1 = P.k(slice(kmin, kmax + 2)), P.k(slice(kmin - 1, kmax + 1))
    rdz = m.lv("rdgz", slice(kmin, kmax + 1))
    n = kmax - kmin + 1
    Pg = []
    for d in range(3):
        c0, c1 = cz[2 * d].k(slice(kmin, kmax + 2)), cz[2 * d + 1].k(slice(kmin, kmax + 2))
        pv = (c0 * Pk + c1 * Pkm1) * rgh
        gf = gh[d].k(slice(kmin, kmax + 1)) + (pv.k(slice(1, n + 1)) - pv.k(slice(0, n))) * rdz
        g = gh[d].setk(kmin - 1, 0.0).setk(kmin, gf.k(1)).setk(slice(kmin + 1, kmax + 1), gf.k(slice(1, n)))
        Pg.append(g.setk(kmax + 1, 0.0))
    Pg = horizontalize(m, *Pg)
    Pgw = P.zeros()
    if vertical:
        ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
        G2, RS = m["GAM2H"], m["RGSGAM2"]
        Pgw = Pgw.setk(ks, G2.k(ks) * (P.k(ks) * RS.k(ks) - P.k(km) * RS.k(km)) * m.lv("rdgzh", ks))
    return Pg, Pgw


def buoyancy(m, rhog):
    """kernels/buoyancy.py:40-81"""
    kmin, kmax = m["kmin"], m["kmax"]
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    c = m["C2Wfact"]
    return rhog.zeros().setk(ks, -m["GRAV"] * (c[0].k(ks) * rhog.k(ks) + c[1].k(ks) * rhog.k(km)))


def advection_momentum(m, core, D, P):
    """mod_src.py:96-497 with kernels/advconvmom.py: (gvx, gvy, gvz, gw)"""
    kmin, kmax = m["kmin"], m["kmax"]
    kc, kp, ks = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2), slice(kmin + 1, kmax + 1)
    w, gb, r = D["w"], m["GRD_x"], m["rscale"]
    wc = m.lv("cfact", kc) * w.k(kp) + m.lv("dfact", kc) * w.k(kc)
    vv = [w.zeros().setk(kc, D[name].k(kc) + wc * g / r) for name, g in zip(("vx", "vy", "vz"), gb)]
    rvx, rvy, rvz, rw = P[I_RHOGVX], P[I_RHOGVY], P[I_RHOGVZ], P[I_RHOGW]
    dv = [advection_convergence(m, core, rvx, rvy, rvz, rw, s, True) for s in vv]
    rh = P[I_RHOG].k(kc)
    dvx = dv[0].k(kc) - (-2.0 * rh * (m["OHM"] * vv[1].k(kc)))
    dvy = dv[1].k(kc) - (2.0 * rh * (m["OHM"] * vv[0].k(kc)))
    dvz = dv[2].k(kc)
    gg = [g / r for g in gb]
    prd = dvx * gg[0] + dvy * gg[1] + dvz * gg[2]
    gwc = prd * m["alpha"]
    c = m["C2Wfact"]
    n = kmax - kmin + 1
    outs = [w.zeros().setk(kc, a - prd * g) for a, g in zip((dvx, dvy, dvz), gg)]
    outs.append(w.zeros().setk(ks, c[0].k(ks) * gwc.k(slice(1, n)) + c[1].k(ks) * gwc.k(slice(0, n - 1))))
    return outs


# ---------------------------------------------------------------------------
# numerical filters (mod_numfilter.py)
# ---------------------------------------------------------------------------
def hdiff_nonlinear_coef(m, lapT):
    """mod_numfilter.py:1153-1206 (NONLINEAR1): Kh from the temperature
    Laplacian of the first pass, 2 AREA^2 / dtl * (|lapT| / 300 * AREA)
    clipped to [Kh_coef_minlim, kh_max(k)], and its half-level average on
    kmin+1..kmax (zero elsewhere)"""
    kmin, kmax, A_ = m["kmin"], m["kmax"], m["nl_area"]
    c1 = 2.0 * (A_ ** 2) / m["dtl"]
    hi = m.lv("nl_khmax", slice(None))
    raw = c1 * (F(lapT.r.abs(), lapT.p.abs()) / 300.0 * A_)
    kh = F(torch.minimum(torch.clamp(raw.r, min=m["nl_minlim"]), hi.r),
           torch.minimum(torch.clamp(raw.p, min=m["nl_minlim"]), hi.p))
    ks, km = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    return kh, kh.zeros().setk(ks, 0.5 * (kh.k(ks) + kh.k(km)))


def rayleigh_damping(m, f, rhog, D):
    """mod_numfilter.py:240-271: the momentum tendencies lose
    rayleigh_coef(k) rhog v (unless only w is damped), the w tendency
    rayleigh_coef_h(k) w (C2Wa rhog(k) + C2Wb rhog(k-1)), rhog(-1) = 0"""
    f = list(f)
    if not m["ray_only_w"]:
        coef = m.lv("ray_c", slice(None)) * rhog
        for n, name in ((I_RHOGVX, "vx"), (I_RHOGVY, "vy"), (I_RHOGVZ, "vz")):
            f[n] = f[n] - coef * D[name]
    km1 = rhog.zeros().setk(slice(1, None), rhog.k(slice(0, -1)))
    c = m["C2Wfact"]
    f[I_RHOGW] = f[I_RHOGW] - m.lv("ray_ch", slice(None)) * D["w"] * (c[0] * rhog + c[1] * km1)
    return f


def hdiffusion(m, core, rhog, D):
    """mod_numfilter.py:845-1578 (DIRECT or NONLINEAR1 Kh, lap_order 2):
    f_TEND in prognostic order, differentiable in the density through the
    Kh rhog weights of the scalar pass as well"""
    kmin, kmax, Kh = m["kmin"], m["kmax"], m["Kh_coef"]
    c = m["C2Wfact"]
    kk, kd = slice(kmin, kmax + 2), slice(kmin - 1, kmax + 1)
    rhog_h = rhog.zeros().setk(kk, c[0].k(kk) * rhog.k(kk) + c[1].k(kk) * rhog.k(kd))
    vt = [D["vx"], D["vy"], D["vz"], D["w"], D["tem"] - m["tem_bs"], D["rho"] - m["rho_bs"]]
    KhA = KhH = Kh
    for p in range(2):
        v2 = [lap(core, vt[n]) for n in range(4)]
        if p == 1:
            if m["nl"]:
                KhA, KhH = hdiff_nonlinear_coef(m, vt[4])
            for s, fac in ((vt[4], m["CVdry"]), (vt[5], m["hdiff_fact_rho"])):
                kh = rhog * fac * KhA
                v2.append(F(*A.diffusion(core, s.r, s.p, kh.r, kh.p)))
        else:
            v2 += [lap(core, vt[4]), lap(core, vt[5])]
        vt = xch(core, [-a for a in v2])
    f = [None] * 6
    f[I_RHOGVX], f[I_RHOGVY], f[I_RHOGVZ] = horizontalize(m, *[-(vt[n] * KhA) * rhog for n in range(3)])
    f[I_RHOGW] = -(vt[3] * KhH) * rhog_h
    f[I_RHOGE] = -vt[4]
    f[I_RHOG] = -vt[5]
    return f


def numfilter_divdamp(m, core, rvx, rvy, rvz, rw):
    """mod_numfilter.py:2032-2268 (lap_order 2): the 3-D operator, exchange,
    the 2-D operator on the negation, coefficient, horizontalize"""
    d = unstack(*A.divdamp3d(core, *stack([rvx, rvy, rvz, rw])))
    o = unstack(*A.divdamp2d(core, *stack([-a for a in d])))
    return horizontalize(m, *[m["divdamp_coef"] * a for a in o])


# ---------------------------------------------------------------------------
# HEVI small steps (mod_vi.py:104-1590, kernels/vipath1.py, vimain.py)
# ---------------------------------------------------------------------------
def rhogkin(m, rhog, rvx, rvy, rvz, rw):
    """kernels/rhogkin.py:38-119"""
    kmin, kmax = m["kmin"], m["kmax"]
    kc, kvi, kcm = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    c, w2c = m["C2Wfact"], m["W2Cfact"]
    kh = 0.5 * (rvx.k(kc) ** 2 + rvy.k(kc) ** 2 + rvz.k(kc) ** 2) / rhog.k(kc)
    v_int = 0.5 * rw.k(kvi) ** 2 / (c[0].k(kvi) * rhog.k(kvi) + c[1].k(kvi) * rhog.k(kcm))
    z = v_int.k(0).zeros()
    vb = cat_k([z, v_int, z])
    n = kmax - kmin + 1
    tot = kh + w2c[0].k(kc) * vb.k(slice(1, n + 1)) + w2c[1].k(kc) * vb.k(slice(0, n))
    return rhog.zeros().setk(kc, tot)


def _per_part(fn, *args):
    """apply a regional/pole function (``pole`` keyword) to both parts"""
    r = fn(*[a.r if isinstance(a, F) else a for a in args], pole=False)
    p = fn(*[a.p if isinstance(a, F) else a for a in args], pole=True)
    if isinstance(r, tuple):
        return tuple(F(a, b) for a, b in zip(r, p))
    return F(r, p)


def vi_main(m, core, S, dt):
    """kernels/vimain.py:127-262 (TIME_split); ``S`` holds the fields named
    as in the reference's P dict.  Returns rhog_s1, rhogw_s1, rhoge_s1"""
    kmin, kmax = m["kmin"], m["kmax"]
    PHI, cz = m["PHI"], m["C2WfactGz"]
    vx, vy, vz = S["rhogvx_s1"], S["rhogvy_s1"], S["rhogvz_s1"]
    drhog = flux_convergence(m, core, vx, vy, vz, S["rhogw_s0"], False)
    drhoge = advection_convergence(m, core, vx, vy, vz, S["rhogw_s0"], S["eth0"], False)
    grhog1 = S["grhog"] + drhog
    gpre = (S["grhoge"] + drhoge) * m["Rdry"] / m["CVdry"]
    c = lambda n: cz[n].k(kmax + 1)
    rw_top = -(c(0) * vx.k(kmax + 1) + c(1) * vx.k(kmax) + c(2) * vy.k(kmax + 1)
               + c(3) * vy.k(kmax) + c(4) * vz.k(kmax + 1) + c(5) * vz.k(kmax))
    rw = vx.zeros().setk(kmax + 1, rw_top)
    Mc, Mu, Ml = S["M"]
    rhogw_s1 = _per_part(lambda *a, pole: A.hevi_solve(core, m["hevi"], *a, dt, pole=pole),
                         rw, S["rhogw_s0"], S["preg_s0"], S["rhog_s0"], grhog1, S["grhogw"], gpre, Mc, Mu, Ml)
    drhog2 = flux_convergence(m, core, vx, vy, vz, rhogw_s1, True)
    rhog_s1 = S["rhog_s0"] + (S["grhog"] + drhog2) * dt
    r0 = [S["rhog0"], S["rhogvx0"], S["rhogvy0"], S["rhogvz0"], S["rhogw0"]]
    kin0 = rhogkin(m, *r0)
    kin10 = rhogkin(m, *[a + b for a, b in zip(r0, [S["rhog_s0"], S["rhogvx_s0"], S["rhogvy_s0"], S["rhogvz_s0"],
                                                     S["rhogw_s0"]])])
    b = [r0[1] + vx, r0[2] + vy, r0[3] + vz, r0[4] + rhogw_s1]
    kin11 = rhogkin(m, r0[0] + rhog_s1, *b)
    ethtot0 = S["eth0"] + kin0 / r0[0] + PHI
    drhogetot = advection_convergence(m, core, *b, ethtot0, True)
    rhoge_s1 = (S["rhoge_s0"] + (S["grhogetot"] + drhogetot) * dt + (kin10 - kin11)
                + (S["rhog_s0"] - rhog_s1) * PHI)
    return rhog_s1, rhogw_s1, rhoge_s1


def vi_small_step(m, core, PROG, D, eth, rhogd, pregd, gT0, PS, nitr, dt):
    """mod_vi.py:104-1590 (numpy path): the large-step sources of the small
    steps, then ``nitr`` small steps of divergence damping, path 1
    (kernels/vipath1.py:68-160) and vi_main, each closed by its exchanges.
    Returns the new prognostics (PROG + PROG_split, momentum horizontalized)."""
    kmin, kmax = m["kmin"], m["kmax"]
    RovCV = m["Rdry"] / m["CVdry"]
    c, w2c = m["C2Wfact"], m["W2Cfact"]
    kk, kd = slice(kmin, kmax + 2), slice(kmin - 1, kmax + 1)
    rhog = PROG[I_RHOG]
    rhog_h = rhog.zeros().setk(kk, c[0].k(kk) * rhog.k(kk) + c[1].k(kk) * rhog.k(kd))
    eth_h = eth.zeros().setk(kk, m.lv("afact", kk) * eth.k(kk) + m.lv("bfact", kk) * eth.k(kd))
    rhog_h = rhog_h.setk(kmin - 1, rhog_h.k(kmin))
    eth_h = eth_h.setk(kmin - 1, eth_h.k(kmin))
    mom = [PROG[I_RHOGVX], PROG[I_RHOGVY], PROG[I_RHOGVZ], PROG[I_RHOGW]]
    drhog = flux_convergence(m, core, *mom, True)
    gd = numfilter_divdamp(m, core, *mom)
    dpg, dpgw = pres_gradient(m, core, pregd, True)
    dbuo = buoyancy(m, rhogd)
    drhoge = advection_convergence(m, core, *mom, eth, True)
    gzt = m["GRAV"] - (dpgw - dbuo) / rhog_h
    pwh = -gzt * PROG[I_RHOGW]
    kc, kp = slice(kmin, kmax + 1), slice(kmin + 1, kmax + 2)
    pw = pwh.zeros().setk(kc, D["vx"].k(kc) * dpg[0].k(kc) + D["vy"].k(kc) * dpg[1].k(kc)
                          + D["vz"].k(kc) * dpg[2].k(kc) + w2c[0].k(kc) * pwh.k(kp) + w2c[1].k(kc) * pwh.k(kc))
    T = [gT0[I_RHOG] + drhog,
         gT0[I_RHOGVX] - dpg[0] + gd[0], gT0[I_RHOGVY] - dpg[1] + gd[1], gT0[I_RHOGVZ] - dpg[2] + gd[2],
         gT0[I_RHOGW] - dpgw + dbuo,
         gT0[I_RHOGE] + drhoge + pw]
    M = _per_part(lambda e, g, pole: A.hevi_matrix(m["hevi"], e, g, dt, pole=pole), eth_h, gzt)
    PS = list(PS)
    for _ in range(nitr):
        re = PS[I_RHOGE].setk(kmin - 1, PS[I_RHOGE].k(kmin)).setk(kmax + 1, PS[I_RHOGE].k(kmax))
        PS[I_RHOGE] = re
        preg_s = re * RovCV
        dd = numfilter_divdamp(m, core, PS[I_RHOGVX], PS[I_RHOGVY], PS[I_RHOGVZ], PS[I_RHOGW])
        pg, _ = pres_gradient(m, core, preg_s, False)
        dvh = []
        for n, iv in enumerate((I_RHOGVX, I_RHOGVY, I_RHOGVZ)):
            v = PS[iv] + (T[iv] - pg[n] + dd[n]) * dt
            top = 1.0 * (v.k(kmax) / rhog.k(kmax)) * rhog.k(kmax + 1)
            btm = -1.0 * (v.k(kmin) / rhog.k(kmin)) * rhog.k(kmin - 1)
            dvh.append(v.setk(kmax + 1, top).setk(kmin - 1, btm))
        dvh = xch(core, dvh)
        S = {"rhogvx_s1": dvh[0], "rhogvy_s1": dvh[1], "rhogvz_s1": dvh[2],
             "rhog_s0": PS[I_RHOG], "rhogvx_s0": PS[I_RHOGVX], "rhogvy_s0": PS[I_RHOGVY],
             "rhogvz_s0": PS[I_RHOGVZ], "rhogw_s0": PS[I_RHOGW], "rhoge_s0": PS[I_RHOGE], "preg_s0": preg_s,
             "rhog0": rhog, "rhogvx0": PROG[I_RHOGVX], "rhogvy0": PROG[I_RHOGVY], "rhogvz0": PROG[I_RHOGVZ],
             "rhogw0": PROG[I_RHOGW], "eth0": eth, "grhog": T[I_RHOG], "grhogw": T[I_RHOGW],
             "grhoge": T[I_RHOGE], "grhogetot": gT0[I_RHOGE], "M": M}
        dwe = xch(core, list(vi_main(m, core, S, dt)))
        PS = [dwe[0], dvh[0], dvh[1], dvh[2], dwe[1], dwe[2]]
    out = [a + b for a, b in zip(PROG, PS)]
    out[I_RHOGVX], out[I_RHOGVY], out[I_RHOGVZ] = horizontalize(m, out[I_RHOGVX], out[I_RHOGVY], out[I_RHOGVZ])
    return out


def dynamics_step(m, core, prog, tracers=()):
    """one RK3-HEVI large step (mod_dynamics.py:1725-2741) of the six
    prognostic fields ``prog`` (list of ``F``), tracer masses held fixed;
    returns the new six fields after the closing exchange"""
    PROG = list(prog)
    PROG0 = list(prog)
    w_prev = PROG[I_RHOGW].zeros()
    nstage = len(m["sstep"])
    for nl in range(nstage):
        D = diagnostics(m, PROG, list(tracers), w_prev)
        D, PROG = bndcnd(m, D, PROG)
        eth = D["ein"] + D["pre"] / D["rho"]
        pregd = (D["pre"] - m["pre_bs"]) * m["GSGAM2"]
        rhogd = (D["rho"] - m["rho_bs"]) * m["GSGAM2"]
        adv = advection_momentum(m, core, D, PROG)
        f = hdiffusion(m, core, PROG[I_RHOG], D)
        if m["ray"]:
            f = rayleigh_damping(m, f, PROG[I_RHOG], D)
        gT = [f[I_RHOG], adv[0] + f[I_RHOGVX], adv[1] + f[I_RHOGVY], adv[2] + f[I_RHOGVZ], adv[3] + f[I_RHOGW],
              f[I_RHOGE]]
        PS = [a.zeros() for a in PROG] if nl == 0 else [a - b for a, b in zip(PROG0, PROG)]
        PROG = vi_small_step(m, core, PROG, D, eth, rhogd, pregd, gT, PS, m["sstep"][nl], m["dts"])
        if nl != nstage - 1:
            PROG = xch(core, PROG)
        w_prev = D["w"]
    return xch(core, PROG)


# ---------------------------------------------------------------------------
# Held-Suarez forcing (forcing/mod_af_heldsuarez.py:38-88 applied as in
# mod_forcing.py:14-28, 323-349): the regional columns only
# ---------------------------------------------------------------------------
HS_SIGMA_B, HS_KF, HS_KA, HS_KS, HS_DTH_Z = 0.7, 1.0 / 86400.0, 1.0 / (40.0 * 86400.0), 1.0 / (4.0 * 86400.0), 10.0


def held_suarez(m, core, prog, lat, tracers=(), moist=False):
    """one forcing step: the diagnostics of the regional prognostics, the
    Held-Suarez tendencies (Rayleigh friction below sigma 0.7, Newtonian
    relaxation to the equilibrium temperature) applied as
    PROG + dtl f rho GSGAM2 to the momenta and RHOGE on kmin..kmax, then
    the halo exchange; ``lat`` the column latitudes (lall, 1, g, g);
    ``moist`` the moist case's profile (T_eq0 294 K, DT_y 65 K)"""
    T_eq0, DT_y = (294.0, 65.0) if moist else (315.0, 60.0)
    kmin, kmax = m["kmin"], m["kmax"]
    D = diagnostics(m, list(prog), list(tracers), prog[I_RHOGW].zeros())
    pre, tem = D["pre"].r, D["tem"].r
    sin2, cos2, cos4 = torch.sin(lat).abs() ** 2, torch.cos(lat).abs() ** 2, torch.cos(lat).abs() ** 4
    psref = 0.5 * (pre[:, kmin:kmin + 1] + pre[:, kmin - 1:kmin])
    factor = torch.clamp((pre / psref - HS_SIGMA_B) / (1.0 - HS_SIGMA_B), min=0.0)
    ap0 = (pre / m["PRE00"]).abs()
    Kt = HS_KA + (HS_KS - HS_KA) * factor * cos4
    T_eq = torch.clamp((T_eq0 - DT_y * sin2 - HS_DTH_Z * torch.log(torch.clamp(ap0, min=1e-30)) * cos2)
                       * ap0 ** (m["Rdry"] / m["CPdry"]), min=200.0)
    valid = torch.zeros_like(pre)
    valid[:, kmin:kmax + 1] = 1.0
    scale = m["dtl"]
    out = list(prog)
    for iv, name in ((I_RHOGVX, "vx"), (I_RHOGVY, "vy"), (I_RHOGVZ, "vz")):
        f = torch.where(valid > 0, -HS_KF * factor * D[name].r, torch.zeros_like(pre))
        out[iv] = F(prog[iv].r + scale * f * D["rho"].r * m["GSGAM2"].r, prog[iv].p)
    fe = torch.where(valid > 0, -Kt * (tem - T_eq) * m["CVdry"], torch.zeros_like(pre))
    out[I_RHOGE] = F(prog[I_RHOGE].r + scale * fe * D["rho"].r * m["GSGAM2"].r, prog[I_RHOGE].p)
    return xch(core, out)


class DynamicsStep:
    """the differentiable dynamics step of one grid.

    ``core``: a ``NicamCuda`` handle of the grid (its halo plan and operator
    coefficients); ``geo``: the setup dict it was made from.  The state is a
    pair (x, x_pl) of tensors (6, lall, kall, g, g) / (6, 6, kall, 2) in
    prognostic order (RHOG, RHOGVX, RHOGVY, RHOGVZ, RHOGW, RHOGE)."""

    def __init__(self, core, geo: dict, device="cuda", hs_lat=None, hs_moist: bool = False):
        """``hs_lat``: the column latitudes (gall_1d, gall_1d, lall) of a
        Held-Suarez run; each step is then followed by its forcing step"""
        self.core, self.m = core, Metrics(geo, device)
        self.hs_lat, self.hs_moist = None, hs_moist
        if hs_lat is not None:
            self.hs_lat = torch.as_tensor(np.ascontiguousarray(np.transpose(np.asarray(hs_lat, np.float64),
                                                                            (2, 1, 0)))[:, None]).to(device)

    def step(self, x, x_pl, tracers=None, tracers_pl=None):
        Q = [] if tracers is None else [F(tracers[n], tracers_pl[n]) for n in range(tracers.shape[0])]
        out = dynamics_step(self.m, self.core, unstack(x, x_pl), Q)
        if self.hs_lat is not None:
            out = held_suarez(self.m, self.core, out, self.hs_lat, Q, self.hs_moist)
        return stack(out)

    def run(self, x, x_pl, nsteps: int, checkpoint: bool = True, tracers=None, tracers_pl=None):
        """``nsteps`` large steps; with ``checkpoint`` each step's
        intermediates are recomputed in the backward pass (one stored state
        per large step)"""
        for _ in range(nsteps):
            if checkpoint:
                x, x_pl = torch.utils.checkpoint.checkpoint(self.step, x, x_pl, tracers, tracers_pl,
                                                            use_reentrant=False)
            else:
                x, x_pl = self.step(x, x_pl, tracers, tracers_pl)
        return x, x_pl

    def surface_pressure(self, x, x_pl, zk, zk_pl):
        """the surface pressure of a state: pre + rho g (z - zsfc) at the
        lowest full level (mod_history_vars.py, sl_ps), ``zk`` the height of
        that level above the surface (lall, 1, g, g) / (6, 1, 2)"""
        m, k = self.m, self.m["kmin"]
        P = unstack(x, x_pl)
        D = diagnostics(m, P, [], P[I_RHOGW].zeros())
        ps = D["pre"].k(k) + D["rho"].k(k) * m["GRAV"] * F(zk, zk_pl)
        return ps.r, ps.p

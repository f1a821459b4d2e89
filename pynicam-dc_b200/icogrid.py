"""Icosahedral grid, metrics, operator coefficients and the Jablonowski-Williamson
initial state for the 40-region (rlevel 1) single-device layout.

This module builds, without the reference installed, everything the dynamics
step consumes: the setup dict of ``NicamCuda`` (reference attribute names and
layouts) and the initial prognostic state.  It restates the reference's setup
chain:

* horizontal grid -- recursive icosahedral division, spring-dynamics smoothing
  and the gravitational-centre pass (prep/hgrid/mod_mkgrd.py:66-195,
  204-320, 547-667);
* model grid -- pole triangle centres, radius scaling, lat/lon, arc midpoints,
  vertical levels (ULLRICH14 layers of prep/vgrid/mkvlayer.py:29-35,56-66) and
  the HYBRID terrain-following heights (share/mod_grd.py:64-340, 542-660, 764-931);
* JW surface height (share/mod_ideal_topo.py ``IDEAL_topo_JW``);
* geometric metrics GMTR_p/t/a (share/mod_gmtr.py:75-736);
* operator coefficients OPRT_coef_div/grad/lap/intp/diff
  (share/mod_oprt.py:125-1386);
* vertical metrics VMTR_* (share/mod_vmtr.py:39-400);
* the JW baroclinic-wave state (nhm/share/mod_ideal_init.py:320-470) converted
  to prognostic variables (nhm/share/mod_cnvvar.py:20-150).

The operator coefficients are assembled from one ring formulation (each cell's
hexagon or pentagon as a cycle of six or five triangles and their edges), not
from per-coefficient formula tables, so sums run in a different order than
the reference's and agree with it to rounding (about 1e-15 relative).  The
spring-dynamics relaxation runs on the host in numpy with the reference's
arithmetic or, at large grid levels, on the device (``nc_grid_spring``).  Halo
exchanges use the reference's own copy lists, stored in ``data/halo_rl01.npz``.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import halo

_HERE = os.path.dirname(os.path.abspath(__file__))

# physical constants of the JW case (share/mod_const.py:150-175 with the
# tutorial cnstparam)
RADIUS = 6.37122e6
OHM = 7.292e-5
GRAV = 9.80616
RDRY = 287.0
CPDRY = 1004.5
CVDRY = CPDRY - RDRY
RVAP = 461.46
PRE00 = 1.0e5
PI = 4.0 * math.atan(1.0)
EPS = float(np.finfo(np.float64).eps)
HUGE = float(np.finfo(np.float64).max)
UNDEF = -9.9999e30

TI, TJ = 0, 1
AI, AIJ, AJ = 0, 1, 2
LP = 2      # poles: 0 north, 1 south


# ---------------------------------------------------------------------------
# halo exchange on region-major arrays  a (L, G, G, ...) and a_pl (2, 6, ...)
# ---------------------------------------------------------------------------
class Exchange:
    """One halo exchange of the single-rank plan (regional + pole points)."""

    def __init__(self, glevel: int, G: int, L: int = 40):
        z = np.load(os.path.join(_HERE, "data", "halo_rl01.npz"))
        key = f"gl{glevel:02d}_"
        self.lists = {k: z[key + k].astype(np.int64) for k in ("r2r", "p2r", "r2p", "sgp")}
        self.have_sgp = z["have_sgp"].copy()
        plan = halo.compose(self.lists["r2r"], self.lists["p2r"], self.lists["r2p"], self.lists["sgp"], G, L)
        self.plan = plan
        r_dst, r_src, p_dst, p_src = plan
        dec = lambda c: (c // (G * G), c % G, (c // G) % G)          # l, i, j
        self.d = dec(r_dst)
        self.m = r_src >= 0
        self.s = dec(r_src[self.m])
        ps = -r_src[~self.m] - 1
        self.sp = (ps % LP, ps // LP)                                 # lp, g
        self.pd = (p_dst % LP, p_dst // LP)
        self.ps = dec(p_src)

    def __call__(self, a, a_pl):
        old = a.copy()
        oldp = a_pl.copy()
        vals = np.empty((len(self.m),) + a.shape[3:], a.dtype)
        vals[self.m] = old[self.s]
        vals[~self.m] = oldp[self.sp]
        a[self.d] = vals
        a_pl[self.pd] = old[self.ps]



# ---------------------------------------------------------------------------
# small vector helpers (component axis last); sums keep x, y, z order
# ---------------------------------------------------------------------------
def _dot(u, v):
    return u[..., 0] * v[..., 0] + u[..., 1] * v[..., 1] + u[..., 2] * v[..., 2]


def _cross(u, v):
    return np.stack([u[..., 1] * v[..., 2] - u[..., 2] * v[..., 1],
                     u[..., 2] * v[..., 0] - u[..., 0] * v[..., 2],
                     u[..., 0] * v[..., 1] - u[..., 1] * v[..., 0]], axis=-1)


def _norm(u):
    return np.sqrt(u[..., 0] * u[..., 0] + u[..., 1] * u[..., 1] + u[..., 2] * u[..., 2])


def _angle(u, v):
    """great-circle angle between two position vectors (atan2 form)"""
    return np.arctan2(_norm(_cross(u, v)), _dot(u, v))


def _tri_area(a, b, c, radius):
    """spherical triangle area by l'Huilier's theorem (unit vectors in)"""
    l1 = _angle(a, b) * 0.5
    l2 = _angle(b, c) * 0.5
    l3 = _angle(c, a) * 0.5
    s = 0.5 * (l1 + l2 + l3)
    x = np.tan(s) * np.tan(s - l1) * np.tan(s - l2) * np.tan(s - l3)
    x = np.maximum(x, 0.0)
    return 4.0 * np.arctan(np.sqrt(x)) * radius * radius


def _arc(u, v, eps=None):
    c = _cross(u, v)
    s = _norm(c)
    ang = np.arctan2(s, _dot(u, v))
    if eps is None:
        with np.errstate(invalid="ignore", divide="ignore"):
            return c * (ang / s)[..., None]
    zsw = 0.5 - np.copysign(0.5, np.abs(s) - eps)
    return c * ((1.0 - zsw) / (s + zsw) * ang)[..., None]


def _unit(a):
    return a / _norm(a)[..., None]


def _tn_vectors(v_from, v_to, radius):
    """arc tangent and normal vectors scaled to the geodesic arc length"""
    dist = np.arctan2(_norm(_cross(v_from, v_to)), _dot(v_from, v_to)) * radius
    t = v_to - v_from
    n = _cross(v_from, v_to)
    with np.errstate(invalid="ignore", divide="ignore"):
        t = t * (dist / _norm(t))[..., None]
        n = n * (dist / _norm(n))[..., None]
    return t, n


def _latlon(x, pole_points=False):
    """latitude/longitude of position vectors.  ``pole_points`` selects the
    point-wise convention of the pole arrays: a vector with z/|x| at +-1 gets
    longitude 0 even when its x, y parts are not exactly zero."""
    X, Y, Z = x[..., 0], x[..., 1], x[..., 2]
    length = np.sqrt(X * X + Y * Y + Z * Z)
    small = length < EPS
    zr = Z / np.where(small, 1.0, length)
    lat = np.where(zr >= 1.0, np.arcsin(1.0), np.where(zr <= -1.0, np.arcsin(-1.0),
                                                        np.arcsin(np.clip(zr, -1.0, 1.0))))
    lh = np.sqrt(X * X + Y * Y)
    small_h = lh < EPS
    xr = X / np.where(small_h, 1.0, lh)
    lon = np.where(xr >= 1.0, np.arccos(1.0), np.where(xr <= -1.0, np.arccos(-1.0),
                                                        np.arccos(np.clip(xr, -1.0, 1.0))))
    lon = np.where(Y < 0.0, -lon, lon)
    lon = np.where(small_h | small, 0.0, lon)
    if pole_points:
        lon = np.where((zr >= 1.0) | (zr <= -1.0), 0.0, lon)
    lat = np.where(small, 0.0, lat)
    return lat, lon


# ---------------------------------------------------------------------------
# horizontal grid generation
# ---------------------------------------------------------------------------
def _divide(g0):
    """one recursive division of (..., n, n, 3) corner points, renormalised"""
    n0 = g0.shape[-2]
    n1 = 2 * n0 - 1
    g1 = np.zeros(g0.shape[:-3] + (n1, n1, 3))
    g1[..., 0::2, 0::2, :] = g0
    g1[..., 1::2, 0::2, :] = g0[..., 1:, :, :] + g0[..., :-1, :, :]
    g1[..., 0::2, 1::2, :] = g0[..., :, 1:, :] + g0[..., :, :-1, :]
    g1[..., 1::2, 1::2, :] = g0[..., 1:, 1:, :] + g0[..., :-1, :-1, :]
    return g1 / _norm(g1)[..., None]


def standard_grid(glevel: int, rlevel: int = 1):
    """Unsmoothed icosahedral points: x (L, G, G, 3) with the interior set,
    x_pl (2, 6, 3) with the pole points set."""
    n_1d = 2 ** rlevel
    L = 10 * n_1d * n_1d
    G = 2 ** (glevel - rlevel) + 2
    a2 = 2.0 * PI / 5.0
    phi = float(np.arcsin(np.cos(a2) / (1.0 - np.cos(a2))))
    c, s = np.cos, np.sin
    r0 = np.zeros((10, 2, 2, 3))
    for d in range(10):
        if d <= 4:
            r = float(d)
            r0[d, 0, 0] = [c(phi) * c(a2 * r), c(phi) * s(a2 * r), s(phi)]
            r0[d, 1, 0] = [c(-phi) * c(a2 * (r + 0.5)), c(-phi) * s(a2 * (r + 0.5)), s(-phi)]
            r0[d, 0, 1] = [0.0, 0.0, 1.0]
            r0[d, 1, 1] = [c(phi) * c(a2 * (r + 1.0)), c(phi) * s(a2 * (r + 1.0)), s(phi)]
        else:
            r = float(d - 5)
            r0[d, 0, 0] = [c(-phi) * c(-a2 * (r + 0.5)), c(-phi) * s(-a2 * (r + 0.5)), s(-phi)]
            r0[d, 1, 0] = [0.0, 0.0, -1.0]
            r0[d, 0, 1] = [c(phi) * c(-a2 * r), c(phi) * s(-a2 * r), s(phi)]
            r0[d, 1, 1] = [c(-phi) * c(-a2 * (r - 0.5)), c(-phi) * s(-a2 * (r - 0.5)), s(-phi)]
    for _ in range(rlevel):
        r0 = _divide(r0)
    rg = np.arange(L)
    dmd, sub = rg // (n_1d * n_1d), rg % (n_1d * n_1d)
    ir, jr = sub % n_1d, sub // n_1d
    g0 = np.stack([np.stack([r0[dmd, ir + a, jr + b] for b in (0, 1)], axis=1) for a in (0, 1)], axis=1)
    for _ in range(rlevel, glevel):
        g0 = _divide(g0)
    x = np.zeros((L, G, G, 3))
    x[:, 1:G - 1, 1:G - 1] = g0[:, :G - 2, :G - 2]
    x_pl = np.zeros((LP, 6, 3))
    x_pl[0, 0] = [0.0, 0.0, 1.0]
    x_pl[1, 0] = [0.0, 0.0, -1.0]
    return x, x_pl


def spring(x, x_pl, glevel: int, exch: Exchange, beta: float = 1.15, device: str = "cpu",
           max_iter: int = 10_000_000):
    """Spring-dynamics smoothing of the interior points (each point pulled
    towards the natural length beta*lambda of its six springs, damped, kept on
    the sphere; pentagon corners fixed) until max |F|/lambda < 1e-4.
    ``device="cuda"`` runs the relaxation in libnicamcuda (nc_grid_spring),
    otherwise numpy on the host.  Returns (x, x_pl, iterations)."""
    dt, crit = 0.02, 1.0e-4
    L, G = x.shape[0], x.shape[1]
    lam = 2.0 * PI / (10.0 * 2.0 ** (glevel - 1))
    dbar = beta * lam
    if device == "cuda":
        from .runtime import grid_spring
        return grid_spring(x.copy(), x_pl.copy(), exch.have_sgp, exch.plan, lam, dbar, dt, crit, max_iter)
    var = np.zeros((L, G, G, 8))
    var[..., 0:3] = x
    var_pl = np.zeros((LP, 6, 8))
    var_pl[..., 0:3] = x_pl
    sgp = np.nonzero(exch.have_sgp)[0]
    nb = [(1, 0), (1, 1), (0, 1), (-1, 0), (-1, -1), (0, -1)]
    s = slice(1, G - 1)
    it = 0
    for it in range(1, max_iter + 1):
        R = var[..., 0:3]
        P0 = R[:, s, s]
        Fsum = None
        for m, (di, dj) in enumerate(nb):
            Pm = R[:, 1 + di:G - 1 + di, 1 + dj:G - 1 + dj]
            if m == 5:
                Pm = Pm.copy()
                Pm[sgp, 0, 0] = R[sgp, 2, 1]
            P0Pm = _cross(P0, Pm)
            P0PmP0 = _cross(P0Pm, P0)
            dist = np.arctan2(_norm(P0Pm), _dot(P0, Pm))
            F = (dist - dbar)[..., None] * P0PmP0 / _norm(P0PmP0)[..., None]
            if m == 5:
                F[sgp, 0, 0] = 0.0
            Fsum = F if Fsum is None else Fsum + F
        W = var[:, s, s, 3:6]
        fixed = var[sgp, 1, 1, 0:3].copy()
        R0 = P0 + W * dt
        R0 = R0 / _norm(R0)[..., None]
        W0 = W + (Fsum - 1.0 * W) * dt
        W0 = W0 - _dot(R0, W0)[..., None] * R0
        var[:, s, s, 0:3] = R0
        var[:, s, s, 3:6] = W0
        var[:, s, s, 6] = _norm(Fsum) / lam
        var[:, s, s, 7] = 0.5 * _dot(W0, W0)
        var[sgp, 1, 1, :] = 0.0
        var[sgp, 1, 1, 0:3] = fixed
        exch(var, var_pl)
        if var[:, s, s, 6].max() < crit:
            break
    return var[..., 0:3].copy(), var_pl[..., 0:3].copy(), it


def gravcenter(x, x_pl, have_sgp, exch: Exchange):
    """Triangle centres from cell centres, then cell centres as the
    gravitational centres of their hexagons/pentagons.  Returns (x, x_pl, xt)
    with xt (L, G, G, 2, 3) valid on indices 0..G-2."""
    L, G = x.shape[0], x.shape[1]
    gmin, gmax = 1, G - 2
    xt = np.zeros((L, G, G, 2, 3))
    A = x[:, 0:G - 1, 0:G - 1]
    Bi = x[:, 1:G, 0:G - 1]
    C = x[:, 1:G, 1:G]
    Cj = x[:, 0:G - 1, 1:G]
    with np.errstate(invalid="ignore", divide="ignore"):
        xt[:, 0:G - 1, 0:G - 1, TI] = _unit(_arc(A, Bi) + _arc(Bi, C) + _arc(C, A))
        xt[:, 0:G - 1, 0:G - 1, TJ] = _unit(_arc(A, C) + _arc(C, Cj) + _arc(Cj, A))
    xt[:, gmax, gmin - 1, TI] = xt[:, gmax, gmin - 1, TJ]
    xt[:, gmin - 1, gmax, TJ] = xt[:, gmin - 1, gmax, TI]
    sg = np.nonzero(have_sgp)[0]
    xt[sg, gmin - 1, gmin - 1, TI] = xt[sg, gmin, gmin - 1, TJ]
    # hexagon centres from their six triangle centres
    s, m = slice(gmin, gmax + 1), slice(gmin - 1, gmax)
    w = [xt[:, s, m, TJ], xt[:, s, s, TI], xt[:, s, s, TJ], xt[:, m, s, TI], xt[:, m, m, TJ],
         xt[:, m, m, TI].copy()]
    w[5][sg, 0, 0] = w[0][sg, 0, 0]
    w.append(w[0])
    gc = _arc(w[0], w[1], EPS)
    for v in range(1, 6):
        gc = gc + _arc(w[v], w[v + 1], EPS)
    x = x.copy()
    x[:, s, s] = _unit(gc)
    x_pl = x_pl.copy()
    for lp in range(LP):
        xtp = [None] * 6
        for v in range(1, 6):
            vp1 = v + 1 if v < 5 else 1
            g = _arc(x_pl[lp, 0], x_pl[lp, v]) + _arc(x_pl[lp, v], x_pl[lp, vp1]) + _arc(x_pl[lp, vp1], x_pl[lp, 0])
            xtp[v] = -_unit(g)
        g = np.zeros(3)
        for v in range(1, 6):
            g = g + _arc(xtp[v], xtp[v + 1 if v < 5 else 1])
        x_pl[lp, 0] = -_unit(g)
    exch(x, x_pl)
    return x, x_pl, xt


# ---------------------------------------------------------------------------
# vertical grid
# ---------------------------------------------------------------------------
def vertical_levels(vlayer: int, ztop: float, layer: str = "ULLRICH14"):
    """ULLRICH14 stretched or EVEN layers with one dummy level at each end
    (prep/vgrid/mkvlayer.py: mk_layer_ullrich14, mk_layer_even,
    generate_layers): returns (gz, gzh) of length vlayer + 2."""
    kall = vlayer + 2
    z_h = np.zeros(kall)
    z_c = np.zeros(kall)
    if layer == "ULLRICH14":
        mu = 15.0
        for k in range(1, vlayer + 2):
            fact = ((k + 1) / vlayer) ** 2
            z_h[k] = ztop * (np.sqrt(mu * fact + 1.0) - 1.0) / (np.sqrt(mu + 1.0) - 1.0)
    elif layer == "EVEN":
        dz = ztop / vlayer
        for k in range(kall):
            z_h[k] = dz * k
    else:
        raise ValueError(f"unknown layer type {layer!r}")
    z_h[0] = z_h[1] - (z_h[2] - z_h[1])
    for k in range(0, vlayer + 1):
        z_c[k] = z_h[k] + 0.5 * (z_h[k + 1] - z_h[k])
    z_c[vlayer + 1] = z_h[vlayer + 1] + 0.5 * (z_h[vlayer + 1] - z_h[vlayer])
    # the reference reads these through a JSON file
    z_c = np.array(json.loads(json.dumps(z_c.tolist())))
    z_h = np.array(json.loads(json.dumps(z_h.tolist())))
    return z_c, z_h


def vertical_factors(gz, gzh):
    kall = len(gz)
    kmin, kmax = 1, kall - 2
    dgz = np.zeros(kall)
    dgzh = np.zeros(kall)
    for k in range(kmin - 1, kmax + 1):
        dgz[k] = gzh[k + 1] - gzh[k]
    dgz[kmax + 1] = dgz[kmax]
    for k in range(kmin, kmax + 2):
        dgzh[k] = gz[k] - gz[k - 1]
    dgzh[kmin - 1] = dgzh[kmin]
    af = np.zeros(kall)
    cf = np.zeros(kall)
    for k in range(kmin, kmax + 2):
        af[k] = (gzh[k] - gz[k - 1]) / (gz[k] - gz[k - 1])
    af[kmin - 1] = 1.0
    for k in range(kmin, kmax + 1):
        cf[k] = (gz[k] - gzh[k]) / (gzh[k + 1] - gzh[k])
    cf[kmin - 1] = 1.0
    cf[kmax + 1] = 0.0
    return dict(dgz=dgz, dgzh=dgzh, rdgz=1.0 / dgz, rdgzh=1.0 / dgzh, afact=af, bfact=1.0 - af, cfact=cf,
                dfact=1.0 - cf)


# ---------------------------------------------------------------------------
# the setup chain
# ---------------------------------------------------------------------------
class Grid:
    """All setup arrays of one grid level in region-major layout."""

    def __init__(self, glevel: int, vlayer: int = 40, ztop: float = 30000.0, device: str = "cpu",
                 h_efold: float = 40000.0, raw=None, layer: str = "ULLRICH14", topo: str = "JW"):
        """``layer``: vertical layering, "ULLRICH14" (the JW cases) or "EVEN"
        (the tracer-transport case); ``topo``: "JW" (the balanced jet's
        surface height) or "NONE" (flat surface, DCMIP 1-1)."""
        self.glevel = glevel
        self.layer, self.topo = layer, topo
        self.G = G = 2 ** (glevel - 1) + 2
        self.L = L = 40
        self.kall = vlayer + 2
        self.exch = Exchange(glevel, G, L)
        self.have_sgp = self.exch.have_sgp
        if raw is None:
            x, x_pl = standard_grid(glevel, 1)
            self.exch(x, x_pl)
            x, x_pl, self.spring_iters = spring(x, x_pl, glevel, self.exch, device=device)
            x, x_pl, xt = gravcenter(x, x_pl, self.have_sgp, self.exch)
        else:
            x, x_pl, xt = raw
            self.spring_iters = -1
        self._model_grid(x, x_pl, xt)
        self._vertical(vlayer, ztop, h_efold)
        self._gmtr()
        self._oprt()
        self._vmtr()

    # -- share/mod_grd.py ---------------------------------------------------
    def _model_grid(self, x, x_pl, xt):
        L, G = self.L, self.G
        gmin, gmax = 1, G - 2
        xt = xt.copy()
        xt_pl = np.zeros((LP, 6, 3))
        # pole triangle centres: the corner triangle of each region touching the
        # pole, matched to the pole ring by position
        for lp, (ci, cj, t) in enumerate(((gmin, gmax, TJ), (gmax, gmin, TI))):
            touch = [l for l in range(L) if np.any(np.all(x_pl[lp, 1:6] == x[l, ci, cj], axis=-1))]
            cand = xt[touch, ci, cj, t]
            for v in range(1, 6):
                vp1 = v + 1 if v < 5 else 1
                ctr = _unit(x_pl[lp, 0] + x_pl[lp, v] + x_pl[lp, vp1])
                xt_pl[lp, v] = cand[np.argmin(_norm(cand - ctr))]
        xt_pl[:, 0] = x_pl[:, 0]
        R = RADIUS
        self.rscale = R
        x = x * R
        xt = xt * R
        x_pl = x_pl * R
        xt_pl = xt_pl * R
        xt[:, G - 1] = xt[:, G - 2]
        xt[:, :, G - 1] = xt[:, :, G - 2]
        self.x, self.x_pl, self.xt, self.xt_pl = x, x_pl, xt, xt_pl
        self.lat, self.lon = _latlon(x)
        self.lat_pl, self.lon_pl = _latlon(x_pl, pole_points=True)
        xr = np.full((L, G, G, 3, 3), UNDEF)
        xr[:, 0:gmax + 1, 1:gmax + 1, AI] = 0.5 * (xt[:, 0:gmax + 1, 0:gmax, TJ] + xt[:, 0:gmax + 1, 1:gmax + 1, TI])
        xr[:, 0:gmax + 1, 0:gmax + 1, AIJ] = 0.5 * (xt[:, 0:gmax + 1, 0:gmax + 1, TI] + xt[:, 0:gmax + 1, 0:gmax + 1, TJ])
        xr[:, 1:gmax + 1, 0:gmax + 1, AJ] = 0.5 * (xt[:, 1:gmax + 1, 0:gmax + 1, TJ] + xt[:, 0:gmax, 0:gmax + 1, TI])
        xr_pl = np.full((LP, 6, 3), UNDEF)
        for v in range(1, 6):
            vm1 = v - 1 if v > 1 else 5
            xr_pl[:, v] = 0.5 * (xt_pl[:, vm1] + xt_pl[:, v])
        self.xr, self.xr_pl = xr, xr_pl

    def _vertical(self, vlayer, ztop, h_efold):
        gz, gzh = vertical_levels(vlayer, ztop, self.layer)
        self.gz, self.gzh = gz, gzh
        self.vf = vertical_factors(gz, gzh)
        kall = len(gz)
        kmin, kmax = 1, kall - 2
        L, G = self.L, self.G
        # JW surface height (geopotential of the balanced state at eta = 1), or flat
        if self.topo == "JW":
            zs = self._jw_surface(self.lat)
            zs_pl = self._jw_surface(self.lat_pl)
        elif self.topo == "NONE":
            zs = np.zeros_like(self.lat)
            zs_pl = np.zeros_like(self.lat_pl)
        else:
            raise ValueError(f"unknown topography {self.topo!r}")
        htop = gzh[kmax + 1] - gzh[kmin]
        vz = np.zeros((L, G, G, kall, 2))
        vz_pl = np.zeros((LP, 6, kall, 2))
        sh = np.sinh(htop / h_efold)
        for k in range(kmin - 1, kmax + 2):
            vz[:, 1:G - 1, 1:G - 1, k, 0] = gz[k] + zs[:, 1:G - 1, 1:G - 1] * np.sinh((htop - gz[k]) / h_efold) / sh
            vz[:, 1:G - 1, 1:G - 1, k, 1] = gzh[k] + zs[:, 1:G - 1, 1:G - 1] * np.sinh((htop - gzh[k]) / h_efold) / sh
            vz_pl[:, 0, k, 0] = gz[k] + zs_pl[:, 0] * np.sinh((htop - gz[k]) / h_efold) / sh
            vz_pl[:, 0, k, 1] = gzh[k] + zs_pl[:, 0] * np.sinh((htop - gzh[k]) / h_efold) / sh
        self.exch(vz, vz_pl)
        self.vz, self.vz_pl = vz, vz_pl
        self.zs, self.zs_pl = zs, zs_pl

    @staticmethod
    def _jw_surface(lat):
        u0 = 35.0
        etav = (1.0 - 0.252) * (PI / 2.0)
        uc = u0 * np.cos(etav) ** 1.5
        f1 = -2.0 * np.sin(lat) ** 6 * (np.cos(lat) ** 2 + 1.0 / 3.0) + 10.0 / 63.0
        f2 = (8.0 / 5.0) * np.cos(lat) ** 3 * (np.sin(lat) ** 2 + 2.0 / 3.0) - PI / 4.0
        return uc * (uc * f1 + RADIUS * OHM * f2) / GRAV

    # -- share/mod_gmtr.py --------------------------------------------------
    def _gmtr(self):
        L, G, R = self.L, self.G, self.rscale
        gmin, gmax = 1, G - 2
        x, xt, x_pl, xt_pl = self.x, self.xt, self.x_pl, self.xt_pl
        sg = np.nonzero(self.have_sgp)[0]
        s, m = slice(gmin, gmax + 1), slice(gmin - 1, gmax)
        # cell polygons
        P = np.zeros((L, G, G, 8))
        ring = [xt[:, s, m, TJ], xt[:, s, s, TI], xt[:, s, s, TJ], xt[:, m, s, TI], xt[:, m, m, TJ],
                xt[:, m, m, TI].copy()]
        ring[5][sg, 0, 0] = ring[0][sg, 0, 0]
        ring.append(ring[0].copy())
        ring[6][sg, 0, 0] = ring[0][sg, 0, 0]
        c0 = x[:, s, s] / R
        ring = [r / R for r in ring]
        area = 0.0
        for v in range(6):
            area = area + _tri_area(c0, ring[v], ring[v + 1], R)
        P[:, s, s, 0] = area
        P[:, s, s, 1] = 1.0 / area
        sl, cl = np.sin(self.lon[:, s, s]), np.cos(self.lon[:, s, s])
        P[:, s, s, 2] = -sl
        P[:, s, s, 3] = cl
        P[:, s, s, 5] = -(x[:, s, s, 2] * cl) / R
        P[:, s, s, 6] = -(x[:, s, s, 2] * sl) / R
        P[:, s, s, 7] = (x[:, s, s, 0] * cl + x[:, s, s, 1] * sl) / R
        P_pl = np.zeros((LP, 6, 8))
        for lp in range(LP):
            w = [x_pl[lp, 0] / R] + [xt_pl[lp, v] / R for v in range(1, 6)] + [xt_pl[lp, 1] / R]
            a = 0.0
            for v in range(1, 6):
                a = a + _tri_area(w[0], w[v], w[v + 1], R)
            P_pl[lp, 0, 0] = a
            P_pl[lp, 0, 1] = 1.0 / a
            sl0, cl0 = np.sin(self.lon_pl[lp, 0]), np.cos(self.lon_pl[lp, 0])
            P_pl[lp, 0, 2] = -sl0
            P_pl[lp, 0, 3] = cl0
            P_pl[lp, 0, 5] = -(x_pl[lp, 0, 2] * cl0) / R
            P_pl[lp, 0, 6] = -(x_pl[lp, 0, 2] * sl0) / R
            P_pl[lp, 0, 7] = (x_pl[lp, 0, 0] * cl0 + x_pl[lp, 0, 1] * sl0) / R
        self.exch(P, P_pl)
        self.P, self.P_pl = P, P_pl
        # triangles: area, inverse, barycentric weights of the three cells
        T = np.zeros((L, G, G, 2, 5))
        e, e1 = slice(0, G - 1), slice(1, G)
        wk_t = {TI: [xt[:, e, e, TI].copy(), x[:, e, e].copy(), x[:, e1, e].copy(), x[:, e1, e1].copy()],
                TJ: [xt[:, e, e, TJ].copy(), x[:, e, e].copy(), x[:, e1, e1].copy(), x[:, e, e1].copy()]}
        for n in range(4):
            wk_t[TI][n][:, gmax, gmin - 1] = wk_t[TJ][n][:, gmax, gmin - 1]
            wk_t[TJ][n][:, gmin - 1, gmax] = wk_t[TI][n][:, gmin - 1, gmax]
            wk_t[TI][n][sg, gmin - 1, gmin - 1] = wk_t[TJ][n][sg, gmin, gmin - 1]
        for t, wk in wk_t.items():
            wk = [a / R for a in wk]
            a1 = _tri_area(wk[0], wk[2], wk[3], R)
            a2 = _tri_area(wk[0], wk[3], wk[1], R)
            a3 = _tri_area(wk[0], wk[1], wk[2], R)
            ar = a1 + a2 + a3
            T[:, e, e, t] = np.stack([ar, 1.0 / ar, a1 / ar, a2 / ar, a3 / ar], axis=-1)
        T_pl = np.zeros((LP, 6, 5))
        for lp in range(LP):
            for v in range(1, 6):
                vp1 = v + 1 if v < 5 else 1
                w0, w1, w2, w3 = (xt_pl[lp, v] / R, x_pl[lp, 0] / R, x_pl[lp, v] / R, x_pl[lp, vp1] / R)
                a1 = _tri_area(w0, w2, w3, R)
                a2 = _tri_area(w0, w3, w1, R)
                a3 = _tri_area(w0, w1, w2, R)
                ar = a1 + a2 + a3
                T_pl[lp, v] = [ar, 1.0 / ar, a1 / ar, a2 / ar, a3 / ar]
        self.T, self.T_pl = T, T_pl
        # arcs: tangent/normal of cell-centre arcs (TN, TT) and of hexagon edges (HN, HT)
        A = np.zeros((L, G, G, 3, 12))
        # AI cell arcs: (i,j) -> (i+1,j), i in [0, G-2], j in [0, G-1]
        f = x[:, 0:G - 1, :].copy()
        t = x[:, 1:G, :].copy()
        f[:, gmax, gmin - 1] = x[:, gmax, gmin - 1]
        t[:, gmax, gmin - 1] = x[:, gmax, gmin]
        f[:, gmin - 1, gmax + 1] = x[:, gmin, gmax + 1]
        t[:, gmin - 1, gmax + 1] = x[:, gmin, gmax]
        f[sg, gmin - 1, gmin - 1] = x[sg, gmin, gmin - 1]
        t[sg, gmin - 1, gmin - 1] = x[sg, gmin + 1, gmin]
        tt, tn = _tn_vectors(f, t, R)
        A[:, 0:G - 1, :, AI, 6:9] = tn
        A[:, 0:G - 1, :, AI, 9:12] = tt
        # AIJ cell arcs: (i,j) -> (i+1,j+1)
        tt, tn = _tn_vectors(x[:, 0:G - 1, 0:G - 1], x[:, 1:G, 1:G], R)
        A[:, 0:G - 1, 0:G - 1, AIJ, 6:9] = tn
        A[:, 0:G - 1, 0:G - 1, AIJ, 9:12] = tt
        # AJ cell arcs: (i,j) -> (i,j+1), i in [0, G-1], j in [0, G-2]
        f = x[:, :, 0:G - 1].copy()
        t = x[:, :, 1:G].copy()
        f[:, gmax + 1, gmin - 1] = x[:, gmax + 1, gmin]
        t[:, gmax + 1, gmin - 1] = x[:, gmax, gmin]
        f[:, gmin - 1, gmax] = x[:, gmin - 1, gmax]
        t[:, gmin - 1, gmax] = x[:, gmin, gmax]
        tt, tn = _tn_vectors(f, t, R)
        A[:, :, 0:G - 1, AJ, 6:9] = tn
        A[:, :, 0:G - 1, AJ, 9:12] = tt
        # AI hexagon edges: xt(i,j,TI) -> xt(i,j-1,TJ), i in [0, G-2], j in [1, G-2]
        tt, tn = _tn_vectors(xt[:, 0:G - 1, 1:G - 1, TI], xt[:, 0:G - 1, 0:G - 2, TJ], R)
        A[:, 0:G - 1, 1:G - 1, AI, 0:3] = tn
        A[:, 0:G - 1, 1:G - 1, AI, 3:6] = tt
        # AIJ hexagon edges: xt(i,j,TJ) -> xt(i,j,TI), i, j in [0, G-2]
        f = xt[:, 0:G - 1, 0:G - 1, TJ].copy()
        t = xt[:, 0:G - 1, 0:G - 1, TI].copy()
        f[:, gmax, gmin - 1] = xt[:, gmax, gmin - 1, TJ]
        t[:, gmax, gmin - 1] = xt[:, gmax, gmin, TI]
        f[:, gmin - 1, gmax] = xt[:, gmin, gmax, TJ]
        t[:, gmin - 1, gmax] = xt[:, gmin - 1, gmax, TI]
        tt, tn = _tn_vectors(f, t, R)
        A[:, 0:G - 1, 0:G - 1, AIJ, 0:3] = tn
        A[:, 0:G - 1, 0:G - 1, AIJ, 3:6] = tt
        # AJ hexagon edges: xt(i-1,j,TI) -> xt(i,j,TJ), i in [1, G-2], j in [0, G-2]
        f = xt[:, 0:G - 2, 0:G - 1, TI].copy()
        t = xt[:, 1:G - 1, 0:G - 1, TJ].copy()
        f[sg, 0, 0] = xt[sg, gmin, gmin, TI]
        t[sg, 0, 0] = xt[sg, gmin, gmin - 1, TJ]
        tt, tn = _tn_vectors(f, t, R)
        A[:, 1:G - 1, 0:G - 1, AJ, 0:3] = tn
        A[:, 1:G - 1, 0:G - 1, AJ, 3:6] = tt
        A_pl = np.zeros((LP, 6, 18))
        for lp in range(LP):
            for v in range(1, 6):
                vp1 = v + 1 if v < 5 else 1
                vm1 = v - 1 if v > 1 else 5
                tt, tn = _tn_vectors(x_pl[lp, 0], x_pl[lp, v], R)
                A_pl[lp, v, 6:9], A_pl[lp, v, 9:12] = tn, tt
                tt, tn = _tn_vectors(x_pl[lp, v], x_pl[lp, vp1], R)
                A_pl[lp, v, 12:15], A_pl[lp, v, 15:18] = tn, tt
                tt, tn = _tn_vectors(xt_pl[lp, vm1], xt_pl[lp, v], R)
                A_pl[lp, v, 0:3], A_pl[lp, v, 3:6] = tn, tt
        self.A, self.A_pl = A, A_pl

    # -- share/mod_oprt.py: one ring formulation ------------------------------
    def _ring(self):
        """For every interior cell: the six triangles around it (CCW from
        TI(i,j)) and the six hexagon edges between them, with edge signs, the
        barycentric weight index of the centre cell and of each neighbour."""
        G = self.G
        s, m = slice(1, G - 1), slice(0, G - 2)
        p = slice(2, G)
        T, A = self.T, self.A
        tri = [T[:, s, s, TI], T[:, s, s, TJ], T[:, m, s, TI], T[:, m, m, TJ], T[:, m, m, TI], T[:, s, m, TJ]]
        edge = [A[:, s, s, AI], A[:, s, s, AIJ], A[:, s, s, AJ], A[:, m, s, AI], A[:, m, m, AIJ], A[:, s, m, AJ]]
        sign = [1.0, 1.0, 1.0, -1.0, -1.0, -1.0]
        # triangle edge (cell-arc) TN vectors e01, e12, e02 of each ring triangle
        tn = lambda a: a[..., 6:9]
        tri_e = [
            (tn(A[:, s, s, AI]), tn(A[:, p, s, AJ]), tn(A[:, s, s, AIJ])),            # TI(i,j)
            (tn(A[:, s, s, AIJ]), -tn(A[:, s, p, AI]), tn(A[:, s, s, AJ])),           # TJ(i,j)
            (tn(A[:, m, s, AI]), tn(A[:, s, s, AJ]), tn(A[:, m, s, AIJ])),            # TI(i-1,j)
            (tn(A[:, m, m, AIJ]), -tn(A[:, m, s, AI]), tn(A[:, m, m, AJ])),           # TJ(i-1,j-1)
            (tn(A[:, m, m, AI]), tn(A[:, s, m, AJ]), tn(A[:, m, m, AIJ])),            # TI(i-1,j-1)
            (tn(A[:, s, m, AIJ]), -tn(A[:, s, s, AI]), tn(A[:, s, m, AJ])),           # TJ(i,j-1)
        ]
        # role (vertex 0/1/2) of the centre cell in each ring triangle and of
        # neighbour n (1..6, directions (i+1,j),(i+1,j+1),(i,j+1),(i-1,j),(i-1,j-1),(i,j-1))
        role_c = [0, 0, 1, 1, 2, 2]
        role_n = {1: {5: 1, 0: 1}, 2: {0: 2, 1: 1}, 3: {1: 2, 2: 2}, 4: {2: 0, 3: 2}, 5: {3: 0, 4: 0},
                  6: {4: 1, 5: 0}}
        return tri, edge, sign, tri_e, role_c, role_n

    def _oprt(self):
        L, G = self.L, self.G
        s = slice(1, G - 1)
        tri, edge, sign, tri_e, role_c, role_n = self._ring()
        rarea = self.P[:, s, s, 1]
        sg = np.nonzero(self.have_sgp)[0]
        hn = lambda e: e[..., 0:3]
        # ring members per cell type: hexagon uses triangles 0..5 with edges k, k+1;
        # the pentagon corner drops triangle 4 and closes triangle 5 on edge 4
        hexa = [(k, k, (k + 1) % 6) for k in range(6)]
        penta = [(0, 0, 1), (1, 1, 2), (2, 2, 3), (3, 3, 4), (5, 4, 0)]

        def assemble(members, pick):
            """pick(c) -> values at the cells selected by c (slice/index)"""
            div = np.zeros(pick(rarea).shape + (3, 7))
            grad = np.zeros_like(div)
            lap = np.zeros(pick(rarea).shape + (7,))
            wcol = lambda role: 2 + role                          # W1, W2, W3 columns
            gw = {0: (-1.0, 2.0, 1.0), 1: (-1.0, -1.0, -2.0), 2: (2.0, -1.0, 1.0)}
            tri_k = [pick(t) for t in tri]
            edge_k = [pick(hn(e)) for e in edge]
            te_k = [tuple(pick(v) for v in te) for te in tri_e]
            clos = 0.0
            for (k, eb, ea) in members:
                flux = sign[eb] * edge_k[eb] + sign[ea] * edge_k[ea]              # (..., 3)
                # centre cell
                div[..., 0] += tri_k[k][..., wcol(role_c[k])][..., None] * flux
                g = sum(c * v for c, v in zip(gw[role_c[k]], te_k[k]))
                lap[..., 0] += tri_k[k][..., 1] * (sign[eb] * _dot(g, edge_k[eb]) + sign[ea] * _dot(g, edge_k[ea]))
                for n in range(1, 7):
                    if k in role_n[n]:
                        r = role_n[n][k]
                        div[..., n] += tri_k[k][..., wcol(r)][..., None] * flux
                        g = sum(c * v for c, v in zip(gw[r], te_k[k]))
                        lap[..., n] += tri_k[k][..., 1] * (sign[eb] * _dot(g, edge_k[eb])
                                                          + sign[ea] * _dot(g, edge_k[ea]))
                clos = clos + sign[eb] * edge_k[eb]
            grad[...] = div
            grad[..., 0] = grad[..., 0] - 2.0 * clos
            ra = pick(rarea)
            div = div * 0.5 * ra[..., None, None]
            grad = grad * 0.5 * ra[..., None, None]
            lap = lap * (ra / 12.0)[..., None]
            return div, grad, lap

        cdiv = np.zeros((L, G, G, 3, 7))
        cgrad = np.zeros_like(cdiv)
        clap = np.zeros((L, G, G, 7))
        d, g_, lp_ = assemble(hexa, lambda a: a)
        cdiv[:, s, s], cgrad[:, s, s], clap[:, s, s] = d, g_, lp_
        d, g_, lp_ = assemble(penta, lambda a: a[sg, 0, 0])
        cdiv[sg, 1, 1], cgrad[sg, 1, 1], clap[sg, 1, 1] = d, g_, lp_
        # interpolation of the triangle gradient and hexagon-edge diffusion coefficients
        A, T = self.A, self.T
        e, e1 = slice(0, G - 1), slice(1, G)
        tn = lambda a: a[..., 6:9]
        cint = np.zeros((L, G, G, 3, 3, 2))
        for t, (e01, e12, e02) in ((TI, (tn(A[:, e, e, AI]), tn(A[:, e1, e, AJ]), tn(A[:, e, e, AIJ]))),
                                   (TJ, (tn(A[:, e, e, AIJ]), -tn(A[:, e, e1, AI]), tn(A[:, e, e, AJ])))):
            h = 0.5 * T[:, e, e, t, 1][..., None]
            cint[:, e, e, :, 0, t] = (e02 - e01) * h
            cint[:, e, e, :, 1, t] = (-e01 - e12) * h
            cint[:, e, e, :, 2, t] = (-e12 + e02) * h
        m = slice(0, G - 2)
        cdiff = np.zeros((L, G, G, 3, 6))
        hr = 0.5 * rarea[..., None]
        for n, (a, sgn) in enumerate(((A[:, s, s, AIJ], 1.0), (A[:, s, s, AJ], 1.0), (A[:, m, s, AI], -1.0),
                                      (A[:, m, m, AIJ], -1.0), (A[:, s, m, AJ], -1.0), (A[:, s, s, AI], 1.0))):
            cdiff[:, s, s, :, n] = sgn * a[..., 0:3] * hr
        cdiff[sg, 1, 1, :, 4] = 0.0
        # pole rows
        T_pl, A_pl, P_pl = self.T_pl, self.A_pl, self.P_pl
        div_pl = np.zeros((LP, 6, 3))
        grad_pl = np.zeros((LP, 6, 3))
        lap_pl = np.zeros((LP, 6))
        int_pl = np.zeros((LP, 6, 3, 3))
        diff_pl = np.zeros((LP, 6, 3))
        for l in range(LP):
            ra = P_pl[l, 0, 1]
            HN = lambda v: A_pl[l, v, 0:3]
            TN = lambda v: A_pl[l, v, 6:9]
            TN2 = lambda v: A_pl[l, v, 12:15]
            W = lambda v, c: T_pl[l, v, 2 + c]
            TR = lambda v: T_pl[l, v, 1]
            nx = lambda v: v + 1 if v < 5 else 1
            pv = lambda v: v - 1 if v > 1 else 5
            acc = np.zeros(3)
            accg = np.zeros(3)
            accl = 0.0
            for v in range(1, 6):
                acc = acc + (W(v, 0) * HN(v) + W(v, 0) * HN(nx(v)))
                accg = accg + 2.0 * (W(v, 0) - 1.0) * HN(nx(v))
                gpm = TN(pv(v)) - 2.0 * TN2(pv(v)) - TN(v)
                gp = TN(v) - 2.0 * TN2(v) - TN(nx(v))
                accl = accl + TR(pv(v)) * _dot(gpm, HN(v)) + TR(v) * _dot(gp, HN(v))
            div_pl[l, 0] = acc * 0.5 * ra
            grad_pl[l, 0] = accg * 0.5 * ra
            lap_pl[l, 0] = accl
            for v in range(1, 6):
                row = (W(pv(v), 2) * HN(pv(v)) + W(pv(v), 2) * HN(v) + W(v, 1) * HN(v) + W(v, 1) * HN(nx(v)))
                div_pl[l, v] = row * 0.5 * ra
                grad_pl[l, v] = div_pl[l, v]
                ga = -2.0 * TN(pv(v)) + TN2(pv(v)) - TN(v)
                gb = TN(v) + TN2(v) + 2.0 * TN(nx(v))
                lap_pl[l, v] = (TR(pv(v)) * (_dot(ga, HN(pv(v))) + _dot(ga, HN(v)))
                                + TR(v) * (_dot(gb, HN(v)) + _dot(gb, HN(nx(v)))))
                int_pl[l, v, :, 0] = (-TN(nx(v)) + TN(v)) * (0.5 * TR(v))
                int_pl[l, v, :, 1] = (TN(v) + TN2(v)) * (0.5 * TR(v))
                int_pl[l, v, :, 2] = (TN2(v) - TN(nx(v))) * (0.5 * TR(v))
                diff_pl[l, v] = HN(v) * 0.5 * ra
            lap_pl[l] = lap_pl[l] * (ra / 12.0)
        self.coef = dict(div=cdiv, grad=cgrad, lap=clap, intp=cint, diff=cdiff)
        self.coef_pl = dict(div=div_pl, grad=grad_pl, lap=lap_pl, intp=int_pl, diff=diff_pl)

    # -- share/mod_vmtr.py --------------------------------------------------
    def _gradient(self, sc, sc_pl):
        """horizontal gradient (L,G,G,K) -> (L,G,G,K,3) on interior cells, pole row"""
        G = self.G
        s = slice(1, G - 1)
        nb = [(0, 0), (1, 0), (1, 1), (0, 1), (-1, 0), (-1, -1), (0, -1)]
        cg = self.coef["grad"][:, s, s]
        out = np.zeros(sc.shape + (3,))
        for d in range(3):
            acc = 0.0
            for n, (di, dj) in enumerate(nb):
                acc = acc + cg[..., d, n][..., None] * sc[:, 1 + di:G - 1 + di, 1 + dj:G - 1 + dj]
            out[:, s, s, :, d] = acc
        out_pl = np.zeros(sc_pl.shape + (3,))
        for d in range(3):
            out_pl[:, 0, :, d] = sum(self.coef_pl["grad"][:, v, d][:, None] * sc_pl[:, v] for v in range(6))
        return out, out_pl

    def _horizontalize(self, v, v_pl):
        G, R = self.G, self.rscale
        s = slice(1, G - 1)
        gx = self.x[:, s, s][:, :, :, None, :]
        w = v[:, s, s]
        prd = (w[..., 0] * gx[..., 0] + w[..., 1] * gx[..., 1] + w[..., 2] * gx[..., 2]) / R
        v[:, s, s] = w - (prd[..., None] * gx) / R
        gp = self.x_pl[:, :, None, :]
        prd = v_pl[..., 0] * gp[..., 0] / R + v_pl[..., 1] * gp[..., 1] / R + v_pl[..., 2] * gp[..., 2] / R
        v_pl[...] = v_pl - (prd[..., None] * gp) / R

    def _vmtr(self):
        vf = self.vf
        kall = self.kall
        kmin, kmax = 1, kall - 2
        vz, vz_pl = self.vz, self.vz_pl
        var = np.zeros(vz.shape[:4] + (6,))
        var_pl = np.zeros(vz_pl.shape[:3] + (6,))
        for half, off in ((1, 0), (0, 3)):
            g, gp = self._gradient(vz[..., half], vz_pl[..., half])
            self._horizontalize(g, gp)
            var[..., off:off + 3] = g
            var_pl[..., off:off + 3] = gp
        self.exch(var, var_pl)
        out = {}
        with np.errstate(invalid="ignore", divide="ignore"):
            for sfx, z, v in (("", vz, var), ("_pl", vz_pl, var_pl)):
                gsq = np.zeros(z.shape[:-1])
                gsqh = np.zeros(z.shape[:-1])
                for k in range(kmin, kmax + 1):
                    gsq[..., k] = (z[..., k + 1, 1] - z[..., k, 1]) / vf["dgz"][k]
                gsq[..., kmin - 1] = gsq[..., kmin]
                gsq[..., kmax + 1] = gsq[..., kmax]
                for k in range(kmin, kmax + 2):
                    gsqh[..., k] = (z[..., k, 0] - z[..., k - 1, 0]) / vf["dgzh"][k]
                gsqh[..., kmin - 1] = gsqh[..., kmin]
                one = np.ones_like(gsq)
                gs2 = one * one * gsq
                gs2h = one * one * gsqh
                rgs2 = 1.0 / gs2
                rgs2h = 1.0 / gs2h
                c2w = np.zeros(gsq.shape + (2,))
                w2c = np.zeros(gsq.shape + (2,))
                c2wgz = np.zeros(gsq.shape + (6,))
                gzh = [-v[..., c] / gsqh for c in (0, 1, 2)]
                for k in range(kmin, kmax + 2):
                    a = vf["afact"][k] * rgs2[..., k] * gs2h[..., k]
                    b = vf["bfact"][k] * rgs2[..., k - 1] * gs2h[..., k]
                    c2w[..., k, 0], c2w[..., k, 1] = a, b
                    for c in range(3):
                        c2wgz[..., k, 2 * c] = vf["afact"][k] * rgs2[..., k] * gs2h[..., k] * gzh[c][..., k]
                        c2wgz[..., k, 2 * c + 1] = vf["bfact"][k] * rgs2[..., k - 1] * gs2h[..., k] * gzh[c][..., k]
                for k in range(kmin - 1, kmax + 1):
                    w2c[..., k, 0] = vf["cfact"][k] * gs2[..., k] * rgs2h[..., k + 1]
                    w2c[..., k, 1] = vf["dfact"][k] * gs2[..., k] * rgs2h[..., k]
                area = self.P[..., 0] if sfx == "" else self.P_pl[..., 0]
                vol = area[..., None] * gs2 * vf["dgz"]
                out["GSGAM2" + sfx], out["GSGAM2H" + sfx] = gs2, gs2h
                out["RGSGAM2" + sfx], out["RGSGAM2H" + sfx] = rgs2, rgs2h
                out["RGSQRTH" + sfx] = 1.0 / gsqh
                out["RGAM" + sfx], out["RGAMH" + sfx], out["GAM2H" + sfx] = one / one, one / one, one * one
                out["C2Wfact" + sfx], out["W2Cfact" + sfx], out["C2WfactGz" + sfx] = c2w, w2c, c2wgz
                out["VOLUME" + sfx] = vol
                out["PHI" + sfx] = z[..., 0] * GRAV
        for k, a in out.items():
            out[k] = np.nan_to_num(a, nan=0.0, posinf=0.0, neginf=0.0)
        self.vmtr = out

    # -- JW initial state (nhm/share/mod_ideal_init.py) ----------------------
    @staticmethod
    def _jw_steady(eta, lat):
        eta0, etaT, t0, delT, gam, u0 = 0.252, 0.2, 288.0, 4.8e5, 0.005, 35.0
        w1 = PI / 2.0
        w2 = RDRY * gam / GRAV
        ev = (eta - eta0) * w1
        wix = u0 * np.cos(ev) ** 1.5 * (np.sin(2.0 * lat)) ** 2
        ew2 = eta ** w2
        tmp_hi = t0 * ew2
        geo_hi = t0 * GRAV / gam * (1.0 - ew2)
        tmp_lo = t0 * ew2 + delT * (etaT - eta) ** 5
        geo_lo = (t0 * GRAV / gam * (1.0 - ew2) - RDRY * delT *
                  ((np.log(eta / etaT) + 137.0 / 60.0) * etaT ** 5 - 5.0 * etaT ** 4 * eta
                   + 5.0 * etaT ** 3 * eta ** 2 - (10.0 / 3.0) * etaT ** 2 * eta ** 3
                   + (5.0 / 4.0) * etaT * eta ** 4 - (1.0 / 5.0) * eta ** 5))
        hi = eta >= etaT
        tmp = np.where(hi, tmp_hi, tmp_lo)
        geo = np.where(hi, geo_hi, geo_lo)
        w2b = 3.0 / 4.0 * (PI * u0 / RDRY)
        cs32 = np.cos(ev) ** 1.5
        A = (-2.0 * (np.sin(lat)) ** 6 * (np.cos(lat) ** 2 + 1.0 / 3.0) + 10.0 / 63.0)
        B = (8.0 / 5.0 * (np.cos(lat)) ** 3 * ((np.sin(lat)) ** 2 + 2.0 / 3.0) - PI / 4.0)
        tmp = tmp + w2b * eta * np.sin(ev) * np.cos(ev) ** 0.5 * (A * 2.0 * u0 * cs32 + B * RADIUS * OHM)
        geo = geo + u0 * cs32 * (A * u0 * cs32 + B * RADIUS * OHM)
        return tmp, geo, wix

    def _jw_columns(self, z, lat, lon):
        """z (..., kall) heights, lat/lon (...): returns pre, tem, vx, vy, vz (..., kall)"""
        latk = lat[..., None]
        crit = max(EPS * 10.0, 1.0e-14)
        eta = np.full(z.shape, 1.0e-7)
        tmp, geo, wix = self._jw_steady(eta, latk)
        active = np.ones(z.shape[:-1], bool)
        for _ in range(1, 100):
            F = -GRAV * z + geo
            Feta = -(RDRY / eta) * tmp
            en = np.maximum(np.minimum(eta - F / Feta, 1.0), EPS)
            am = active[..., None]
            diff = np.where(am, np.abs(en - eta), 0.0)
            eta = np.where(am, en, eta)
            newly = np.max(diff, axis=-1) < crit
            tn, gn, wn = self._jw_steady(eta, latk)
            tmp = np.where(am, tn, tmp)
            geo = np.where(am, gn, geo)
            wix = np.where(am, wn, wix)
            active = active & ~newly
            if not active.any():
                break
        # hydrostatic-gradient-wind pressure, upward: trapezoid then Simpson
        cosl = np.cos(lat)
        kdim = z.shape[-1]
        pp = np.zeros(z.shape)
        pp[..., 0] = 1.0e5
        for k in range(1, kdim):
            dz = (geo[..., k] - geo[..., k - 1]) / GRAV
            ua = (wix[..., k] + wix[..., k - 1]) * 0.5
            fcf = 2.0 * OHM * ua * cosl + ua ** 2 / RADIUS
            num = 1.0 + dz * (fcf - GRAV) / (2.0 * RDRY * tmp[..., k - 1])
            den = 1.0 - dz * (fcf - GRAV) / (2.0 * RDRY * tmp[..., k])
            pp[..., k] = pp[..., k - 1] * num / den
        prs = pp.copy()
        for k in range(2, kdim):
            dz = (geo[..., k] - geo[..., k - 2]) / GRAV * 0.5
            f = [2.0 * OHM * u * cosl + u ** 2 / RADIUS for u in (wix[..., k], wix[..., k - 1], wix[..., k - 2])]
            r = [prs[..., k - n] / (RDRY * tmp[..., k - n]) for n in (0, 1, 2)]
            fac = (1.0 / 3.0) * r[0] * (f[0] - GRAV) + (4.0 / 3.0) * r[1] * (f[1] - GRAV) \
                + (1.0 / 3.0) * r[2] * (f[2] - GRAV)
            pp[..., k] = prs[..., k - 2] + fac * dz
        lonk = lon[..., None]
        ex, ey = -np.sin(lonk), np.cos(lonk)
        nxv, nyv, nzv = -np.sin(latk) * np.cos(lonk), -np.sin(latk) * np.sin(lonk), np.cos(latk)
        zero = np.zeros_like(wix)
        vx = ex * wix + nxv * zero
        vy = ey * wix + nyv * zero
        vzz = nzv * zero
        # 1 m/s zonal-wind bump centred at 20E / 40N
        cla, clo = 40.0 * (PI / 180.0), 20.0 * (PI / 180.0)
        r = RADIUS * np.arccos(np.sin(cla) * np.sin(lat) + np.cos(cla) * np.cos(lat) * np.cos(lon - clo))
        pw = (1.0 * np.exp(-(r / (RADIUS / 10.0)) ** 2))[..., None]
        vx = vx + (ex * pw + nxv * np.zeros_like(pw))
        vy = vy + (ey * pw + nyv * np.zeros_like(pw))
        vzz = vzz + nzv * np.zeros_like(pw)
        return pp, tmp, vx, vy, vzz

    def _jw_chunked(self, z, lat, lon):
        """the column solve over chunks of the leading axis on host threads
        (every operation is per column, so chunking does not change results)"""
        n = z.shape[0]
        workers = min(n, os.cpu_count() or 1, 16)
        if workers <= 1 or z.size < 1_000_000:
            return self._jw_columns(z, lat, lon)
        from concurrent.futures import ThreadPoolExecutor
        bounds = np.linspace(0, n, workers + 1).astype(int)
        with ThreadPoolExecutor(workers) as ex:
            parts = list(ex.map(lambda b: self._jw_columns(z[b[0]:b[1]], lat[b[0]:b[1]], lon[b[0]:b[1]]),
                                zip(bounds[:-1], bounds[1:])))
        return tuple(np.concatenate([p[v] for p in parts], axis=0) for v in range(5))

    def _diag_to_prg(self, diag, diag_pl, q=None, q_pl=None):
        """PRG_var / PRG_var_pl in the reference layout from the diagnostic
        columns (pre, tem, vx, vy, vz, w) in region-major layout and optional
        tracer mixing ratios (..., nq) (the reference's cnvvar diag -> prg for a
        dry state: rho = p / (Rdry T), RHOG = rho GSGAM2, RHOGV = RHOG v,
        RHOGE = RHOG cv T, RHOGW = rho_h w, RHOGQ = RHOG q)"""
        prg = []
        for d, qq, sfx in ((diag, q, ""), (diag_pl, q_pl, "_pl")):
            gs2 = self.vmtr["GSGAM2" + sfx]
            c2w = self.vmtr["C2Wfact" + sfx]
            pre, tem = d[..., 0], d[..., 1]
            qv = np.zeros(pre.shape)
            cv = 0.0 + qv * CVDRY
            qd = 1.0 - qv
            cv = cv + qd * CVDRY
            rho = pre / ((qd * RDRY + qv * RVAP) * tem)
            ein = tem * cv
            nq = 1 if qq is None else qq.shape[-1]
            P = np.zeros(pre.shape + (6 + nq,))
            P[..., 0] = rho * gs2
            P[..., 1] = P[..., 0] * d[..., 2]
            P[..., 2] = P[..., 0] * d[..., 3]
            P[..., 3] = P[..., 0] * d[..., 4]
            P[..., 5] = P[..., 0] * ein
            rh = np.zeros(pre.shape)
            rh[..., 1:] = c2w[..., 1:, 0] * P[..., 1:, 0] + c2w[..., 1:, 1] * P[..., :-1, 0]
            rh[..., 0] = rh[..., 1]
            P[..., 4] = rh * d[..., 5]
            if qq is not None:
                P[..., 6:] = P[..., 0:1] * qq
            prg.append(P)
        return (np.ascontiguousarray(prg[0].transpose(1, 2, 3, 0, 4)),
                np.ascontiguousarray(prg[1].transpose(1, 2, 0, 3)))

    def _column_coords(self):
        """per region-major grid (regional, pole): (z, lat, lon) of the state
        evaluation -- full-level heights with the bottom dummy level at the
        lowest half level, the column latitude / longitude (the pole columns
        like the region halo cells that carry the pole point)"""
        kmin, kmax = 1, self.kall - 2
        lat_p, lon_p = _latlon(self.x_pl)
        out = []
        for z3, lat, lon in ((self.vz, self.lat, self.lon), (self.vz_pl, lat_p, lon_p)):
            z = np.zeros(z3.shape[:-1])
            z[..., kmin - 1] = z3[..., kmin, 1]
            z[..., kmin:kmax + 2] = z3[..., kmin:kmax + 2, 0]
            out.append((z, lat, lon))
        return out

    def jw_state(self, nq: int = 1):
        """JW balanced jet + perturbation as PRG_var (G, G, kall, L, 6+nq) and
        PRG_var_pl (6, kall, 2, 6+nq) in the reference layout."""
        out = [self._jw_chunked(z, lat, lon) for z, lat, lon in self._column_coords()]
        diag = np.stack(out[0] + (np.zeros_like(out[0][0]),), axis=-1)        # (L,G,G,K,6) pre,tem,vx,vy,vz,w
        diag_pl = np.stack(out[1] + (np.zeros_like(out[1][0]),), axis=-1)
        self.exch(diag, diag_pl)
        s, s_pl = self._diag_to_prg(diag, diag_pl)
        if nq != 1:
            s = np.concatenate([s[..., :6], np.zeros(s.shape[:4] + (nq,))], axis=-1)
            s_pl = np.concatenate([s_pl[..., :6], np.zeros(s_pl.shape[:3] + (nq,))], axis=-1)
        return s, s_pl

    @staticmethod
    def dcmip11_fields(lon, lat, z):
        """DCMIP2012 test 1-1 (3-D deformational flow) at time 0 on columns of
        longitude / latitude and heights z (..., kall): pressure, temperature,
        zonal / meridional / vertical wind, and the test's own four tracers
        (restating nhm/share/mod_dcmip_ic.py test1_advection_deformation:
        isothermal T0 = 300 K, p = p0 exp(-z / H), period 12 days)"""
        a, Rd, g, p0, pi = 6371220.0, 287.0, 9.80616, 100000.0, 3.141592653589793238
        tau = 12.0 * 86400.0
        u0 = (2.0 * pi * a) / tau
        k0 = (10.0 * a) / tau
        omega0 = (23000.0 * pi) / tau
        T0 = 300.0
        H = Rd * T0 / g
        lon = lon[..., None]
        lat = lat[..., None]
        p = p0 * np.exp(-z / H)
        ptop = p0 * np.exp(-12000.0 / H)
        bs = 0.2
        sfac = (1.0 + np.exp((ptop - p0) / (bs * ptop)) - np.exp((p - p0) / (bs * ptop)) -
                np.exp((ptop - p) / (bs * ptop)))
        ud = (omega0 * a) / (bs * ptop) * np.cos(lon) * (np.cos(lat) ** 2) * (
            -np.exp((p - p0) / (bs * ptop)) + np.exp((ptop - p) / (bs * ptop)))
        u = k0 * np.sin(lon) * np.sin(lon) * np.sin(2.0 * lat) + u0 * np.cos(lat) + ud
        v = k0 * np.sin(2.0 * lon) * np.cos(lat)
        w = -((Rd * T0) / (g * p)) * omega0 * np.sin(lon) * np.cos(lat) * sfac
        t = np.full_like(p, T0)
        RR, ZZ, z0 = 0.5, 1000.0, 5000.0
        lam0, lam1 = 5.0 * pi / 6.0, 7.0 * pi / 6.0
        r = np.arccos(np.sin(lat) * 0.0 + np.cos(lat) * 1.0 * np.cos(lon - lam0))
        r2 = np.arccos(np.sin(lat) * 0.0 + np.cos(lat) * 1.0 * np.cos(lon - lam1))
        d1 = np.minimum(1.0, (r / RR) ** 2 + ((z - z0) / ZZ) ** 2)
        d2 = np.minimum(1.0, (r2 / RR) ** 2 + ((z - z0) / ZZ) ** 2)
        q1 = 0.5 * (1.0 + np.cos(pi * d1)) + 0.5 * (1.0 + np.cos(pi * d2))
        q2 = 0.9 - 0.8 * q1 ** 2
        q3 = np.where((d1 <= RR) | (d2 <= RR), 1.0, 0.1)
        q3 = np.where((z > z0) & (np.abs(lat) < 0.125), 0.1, q3)
        q4 = 1.0 - 0.3 * (q1 + q2 + q3)
        shape = p.shape
        u, v, w = (np.broadcast_to(x, shape) for x in (u, v, w))
        return p, t, u, v, w, np.stack([np.broadcast_to(x, shape) for x in (q1, q2, q3, q4)], axis=-1)

    def trcadv_state(self, tracers=None):
        """The DCMIP 1-1 offline tracer-advection state (initial winds, the
        isothermal atmosphere) as PRG_var / PRG_var_pl.  ``tracers``: a
        function (lon, lat, z) -> mixing ratios (..., kall, nq) on the state's
        columns; default the test's own four tracers."""
        diag, qs = [], []
        for z, lat, lon in self._column_coords():
            p, t, u, v, w, q4 = self.dcmip11_fields(lon, lat, z)
            lonk, latk = lon[..., None], lat[..., None]
            ex, ey = -np.sin(lonk), np.cos(lonk)
            nx, ny, nz = -np.sin(latk) * np.cos(lonk), -np.sin(latk) * np.sin(lonk), np.cos(latk)
            d = np.stack([p, t, ex * u + nx * v, ey * u + ny * v, nz * v, w], axis=-1)
            diag.append(d)
            qs.append(q4 if tracers is None else tracers(lon, lat, z))
        self.exch(diag[0], diag[1])
        for n in range(qs[0].shape[-1]):
            a, b = np.ascontiguousarray(qs[0][..., n]), np.ascontiguousarray(qs[1][..., n])
            self.exch(a, b)
            qs[0][..., n], qs[1][..., n] = a, b
        return self._diag_to_prg(diag[0], diag[1], qs[0], qs[1])

    # -- the setup dict of NicamCuda ----------------------------------------
    def setup(self, dtl: float, gamma: float, nq: int = 1, trcadv: bool = False) -> dict:
        """Setup arrays in the reference's attribute names and layouts;
        ``trcadv``: the offline tracer-advection configuration (integ_type
        TRCADV, no acoustic steps) with the coordinates its prescribed winds
        are computed from."""
        L, G, K = self.L, self.G, self.kall
        # regional (L,G,G,K,...) -> (G,G,K,L,...)
        to3 = lambda a: np.ascontiguousarray(np.moveaxis(a, 0, 3))
        # regional 2-D (L,G,G,...) -> (G,G,1,L,...)
        to2 = lambda a: np.ascontiguousarray(np.moveaxis(a, 0, 2)[:, :, None])
        # pole 3-D (2,6,K,...) -> (6,K,2,...)
        pl3 = lambda a: np.ascontiguousarray(np.moveaxis(a, 0, 2))
        # pole 2-D (2,6,...) -> (6,1,2,...)
        pl2 = lambda a: np.ascontiguousarray(np.moveaxis(a, 0, 1)[:, None])
        g = dict(kall=K, kmin=1, kmax=K - 2, gall_1d=G, gmin=1, gmax=G - 2, lall=L, nq=nq,
                 have_sgp=self.have_sgp.copy(),
                 pntmask=np.stack([(~self.have_sgp).astype(np.int32), self.have_sgp.astype(np.int32)],
                                  axis=-1)[None],
                 GRAV=GRAV, Rdry=RDRY, CVdry=CVDRY, CPdry=CPDRY, Rvap=RVAP, OHM=OHM, RADIUS=RADIUS, EPS=EPS,
                 HUGE=HUGE, PRE00=PRE00, rscale=self.rscale, alpha=1.0, dtl=float(dtl), dts=float(dtl) / 6.0,
                 Kh_coef=float(gamma), divdamp_coef=float(gamma), hdiff_fact_rho=1.0e-2,
                 sstep=np.array([2, 3, 6]), CVW=np.array([CVDRY] * nq), NQW_END=np.asarray(0))
        for k, v in self.exch.lists.items():
            g["copy_" + k] = v
        g["GRD_gz"], g["GRD_gzh"] = self.gz, self.gzh
        for k in ("afact", "bfact", "cfact", "dfact", "rdgz", "rdgzh"):
            g["GRD_" + k] = self.vf[k]
        g["GRD_x"] = to2(self.x)
        g["GRD_x_pl"] = pl2(self.x_pl)
        g["GRD_xr"] = to2(self.xr)
        g["GRD_xr_pl"] = pl2(self.xr_pl)
        g["GMTR_p"] = to2(self.P)
        g["GMTR_p_pl"] = pl2(self.P_pl)
        g["GMTR_t"] = to2(self.T)
        g["GMTR_t_pl"] = pl2(self.T_pl)
        g["GMTR_a"] = to2(self.A)
        g["GMTR_a_pl"] = pl2(self.A_pl)
        for k in ("div", "grad", "lap", "intp", "diff"):
            g["OPRT_coef_" + k] = to2(self.coef[k])
            g["OPRT_coef_" + k + "_pl"] = pl2(self.coef_pl[k])
        for k, v in self.vmtr.items():
            if k.endswith("_pl"):
                g["VMTR_" + k] = pl3(v)
            else:
                g["VMTR_" + k] = to3(v)
        for k in ("rho_bs", "pre_bs", "tem_bs"):
            g[k] = np.zeros((G, G, K, L))
            g[k + "_pl"] = np.zeros((6, K, LP))
        if trcadv:
            g["integ_type"] = "TRCADV"
            g["sstep"] = np.zeros(0, np.int64)
            g["dts"] = float(dtl)
            g["GRD_LON"] = np.ascontiguousarray(np.moveaxis(self.lon, 0, 2))
            g["GRD_LAT"] = np.ascontiguousarray(np.moveaxis(self.lat, 0, 2))
            g["GRD_LON_pl"] = np.ascontiguousarray(np.moveaxis(self.lon_pl, 0, 1))
            g["GRD_LAT_pl"] = np.ascontiguousarray(np.moveaxis(self.lat_pl, 0, 1))
            g["GRD_Z"] = to3(self.vz[..., 0])
            g["GRD_ZH"] = to3(self.vz[..., 1])
            g["GRD_Z_pl"] = pl3(self.vz_pl[..., 0])
            g["GRD_ZH_pl"] = pl3(self.vz_pl[..., 1])
        # heights of the surface-pressure diagnostic (not uploaded): the
        # lowest full level and the surface, (G, G, L) and pole (6, 2)
        g["sfc_zkmin"] = np.ascontiguousarray(np.moveaxis(self.vz[:, :, :, 1, 0], 0, 2))
        g["sfc_zs"] = np.ascontiguousarray(np.moveaxis(self.zs, 0, 2))
        g["sfc_zkmin_pl"] = np.ascontiguousarray(np.moveaxis(self.vz_pl[:, :, 1, 0], 0, 1))
        g["sfc_zs_pl"] = np.ascontiguousarray(np.moveaxis(np.broadcast_to(self.zs_pl[:, :1], (LP, 6)), 0, 1))
        return {k: np.asarray(v) for k, v in g.items()}

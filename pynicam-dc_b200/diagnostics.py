"""Host-side diagnostics used to state the error of a run against another:
surface pressure (the reference's ``sl_ps``) and per-prognostic relative L2.

``surface_pressure`` restates the history diagnostic of
pynicamdc/nhm/driver/mod_history_vars.py:115-118, ps = pre(kmin) +
rho(kmin) * GRAV * (z(kmin) - z_surface), with pre and rho formed from the
prognostic state as the dynamics' diagnostics do (nhm/dynamics/kernels/diag.py:
rho = RHOG / GSGAM2, T = (RHOGE / RHOG) / cv, p = rho T (qd Rdry + qv Rvap),
the first tracer being water vapour).
"""
from __future__ import annotations

import numpy as np

PROG_NAMES = ("RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE")


def _scalar(x):
    return float(np.asarray(x).reshape(-1)[0])


def surface_pressure(geo: dict, prg: np.ndarray, prg_pl: np.ndarray):
    """(ps regional (G, G, L) with the halo ring set to 0, ps at the two pole
    points (2,)) of a state in the reference layout; ``geo`` needs the
    sfc_zkmin / sfc_zs heights of ``icogrid.Grid.setup``"""
    k = int(_scalar(geo["kmin"]))
    g, rd, rv, cvd = (_scalar(geo[n]) for n in ("GRAV", "Rdry", "Rvap", "CVdry"))
    cvw = _scalar(geo["CVW"])

    def ps_of(rhog, rhoge, rhogq, gs, z0, zs):
        rho = rhog / gs
        q = rhogq / rhog
        qd = 1.0 - q
        tem = (rhoge / rhog) / (q * cvw + qd * cvd)
        pre = rho * tem * (qd * rd + q * rv)
        return pre + rho * g * (z0 - zs)

    s = prg[:, :, k]
    ps = ps_of(s[..., 0], s[..., 5], s[..., 6], geo["VMTR_GSGAM2"][:, :, k], geo["sfc_zkmin"], geo["sfc_zs"])
    ps[0, :] = ps[-1, :] = ps[:, 0] = ps[:, -1] = 0.0
    sp = prg_pl[0, k]
    ps_pl = ps_of(sp[:, 0], sp[:, 5], sp[:, 6], geo["VMTR_GSGAM2_pl"][0, k], geo["sfc_zkmin_pl"][0],
                  geo["sfc_zs_pl"][0])
    return ps, ps_pl


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b||"""
    den = float(np.sqrt(np.sum(b * b)))
    d = float(np.sqrt(np.sum((a - b) ** 2)))
    return d / den if den > 0 else d


def state_errors(geo: dict, test, ref) -> dict:
    """relative L2 of each prognostic (interior cells, levels kmin..kmax,
    tracers as RHOGQn) and of the surface pressure of state ``test`` against
    state ``ref``; both (prg, prg_pl) in the reference layout"""
    kmin, kmax = int(_scalar(geo["kmin"])), int(_scalar(geo["kmax"]))
    a, b = test[0][1:-1, 1:-1, kmin:kmax + 1], ref[0][1:-1, 1:-1, kmin:kmax + 1]
    out = {}
    for v in range(a.shape[-1]):
        name = PROG_NAMES[v] if v < 6 else f"RHOGQ{v - 5}"
        out[name] = rel_l2(a[..., v], b[..., v])
    pa, _ = surface_pressure(geo, *test)
    pb, _ = surface_pressure(geo, *ref)
    out["ps"] = rel_l2(pa[1:-1, 1:-1], pb[1:-1, 1:-1])
    return out

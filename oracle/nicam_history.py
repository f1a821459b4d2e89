"""CPU oracle of the derived history diagnostics: numpy restatement.

TEST INFRASTRUCTURE ONLY.  The checker the device history diagnostics
(``nc_history_vars``) are compared against; imported by ``tests/`` and by
nothing in the product path.

Restates ``Hvar.history_vars`` (pynicamdc/nhm/driver/mod_history_vars.py:30-186)
as ``Dyn.history_vars_step`` (pynicamdc/nhm/dynamics/mod_dynamics.py:737-772)
calls it: the diagnostic state re-derived from the current prognostic
(kernels/diag.py:53-143), then the model-level fields, the pressure-level
slices (``_plev_interp``, mod_history_vars.py:188-209), the column integrals,
the saturation ratios (nhm/share/mod_saturation.py:83-98), the per-layer
potential-temperature deviation and the interval tendencies.  The half-level
w outside kmin+1..kmax (the boundary rows kmin and kmax+1 among them) is
taken from the diagnostic w the last large step left behind, as the
reference takes it from its persistent diagnostic buffer, with the reference's
filter (non-finite or UNDEF-sized values read as zero; before any step the
buffer holds UNDEF, so zero).

Pinned against the reference: ``tests/test_oracle_golden.py`` compares this
module with the outputs of the reference's own ``history_vars_step``
(``tests/golden/make_hist.py``).
"""
from __future__ import annotations

import numpy as np

ML = ('ml_u', 'ml_v', 'ml_w', 'ml_th', 'ml_thv', 'ml_omg', 'ml_pres', 'ml_tem', 'ml_rho', 'ml_hgt', 'ml_mse',
      'ml_rh', 'ml_rha', 'ml_rhi', 'ml_du', 'ml_dv', 'ml_dw', 'ml_dtem', 'ml_dq', 'ml_ucos', 'ml_vcos',
      'ml_th_prime')
SL = ('sl_ps', 'sl_pw', 'sl_lwp', 'sl_iwp') + tuple(f'sl_{f}{lev}' for lev in ('850', '500', '250', '100')
                                                  for f in ('u', 'v', 'w', 't'))
TEND = ('ml_du', 'ml_dv', 'ml_dw', 'ml_dtem', 'ml_dq')


def _plev_interp(pre, fields, plev, kmin):
    below = pre < plev
    below[:, :, :kmin, :] = False
    ku = np.argmax(below, axis=2)
    ku = np.maximum(ku, kmin)
    kl = ku - 1
    ku_e, kl_e = ku[:, :, None, :], kl[:, :, None, :]
    pre_ku = np.take_along_axis(pre, ku_e, axis=2)[:, :, 0, :]
    pre_kl = np.take_along_axis(pre, kl_e, axis=2)[:, :, 0, :]
    denom = np.log(pre_kl) - np.log(pre_ku)
    lp = np.log(plev)
    wght_l = (lp - np.log(pre_ku)) / denom
    wght_u = (np.log(pre_kl) - lp) / denom
    out = []
    for f in fields:
        f_ku = np.take_along_axis(f, ku_e, axis=2)[:, :, 0, :]
        f_kl = np.take_along_axis(f, kl_e, axis=2)[:, :, 0, :]
        out.append(wght_l * f_kl + wght_u * f_ku)
    return out


class History:
    """Stateful like the reference's ``Hvar``: keeps the previous output of the
    tendency fields and its step count."""

    def __init__(self):
        self.tend = {}
        self.tend_nstep = None

    def __call__(self, g, hg, prg, items=None, dt=None, nstep=None, w_prev=None):
        """g: the oracle's ``Geo``; hg: dict with GRD_Z (i,j,k,l), GRD_LAT,
        GRD_zsfc, GMTR_area (i,j,l), GMTR_p_IJ (i,j,l,6: IX,IY,IZ,JX,JY,JZ),
        GRD_dgz (k), the constants LHV, UNDEF, PSAT0, RTEM00, CPovR_liq,
        CPovR_ice, LovR_liq, LovR_ice, SAT_ULIMIT, SAT_LLIMIT and the tracer
        indices I_QV, I_QC, I_QR, I_QI, I_QS, I_QG (-1 when absent); w_prev:
        the diagnostic w (i,j,k,l) of the last step (``dynamics_step(keep=)``)
        or None."""
        kmin, kmax = g.kmin, g.kmax
        GRAV = g.GRAV
        want = None if items is None else set(items)
        W = lambda *n: want is None or any(x in want for x in n)
        sc = lambda k: np.asarray(hg[k]).item()
        # kernels/diag.py:53-143 on the regional prognostic
        P = prg[..., :6]
        q = prg[..., 6:] / P[..., 0][..., None]
        RHOG = P[..., 0]
        rho = RHOG / g.VMTR_GSGAM2
        vx, vy, vz = P[..., 1] / RHOG, P[..., 2] / RHOG, P[..., 3] / RHOG
        ein = P[..., 5] / RHOG
        nw = getattr(g, "nqw", 1)
        qd = 1.0 - np.sum(q[..., 0:nw], axis=4)
        cv = np.sum(q[..., 0:nw] * g.CVW[0:nw], axis=4) + qd * g.CVdry
        tem = ein / cv
        pre = rho * tem * (qd * g.Rdry + q[..., 0] * g.Rvap)
        w = np.zeros_like(tem) if w_prev is None else np.array(w_prev, np.float64, copy=True)
        C2W = g.VMTR_C2Wfact
        w[:, :, kmin + 1:kmax + 1, :] = P[:, :, kmin + 1:kmax + 1, :, 4] / (
            C2W[:, :, kmin + 1:kmax + 1, :, 0] * RHOG[:, :, kmin + 1:kmax + 1, :]
            + C2W[:, :, kmin + 1:kmax + 1, :, 1] * RHOG[:, :, kmin:kmax, :])

        iqv = int(sc("I_QV"))
        ntrc = q.shape[-1]
        qv = q[..., iqv] if ntrc > 0 else None
        need_slices = want is None or bool(want & set(SL[4:]))
        need_paths = W('sl_pw', 'sl_lwp', 'sl_iwp', 'sl_cl', 'sl_cl2', 'sl_cly')
        need_tend = dt is not None and W(*TEND)
        res = {'ml_rho': rho, 'ml_tem': tem, 'ml_pres': pre}
        hgt = np.asarray(hg["GRD_Z"])
        res['ml_hgt'] = hgt
        qv0 = qv if qv is not None else np.zeros_like(tem)
        IJ = np.asarray(hg["GMTR_p_IJ"])
        m = lambda c: IJ[:, :, None, :, c]
        u = v = None
        if W('ml_u', 'ml_v') or need_slices or need_tend:
            u = (vx * m(0) + vy * m(1) + vz * m(2)) * 1.0
            v = (vx * m(3) + vy * m(4) + vz * m(5)) * 1.0
            res['ml_u'], res['ml_v'] = u, v
        wc = None
        if W('ml_w', 'ml_omg') or need_slices or need_tend:
            UNDEF = sc("UNDEF")
            w = np.where(np.isfinite(w) & (np.abs(w) < np.abs(UNDEF) * 0.1), w, 0.0)
            W2C = g.VMTR_W2Cfact
            wc = np.zeros_like(w)
            ks = slice(kmin, kmax + 1)
            wc[:, :, ks, :] = (W2C[:, :, ks, :, 0] * w[:, :, kmin + 1:kmax + 2, :]
                               + W2C[:, :, ks, :, 1] * w[:, :, kmin:kmax + 1, :])
            res['ml_w'] = wc
            if W('ml_omg'):
                res['ml_omg'] = -GRAV * rho * wc
        th = None
        if W('ml_th', 'ml_thv', 'ml_th_prime'):
            ratio = g.PRE00 / pre
            th = tem * np.power(ratio, g.Rdry / g.CPdry)
            res['ml_th'] = th
            res['ml_thv'] = th if qv is None else th * (1.0 + 0.61 * qv)
        if W('ml_ucos', 'ml_vcos'):
            coslat = np.cos(np.asarray(hg["GRD_LAT"]))[:, :, None, :]
            res['ml_ucos'] = (vx * m(0) + vy * m(1) + vz * m(2)) * coslat
            res['ml_vcos'] = (vx * m(3) + vy * m(4) + vz * m(5)) * coslat
        if W('ml_th_prime'):
            gmin, gmax = g.gmin, g.gmax
            area = np.asarray(hg["GMTR_area"])[gmin:gmax + 1, gmin:gmax + 1, :]
            wt = area[:, :, None, :] / g.VMTR_RGAM[gmin:gmax + 1, gmin:gmax + 1, :, :] ** 2
            thsub = th[gmin:gmax + 1, gmin:gmax + 1, :, :]
            a_loc = np.sum(wt, axis=(0, 1, 3))
            t_loc = np.sum(thsub * wt, axis=(0, 1, 3))
            mean = np.array([t_loc[k] / a_loc[k] for k in range(th.shape[2])])
            res['ml_th_prime'] = th - mean[None, None, :, None]
        if need_slices:
            for tag, plev in (('850', 850.0e2), ('500', 500.0e2), ('250', 250.0e2), ('100', 100.0e2)):
                up, vp, wp, tp = _plev_interp(pre, (u, v, wc, tem), np.float64(plev), kmin)
                res['sl_u' + tag], res['sl_v' + tag], res['sl_w' + tag], res['sl_t' + tag] = up, vp, wp, tp
        if W('sl_ps'):
            res['sl_ps'] = pre[:, :, kmin, :] + rho[:, :, kmin, :] * GRAV * (hgt[:, :, kmin, :]
                                                                           - np.asarray(hg["GRD_zsfc"]))
        if W('ml_mse'):
            res['ml_mse'] = tem * g.CPdry + hgt * GRAV + qv0 * sc("LHV")
        if W('ml_rh', 'ml_rha', 'ml_rhi'):
            rh_num = qv0 * rho * g.Rvap * tem * 100.0
            R0, P0 = sc("RTEM00"), sc("PSAT0")
            liq = lambda t: P0 * (t * R0) ** sc("CPovR_liq") * np.exp(sc("LovR_liq") * (R0 - 1.0 / t))
            ice = lambda t: P0 * (t * R0) ** sc("CPovR_ice") * np.exp(sc("LovR_ice") * (R0 - 1.0 / t))
            lo, hi = sc("SAT_LLIMIT"), sc("SAT_ULIMIT")
            if W('ml_rha'):
                alpha = np.clip((tem - lo) / (hi - lo), 0.0, 1.0)
                res['ml_rha'] = rh_num / (liq(tem) * alpha + ice(tem) * (1.0 - alpha))
            if W('ml_rh'):
                res['ml_rh'] = rh_num / liq(tem)
            if W('ml_rhi'):
                res['ml_rhi'] = rh_num / ice(tem)
        if need_paths:
            ks = slice(kmin, kmax + 1)
            wcol = g.VMTR_GSGAM2[:, :, ks, :] * np.asarray(hg["GRD_dgz"])[kmin:kmax + 1][None, None, :, None]
            colint = lambda qx: np.sum(rho[:, :, ks, :] * qx[:, :, ks, :] * wcol, axis=2)

            def sum_tracers(idxs):
                s = np.zeros_like(tem)
                for idx in idxs:
                    if idx is not None and idx >= 0:
                        s = s + q[..., idx]
                return s
            if W('sl_pw'):
                res['sl_pw'] = colint(qv0)
            if W('sl_lwp'):
                res['sl_lwp'] = colint(sum_tracers((int(sc("I_QC")), int(sc("I_QR")))))
            if W('sl_iwp'):
                res['sl_iwp'] = colint(sum_tracers((int(sc("I_QI")), int(sc("I_QS")), int(sc("I_QG")))))
            # the terminator chemistry's column means (mod_history_vars.py:149-156), with
            # hg["NCHEM"] = (NCHEM_STR, NCHEM_END) for AF_TYPE 'DCMIP' with the chemistry
            if "NCHEM" in hg and W('sl_cl', 'sl_cl2', 'sl_cly'):
                ns, ne = (int(x) for x in np.asarray(hg["NCHEM"]))
                rhodz = colint(np.ones_like(tem))
                res['sl_cl'] = colint(q[..., ns]) / rhodz
                res['sl_cl2'] = colint(q[..., ne]) / rhodz
                res['sl_cly'] = colint(q[..., ns] + 2.0 * q[..., ne]) / rhodz
        if need_tend:
            dday = 86400.0 / dt
            prev_n = self.tend_nstep
            dn = (nstep - prev_n) if (prev_n is not None and nstep is not None) else 0
            cur = {'ml_du': (u, dday), 'ml_dv': (v, dday), 'ml_dw': (wc, dday), 'ml_dtem': (tem, dday),
                   'ml_dq': (qv0, dday * 1.0e3)}
            for nm, (c, fac) in cur.items():
                if not W(nm):
                    continue
                old = self.tend.get(nm)
                res[nm] = np.zeros_like(c) if (old is None or dn <= 0) else (old - c) * fac / dn
                self.tend[nm] = c.copy()
            self.tend_nstep = nstep
        if want is not None:
            res = {k: x for k, x in res.items() if k in want}
        return res

"""Halo-exchange plan of the single-device COMM.

The reference exchanges halos with four ordered copy lists on one rank
(share/mod_comm.py:1613-1641): region-to-region ``copy_r2r``, pole-to-region
``copy_p2r``, region-to-pole ``copy_r2p`` and finally the singular-point copies,
each a gather from the state *after* the previous list.  Composing the lists on
the host turns the whole exchange into one gather in which every destination
reads an original interior (or pole) value, so the device kernel is a single
race-free pass.

List rows follow the reference's ``Copy_list_*`` layout: 0 i_from, 1 j_from,
2 l_from, 3 i_to, 4 j_to, 5 l_to (pole entries use i as the pole point g and
l as the pole index).
"""
from __future__ import annotations

import numpy as np


def compose(copy_r2r, copy_p2r, copy_r2p, copy_sgp, gall_1d: int, lall: int, lall_pl: int = 2):
    """Return ``(r_dst, r_src, p_dst, p_src)`` int64 arrays.

    Regional cells are encoded ``(l*G + j)*G + i``; pole points ``g*LP + lp``.
    ``r_src >= 0`` is a regional source, ``r_src < 0`` encodes the pole source
    ``-(1 + g*LP + lp)``.  Raises ``ValueError`` if the composed plan would read
    a cell that the same pass writes.
    """
    G = int(gall_1d)
    LP = int(lall_pl)
    reg = lambda i, j, l: (int(l) * G + int(j)) * G + int(i)
    pole = lambda g, lp: -(1 + int(g) * LP + int(lp))
    # value source of every cell after each phase: dict dst -> src token
    src_of = {}

    def resolve(tok):
        return src_of.get(tok, tok)

    # phase 1: region -> region, all sources read before any write
    upd = {}
    for n in range(copy_r2r.shape[1]):
        i_f, j_f, l_f, i_t, j_t, l_t = (int(x) for x in copy_r2r[:, n])
        upd[("r", reg(i_t, j_t, l_t))] = resolve(("r", reg(i_f, j_f, l_f)))
    src_of.update(upd)
    # phase 2: pole -> region (the pole point value, all levels)
    upd = {}
    for n in range(copy_p2r.shape[1]):
        g_f, _, lp_f, i_t, j_t, l_t = (int(x) for x in copy_p2r[:, n])
        upd[("r", reg(i_t, j_t, l_t))] = resolve(("p", pole(g_f, lp_f)))
    src_of.update(upd)
    # phase 3: region -> pole
    upd = {}
    for n in range(copy_r2p.shape[1]):
        i_f, j_f, l_f, g_t, _, lp_t = (int(x) for x in copy_r2p[:, n])
        upd[("p", pole(g_t, lp_t))] = resolve(("r", reg(i_f, j_f, l_f)))
    src_of.update(upd)
    # phase 4: singular points (read after all previous copies)
    upd = {}
    for n in range(copy_sgp.shape[1]):
        i_f, j_f, l_f, i_t, j_t, l_t = (int(x) for x in copy_sgp[:, n])
        upd[("r", reg(i_t, j_t, l_t))] = resolve(("r", reg(i_f, j_f, l_f)))
    src_of.update(upd)

    dsts = set(src_of)
    for d, s in src_of.items():
        if s in dsts:
            raise ValueError(f"halo plan: source {s} of {d} is itself written by the exchange")
    r_dst, r_src, p_dst, p_src = [], [], [], []
    for (kind, d), (skind, s) in sorted(src_of.items()):
        if kind == "r":
            r_dst.append(d)
            r_src.append(s if skind == "r" else s)   # pole tokens are already negative
        else:
            if skind != "r":
                raise ValueError("halo plan: pole destination fed by a pole source")
            p_dst.append(-d - 1)
            p_src.append(s)
    as64 = lambda a: np.asarray(a, dtype=np.int64)
    return as64(r_dst), as64(r_src), as64(p_dst), as64(p_src)


def apply_numpy(plan, var, var_pl):
    """Apply a composed plan to ``var (i,j,k,l,v)`` / ``var_pl (g,k,l,v)`` in
    place with numpy (host-side check of the plan; the device kernel does the
    same gather)."""
    r_dst, r_src, p_dst, p_src = plan
    G = var.shape[0]
    LP = var_pl.shape[2]
    di, dj, dl = r_dst % G, (r_dst // G) % G, r_dst // (G * G)
    old = var.copy()
    oldp = var_pl.copy()
    m = r_src >= 0
    s = r_src[m]
    var[di[m], dj[m], :, dl[m], :] = old[s % G, (s // G) % G, :, s // (G * G), :]
    ps = -r_src[~m] - 1
    var[di[~m], dj[~m], :, dl[~m], :] = oldp[ps // LP, :, ps % LP, :]
    var_pl[p_dst // LP, :, p_dst % LP, :] = old[p_src % G, (p_src // G) % G, :, p_src // (G * G), :]

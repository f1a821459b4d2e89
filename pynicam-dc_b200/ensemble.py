"""Ensembles of the dynamics step: many members of one grid level in one handle.

Members of the same grid level are stacked along the region axis: M members
of a 40-region grid become one handle of 40 * M regions and 2 * M pole points
(set-up entry ``members``), with every set-up array repeated per member and
the halo plan of one member offset to each member's regions and poles, so
that no exchange crosses members.  Every kernel of the step then covers all
members in one launch and one captured CUDA graph replays the whole
ensemble's step; a member's arithmetic is exactly that of a lone run (the
kernels work per region and per column).

Members on different grid levels (the north star's 48 x gl05 + 12 x gl06) go
into one handle per level; ``Ensemble.step`` replays the levels' graphs one
after the other (the run constants of a handle are device-global, so handles
on one device do not overlap).  Each level takes its own time step, and the
launch shapes of each handle are chosen by ``autotune.tune``.

``perturbed_members`` makes the members of the ensemble configuration: the
balanced-jet state with independent seeded Gaussian temperature perturbations
(standard deviation sigma, horizontally smoothed with a Gaussian of the given
length scale, the same at every level), added at fixed density.
"""
from __future__ import annotations

import numpy as np

from . import autotune, halo
from .runtime import NicamCuda


def _stacked_plan(geo: dict, members: int):
    """the composed halo plan of one member, repeated for each member with
    its region and pole offsets (encoding of halo.compose with LP = 2 * M)"""
    G, L = int(np.asarray(geo["gall_1d"])), int(np.asarray(geo["lall"]))
    r_dst, r_src, p_dst, p_src = halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"], geo["copy_sgp"],
                                              G, L)
    LP1, LPM, span = 2, 2 * members, L * G * G
    out = ([], [], [], [])
    for m in range(members):
        out[0].append(r_dst + m * span)
        pole = r_src < 0
        gp = -r_src[pole] - 1
        src = r_src + m * span
        src[pole] = -(1 + (gp // LP1) * LPM + gp % LP1 + 2 * m)
        out[1].append(src)
        out[2].append((p_dst // LP1) * LPM + p_dst % LP1 + 2 * m)
        out[3].append(p_src + m * span)
    return tuple(np.ascontiguousarray(np.concatenate(a), dtype=np.int64) for a in out)


def stack_setup(geo: dict, members: int) -> dict:
    """the set-up dict of ``members`` copies of one grid, stacked along the
    region axis (and the pole axis)"""
    G, L = int(np.asarray(geo["gall_1d"])), int(np.asarray(geo["lall"]))
    out = {}
    for k, v in geo.items():
        a = np.asarray(v)
        if k.startswith("copy_"):
            continue
        if a.ndim >= 4 and a.shape[0] == G and a.shape[1] == G and a.shape[3] == L:
            a = np.concatenate([a] * members, axis=3)
        elif k.endswith("_pl") and a.ndim >= 3 and a.shape[2] == 2:
            a = np.concatenate([a] * members, axis=2)
        elif k.startswith("sfc_") and k.endswith("_pl"):
            a = np.concatenate([a] * members, axis=1)
        elif k.startswith("sfc_"):
            a = np.concatenate([a] * members, axis=2)
        elif k == "pntmask":
            a = np.concatenate([a] * members, axis=1)
        elif k == "have_sgp":
            a = np.concatenate([a] * members, axis=0)
        out[k] = a
    out["lall"] = np.asarray(L * members)
    out["members"] = np.asarray(members)
    out["halo_plan"] = _stacked_plan(geo, members)
    return out


def stack_states(states):
    """[(prg, prg_pl), ...] -> one state of all members"""
    return (np.ascontiguousarray(np.concatenate([s for s, _ in states], axis=3)),
            np.ascontiguousarray(np.concatenate([p for _, p in states], axis=2)))


def unstack_states(prg, prg_pl, members: int):
    L = prg.shape[3] // members
    return [(prg[:, :, :, m * L:(m + 1) * L], prg_pl[:, :, 2 * m:2 * m + 2]) for m in range(members)]


def smoothing_operator(geo: dict, length: float):
    """sparse matrix of normalised Gaussian weights exp(-d^2 / (2 length^2))
    between the interior cells of the grid (chord distance, cut at 3 length),
    rows summing to one"""
    from scipy.sparse import csr_matrix
    from scipy.spatial import cKDTree
    x = np.asarray(geo["GRD_x"])[1:-1, 1:-1, 0]            # (i, j, l, 3)
    pts = x.reshape(-1, 3)
    tree = cKDTree(pts)
    pairs = tree.query_pairs(3.0 * length, output_type="ndarray")
    n = len(pts)
    rows = np.concatenate([pairs[:, 0], pairs[:, 1], np.arange(n)])
    cols = np.concatenate([pairs[:, 1], pairs[:, 0], np.arange(n)])
    d2 = np.sum((pts[rows] - pts[cols]) ** 2, axis=1)
    w = np.exp(-d2 / (2.0 * length ** 2))
    W = csr_matrix((w, (rows, cols)), shape=(n, n))
    rs = np.asarray(W.sum(axis=1)).ravel()
    return csr_matrix((w / rs[rows], (rows, cols)), shape=(n, n))


def perturbed_members(geo: dict, prg, prg_pl, members: int, seed: int, sigma: float = 0.5,
                      length: float = 500e3):
    """``members`` copies of the state, each with its own seeded temperature
    perturbation: white noise on the interior cells, smoothed by a Gaussian of
    ``length``, scaled to standard deviation ``sigma`` (K), copied to the halo
    cells by the exchange, pole points unperturbed; RHOGE += RHOG * CVdry * T'
    on every level"""
    G, L = int(np.asarray(geo["gall_1d"])), int(np.asarray(geo["lall"]))
    cv = float(np.asarray(geo["CVdry"]))
    W = smoothing_operator(geo, length)
    plan = halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"], geo["copy_sgp"], G, L)
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(members):
        t = W @ rng.standard_normal(W.shape[0])
        t *= sigma / t.std()
        field = np.zeros((G, G, 1, L, 1))
        field[1:-1, 1:-1, 0, :, 0] = t.reshape(G - 2, G - 2, L)
        fpl = np.zeros((6, 1, 2, 1))
        halo.apply_numpy(plan, field, fpl)
        s, sp = prg.copy(), prg_pl.copy()
        s[..., 5] += s[..., 0] * cv * field[..., 0]
        out.append((s, sp))
    return out


class Ensemble:
    """Members of one or several grid levels, each level in one handle.

    ``groups``: [(geo, [(prg, prg_pl), ...]), ...], the members of one grid
    level per entry.  ``tune_cache``: a JSON file for the autotuner (None
    skips tuning)."""

    def __init__(self, groups, precision: str = "mixed", graph: bool = True, tune_cache: str | None = None):
        self.handles = []
        for geo, states in groups:
            m = len(states)
            core = NicamCuda(stack_setup(geo, m), graph=graph, precision=precision)
            s, sp = stack_states(states)
            core.upload(s, sp)
            if tune_cache is not None:
                autotune.tune(core, members=m, cache=tune_cache)
                core.upload(s, sp)
            self.handles.append((core, m))

    @property
    def members(self) -> int:
        return sum(m for _, m in self.handles)

    def step(self, nsteps: int = 1):
        """nsteps large steps of every member (each level with its own dt);
        the members do not interact, so each level's handle replays its
        nsteps graph launches in one go"""
        for core, _ in self.handles:
            core.step(nsteps)

    def sync(self):
        for core, _ in self.handles:
            core.sync()

    def download(self):
        """per level, the list of member states"""
        return [unstack_states(*core.download(), m) for core, m in self.handles]

    def close(self):
        for core, _ in self.handles:
            core.close()

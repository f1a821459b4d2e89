"""Composed halo plan == the reference's ordered copy lists (oracle.comm)."""
import numpy as np

from oracle import nicam_step as O


def test_composed_plan_equals_ordered_copies(pkg, golden):
    geo, _ = golden
    G = O.Geo(geo)
    plan = pkg.halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"], geo["copy_sgp"],
                            int(geo["gall_1d"]), int(geo["lall"]))
    rng = np.random.default_rng(7)
    shp = (int(geo["gall_1d"]),) * 2 + (int(geo["kall"]), int(geo["lall"]), 3)
    a = rng.standard_normal(shp)
    ap = rng.standard_normal((6, int(geo["kall"]), 2, 3))
    b, bp = a.copy(), ap.copy()
    O.comm(G, a, ap)
    pkg.halo.apply_numpy(plan, b, bp)
    assert np.array_equal(a, b) and np.array_equal(ap, bp)


def test_plan_covers_every_halo_cell_once(pkg, golden):
    geo, _ = golden
    Gl, L = int(geo["gall_1d"]), int(geo["lall"])
    r_dst, r_src, p_dst, p_src = pkg.halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"],
                                                  geo["copy_sgp"], Gl, L)
    i, j = r_dst % Gl, (r_dst // Gl) % Gl
    assert len(set(r_dst.tolist())) == len(r_dst) == L * (4 * Gl - 4)
    assert np.all((i == 0) | (j == 0) | (i == Gl - 1) | (j == Gl - 1))
    src = r_src[r_src >= 0]
    si, sj = src % Gl, (src // Gl) % Gl
    assert np.all((si > 0) & (sj > 0) & (si < Gl - 1) & (sj < Gl - 1)), "sources must be interior"
    assert sorted((p_dst % 2).tolist()).count(0) == 5 and len(p_dst) == 10


def test_every_halo_cell_is_written_at_all_levels(pkg):
    """kernels that compute interior cells only rely on the exchange to write
    every halo cell (and the five pole neighbours) at every grid level"""
    import os
    import numpy as np
    z = np.load(os.path.join(os.path.dirname(pkg.__file__), "data", "halo_rl01.npz"))
    for gl in range(3, 9):
        G = 2 ** (gl - 1) + 2
        k = f"gl{gl:02d}_"
        r_dst, r_src, p_dst, p_src = pkg.halo.compose(*(z[k + n].astype(np.int64) for n in ("r2r", "p2r", "r2p", "sgp")),
                                                      G, 40)
        assert len(set(r_dst.tolist())) == len(r_dst) == 40 * (4 * G - 4), gl
        assert sorted(p_dst.tolist()) == sorted(g * 2 + lp for g in range(1, 6) for lp in range(2)), gl

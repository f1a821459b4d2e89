"""Parity at a large grid: gl07 z40 (163,842 cells, 40 regions of 64x64), the
benchmark's workload one level down, built on the device by the same grid
generator and spring relaxation the benchmark uses.  One large step on the
device and one oracle step on the host from the same state must agree bit for
bit (the gl03 and gl05 cases do); the tolerance the north star states, relative
L2 <= 1e-12 per prognostic after one step, is checked first so that a failure
says how far apart they are.  The mass sums of the device and the host agree
to 1e-12 relative.

This exercises what only large grids reach: multi-wave column launches, the
32-bit index arithmetic near its larger sizes, and the device-spring grid.
The oracle step takes a few minutes on one host core.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NAMES = ("RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE", "RHOGQ1")


def _rel_l2(a, b):
    out = {}
    for v, nm in enumerate(NAMES):
        x, y = a[..., v], b[..., v]
        den = np.sqrt(np.sum(y * y))
        out[nm] = float(np.sqrt(np.sum((x - y) ** 2)) / den) if den > 0 else float(np.abs(x - y).max())
    return out


@pytest.fixture(scope="module")
def gl07(pkg):
    import bench
    from oracle import nicam_step as O
    geo, prg, prg_pl, _ = bench.make_case(7, 40, device="cuda")
    core = pkg.NicamCuda(geo, graph=True)
    try:
        core.upload(prg, prg_pl)
        core.step(1)
        out, out_pl = core.download()
        mass = core.mass_sums()
    finally:
        core.close()
    G = O.Geo(geo)
    want, want_pl = O.dynamics_step(G, prg, prg_pl)
    return geo, out, out_pl, want, want_pl, mass


def test_gl07_step_within_tolerance(gl07):
    _, out, out_pl, want, want_pl, _ = gl07
    err, err_pl = _rel_l2(out, want), _rel_l2(out_pl, want_pl)
    assert max(err.values()) <= 1e-12, err
    assert max(err_pl.values()) <= 1e-12, err_pl


def test_gl07_step_bit_exact(gl07):
    _, out, out_pl, want, want_pl, _ = gl07
    assert np.array_equal(out, want), "regional state differs from the oracle"
    assert np.array_equal(out_pl, want_pl), "pole state differs from the oracle"


def test_gl07_mass_matches_host(gl07):
    geo, out, out_pl, _, _, mass = gl07
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    ks = slice(kmin, kmax + 1)
    w = geo["VMTR_VOLUME"][1:-1, 1:-1, ks] / geo["VMTR_GSGAM2"][1:-1, 1:-1, ks]
    w_pl = geo["VMTR_VOLUME_pl"][0, ks] / geo["VMTR_GSGAM2_pl"][0, ks]
    for n, v in enumerate((0, 6)):
        host = np.sum(out[1:-1, 1:-1, ks, :, v] * w) + np.sum(out_pl[0, ks, :, v] * w_pl)
        assert abs(mass[n] - host) <= 1e-12 * abs(host), (n, mass[n], host)

"""One simulated day on the device against the oracle's digest of the same day.

The case is gl05 z40, dtl 600 s, 144 large steps (one day) of the JW wave with
a sharp tracer, rebuilt here with the package's grid generator exactly as
``tests/golden/make_day.py`` built it when it ran the oracle over the day.  The
fixture holds the oracle's state hashes, a strided sample of the regional
state and the full pole state after steps 1, 36 (6 h) and 144, and the oracle's
mass sums after every step.

Tolerances (relative L2 over the sample, per prognostic): 1e-12 after one step,
1e-8 after one day; dry-air and tracer mass drift over the day: 1e-13 relative.
The device path is also expected to reproduce the oracle bit for bit.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = ("RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE", "RHOGQ1")


@pytest.fixture(scope="module")
def day(pkg):
    import make_day as M
    from oracle import nicam_step as O
    d = np.load(os.path.join(GOLDEN, "gl05_z40_day.npz"))
    geo, s, s_pl = M.build_case()
    assert M.geo_sha(geo) == str(d["geo_sha"]), "the regenerated gl05 setup differs from the digest's"
    O.comm(O.Geo(geo), s, s_pl)
    assert M.state_sha(s, s_pl) == str(d["init_sha"]), "the regenerated initial state differs from the digest's"
    core = pkg.NicamCuda(geo, graph=True)
    try:
        core.upload(s, s_pl)
        mass = [core.mass_sums()]
        states = {}
        for n in range(1, M.NSTEPS + 1):
            core.step(1)
            mass.append(core.mass_sums())
            if n in M.RECORD:
                states[n] = core.download()
    finally:
        core.close()
    return M, d, states, np.array(mass)


def _rel_l2(a, b):
    out = {}
    for v, nm in enumerate(NAMES):
        x, y = a[..., v], b[..., v]
        den = np.sqrt(np.sum(x * x))
        out[nm] = float(np.sqrt(np.sum((x - y) ** 2)) / den) if den > 0 else float(np.abs(x - y).max())
    return out


@pytest.mark.parametrize("step,tol", [(1, 1e-12), (36, 1e-8), (144, 1e-8)])
def test_day_within_tolerance(day, step, tol):
    M, d, states, _ = day
    s, s_pl = states[step]
    err = _rel_l2(M.sample(s), d[f"s{step}_sample"])
    err_pl = _rel_l2(s_pl, d[f"s{step}_pl"])
    assert max(err.values()) <= tol, (step, err)
    assert max(err_pl.values()) <= tol, (step, err_pl)


def test_day_bit_exact(day):
    M, d, states, _ = day
    for n in M.RECORD:
        assert M.state_sha(*states[n]) == str(d[f"s{n}_sha"]), f"state after step {n}"


def test_day_mass_conserved(day):
    _, d, _, mass = day
    drift = np.abs(mass - mass[0]) / np.abs(mass[0])
    assert drift.max() <= 1e-13, drift.max(axis=0)
    # compensated device sums against the oracle's host sums of the same states
    assert np.allclose(mass, d["mass"], rtol=1e-12, atol=0.0)

"""Host logic of the ensemble form and the autotuner (no GPU).

* the stacked halo plan of M members applied to the stacked state equals the
  single-member plan applied to each member (no exchange crosses members);
* every set-up array is repeated per member along its region or pole axis;
* the members' temperature perturbations have the stated standard deviation,
  are smooth on the stated length scale and independent between members;
* the autotuner keeps the fastest block size of each kernel and reuses its
  cache (a stand-in handle with made-up kernel times).
"""
import importlib
import json

import numpy as np
import pytest


@pytest.fixture(scope="module")
def case3():
    ig = importlib.import_module("pynicam-dc_b200.icogrid")
    g = ig.Grid(3, vlayer=6, ztop=30000.0)
    geo = g.setup(dtl=1200.0, gamma=7.68e17, nq=1)
    s, sp = g.jw_state(nq=1)
    return geo, s, sp


def test_stacked_plan_is_per_member(case3):
    ens = importlib.import_module("pynicam-dc_b200.ensemble")
    halo = importlib.import_module("pynicam-dc_b200.halo")
    geo, s, sp = case3
    M = 3
    G, L = int(geo["gall_1d"]), int(geo["lall"])
    rng = np.random.default_rng(0)
    states = [(rng.standard_normal(s.shape), rng.standard_normal(sp.shape)) for _ in range(M)]
    big, big_pl = ens.stack_states(states)
    halo.apply_numpy(ens.stack_setup(geo, M)["halo_plan"], big, big_pl)
    plan1 = halo.compose(geo["copy_r2r"], geo["copy_p2r"], geo["copy_r2p"], geo["copy_sgp"], G, L)
    for (a, ap), (b, bp) in zip(ens.unstack_states(big, big_pl, M), states):
        b, bp = b.copy(), bp.copy()
        halo.apply_numpy(plan1, b, bp)
        assert np.array_equal(a, b) and np.array_equal(ap, bp)


def test_stacked_setup_repeats_each_member(case3):
    ens = importlib.import_module("pynicam-dc_b200.ensemble")
    geo, _, _ = case3
    st = ens.stack_setup(geo, 4)
    L = int(geo["lall"])
    assert int(st["lall"]) == 4 * L and int(st["members"]) == 4
    for k in ("VMTR_GSGAM2", "OPRT_coef_div", "GRD_x"):
        a = np.asarray(st[k])
        assert a.shape[3] == 4 * L and np.array_equal(a[:, :, :, 3 * L:], geo[k])
    for k in ("VMTR_GSGAM2_pl", "OPRT_coef_div_pl"):
        a = np.asarray(st[k])
        assert a.shape[2] == 8 and np.array_equal(a[:, :, 6:8], geo[k])
    assert st["pntmask"].shape == (1, 4 * L, 2) and st["have_sgp"].shape == (4 * L,)


def test_member_perturbations(case3):
    ens = importlib.import_module("pynicam-dc_b200.ensemble")
    geo, s, sp = case3
    cv = float(geo["CVdry"])
    mem = ens.perturbed_members(geo, s, sp, 3, seed=7, sigma=0.5, length=2000e3)
    t = [(m[0][..., 5] - s[..., 5]) / (s[..., 0] * cv) for m in mem]
    for x in t:
        inner = x[1:-1, 1:-1, 3]
        assert abs(inner.std() - 0.5) < 1e-12                       # stated standard deviation
        assert np.allclose(x[1:-1, 1:-1, 1], x[1:-1, 1:-1, 4])      # the same at every level
        assert np.array_equal(mem[0][1], sp)                         # poles unperturbed
    assert abs(np.corrcoef(t[0][1:-1, 1:-1, 3].ravel(), t[1][1:-1, 1:-1, 3].ravel())[0, 1]) < 0.5
    # smooth: neighbouring cells are strongly correlated at a 2000 km scale on a ~1000 km grid
    x = t[0][1:-1, 1:-1, 3]
    assert np.corrcoef(x[:-1].ravel(), x[1:].ravel())[0, 1] > 0.5


class FakeCore:
    """records block sizes; a kernel's time is a made-up function of its size"""
    shape = (6, 6, 12, 40, 7)
    precision = "mixed"

    def __init__(self):
        self.blk = {}
        self.prof = False

    def set_block(self, k, t):
        self.blk[k] = t

    def profile(self, on):
        self.prof = on

    def step(self, n):
        pass

    def kernel_stats(self):
        best = {"diag": 64, "vi_solve": 128, "gtend": 256}
        return {k: (1.0 + abs(np.log2(self.blk.get(k, 128) / best.get(k, 128))), 1) for k in self.blk}


def test_autotune_picks_fastest_and_caches(tmp_path):
    at = importlib.import_module("pynicam-dc_b200.autotune")
    core = FakeCore()
    cache = str(tmp_path / "tune.json")
    choice = at.tune(core, members=2, cache=cache)
    assert choice["diag"] == 64 and choice["vi_solve"] == 128 and choice["gtend"] == 256
    assert all(choice[k] <= at.TUNABLE[k] for k in choice)
    with open(cache) as f:
        stored = json.load(f)
    assert list(stored.values())[0] == choice
    core2 = FakeCore()
    assert at.tune(core2, members=2, cache=cache) == choice and core2.blk == choice

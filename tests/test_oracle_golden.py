"""The CPU oracle against the golden states written by the reference itself
(tests/golden/make_golden.py): bit-for-bit on two consecutive large steps."""
import numpy as np

from oracle import nicam_step as O


def test_oracle_matches_reference_two_steps(golden):
    geo, st = golden
    G = O.Geo(geo)
    for s in (0, 1):
        out, out_pl = O.dynamics_step(G, st[f"state{s}"], st[f"state{s}_pl"])
        assert np.array_equal(out, st[f"state{s + 1}"]), f"step {s + 1} regional"
        assert np.array_equal(out_pl, st[f"state{s + 1}_pl"]), f"step {s + 1} pole"


def test_golden_tracer_is_nontrivial(golden):
    _, st = golden
    q = st["state0"][..., 6]
    assert q.max() > 1e-3 and (q > 0).mean() > 0.5

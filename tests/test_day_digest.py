"""The one-day gl05 digest (written by tests/golden/make_day.py) as CPU checks.

* The oracle conserves dry-air and tracer mass over the simulated day to 1e-13
  relative (volume-weighted sums of every step, poles included).
* The record of the oracle run against the reference's own numpy model over
  the same day (``gl05_z40_day_pin.json``, ``make_day.py --mode compare``)
  shows bit-for-bit equal states after 1, 36 and 144 steps.
"""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_oracle_day_conserves_mass():
    d = np.load(os.path.join(GOLDEN, "gl05_z40_day.npz"))
    m = d["mass"]
    assert m.shape[0] == 145
    drift = np.abs(m - m[0]) / np.abs(m[0])
    assert drift.max() <= 1e-13, drift.max(axis=0)


def test_oracle_day_matches_reference_record():
    with open(os.path.join(GOLDEN, "gl05_z40_day_pin.json")) as f:
        pin = json.load(f)
    assert set(pin["steps"]) == {"1", "36", "144"}
    for step, rec in pin["steps"].items():
        assert rec["bit_exact"], step
        assert max(v for k, v in rec.items() if k != "bit_exact") == 0.0, step

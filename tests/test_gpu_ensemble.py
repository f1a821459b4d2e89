"""Ensembles on the device (ensemble.py).

* Stacking is exact: three perturbed gl04 members in one handle (one launch
  per kernel for all of them, one graph) give, after two steps, each member's
  lone-run state bit for bit, in both forms.
* The north star's ensemble configuration: 48 members at grid level 5
  (dtl 600 s) and 12 at grid level 6 (dtl 300 s), 40 layers, the balanced jet
  with independent seeded temperature perturbations (sigma 0.5 K, smoothed to
  500 km), one handle per grid level with its launch shapes from the
  autotuner.  Reported: members-steps/s and cell-level-steps/s of the mixed
  and float64 ensembles against running every member alone (one handle, one
  member at a time); the ensemble-mean surface-pressure error of the mixed
  form against float64.  The batched ensemble must beat the one-by-one runs,
  and the ensemble-mean surface pressure must agree to 1e-4.
"""
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIGMA, LENGTH = 0.5, 500e3


def _case(glevel):
    import importlib
    ig = importlib.import_module("pynicam-dc_b200.icogrid")
    dtl = {4: 900.0, 5: 600.0, 6: 300.0}[glevel]
    gamma = {4: 9.6e16, 5: 1.2e16, 6: 1.5e15}[glevel]
    g = ig.Grid(glevel, vlayer=40, ztop=30000.0, device="cuda")
    geo = g.setup(dtl=dtl, gamma=gamma, nq=1)
    s, sp = g.jw_state(nq=1)
    return geo, s, sp


@pytest.fixture(scope="module")
def ens():
    import importlib
    return importlib.import_module("pynicam-dc_b200.ensemble")


@pytest.mark.parametrize("prec", ["float64", "mixed"])
def test_stacked_members_equal_lone_runs(pkg, ens, prec):
    geo, s, sp = _case(4)
    members = ens.perturbed_members(geo, s, sp, 3, seed=1, sigma=SIGMA, length=1000e3)
    e = ens.Ensemble([(geo, members)], precision=prec)
    try:
        e.step(2)
        got = e.download()[0]
    finally:
        e.close()
    for (a, ap), (m, mp) in zip(got, members):
        c = pkg.NicamCuda(geo, graph=True, precision=prec)
        try:
            c.upload(m, mp)
            c.step(2)
            b, bp = c.download()
        finally:
            c.close()
        assert np.array_equal(a, b) and np.array_equal(ap, bp)


def _timed(fn, n):
    import torch
    torch.cuda.synchronize()
    t = time.perf_counter()
    fn(n)
    torch.cuda.synchronize()
    return (time.perf_counter() - t) / n


def test_ensemble_configuration(pkg, ens, tmp_path):
    dg = __import__("importlib").import_module("pynicam-dc_b200.diagnostics")
    groups = []
    for glevel, nmem, seed in ((5, 48, 105), (6, 12, 106)):
        geo, s, sp = _case(glevel)
        groups.append((geo, ens.perturbed_members(geo, s, sp, nmem, seed=seed, sigma=SIGMA, length=LENGTH)))
    cl = [(int(geo["lall"]) * (int(geo["gall_1d"]) - 2) ** 2 + 2) * (int(geo["kall"]) - 2) for geo, _ in groups]
    nsteps, report = 6, {}
    mean_ps = {}
    for prec in ("mixed", "float64"):
        e = ens.Ensemble(groups, precision=prec, tune_cache=str(tmp_path / "tune.json"))
        try:
            e.step(1)                                  # graph capture
            sec = _timed(e.step, nsteps)               # one ensemble step: every member one large step
            e.step(0)
            out = e.download()
        finally:
            e.close()
        mean_ps[prec] = [np.mean([dg.surface_pressure(geo, *m)[0] for m in mem], axis=0)
                         for (geo, _), mem in zip(groups, out)]
        lone = 0.0
        for geo, members in groups:
            c = pkg.NicamCuda(geo, graph=True, precision=prec)
            try:
                c.upload(*members[0])
                c.step(1)
                lone += len(members) * _timed(c.step, nsteps)     # every member alone, one after the other
            finally:
                c.close()
        report[prec] = {"ensemble_s_per_step": sec, "one_by_one_s_per_step": lone,
                        "members_steps_per_s": 60 / sec, "cell_level_steps_per_s": sum(n * x for n, x in
                                                                                          zip((48, 12), cl)) / sec,
                        "speedup_vs_one_by_one": lone / sec}
    err = [dg.rel_l2(a[1:-1, 1:-1], b[1:-1, 1:-1]) for a, b in zip(mean_ps["mixed"], mean_ps["float64"])]
    report["ensemble_mean_ps_rel_l2_mixed_vs_f64"] = {"gl05": err[0], "gl06": err[1], "steps": nsteps + 1}
    print("ensemble configuration:", report)
    out_dir = os.environ.get("NC_REPORT_DIR")
    if out_dir:
        import json
        with open(os.path.join(out_dir, "ensemble_report.json"), "w") as f:
            json.dump(report, f, indent=1)
    for prec in ("mixed", "float64"):
        assert report[prec]["speedup_vs_one_by_one"] > 1.0, report
    assert max(err) <= 1e-4, err

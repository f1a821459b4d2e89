"""The mixed-precision form against the float64 form.

Mixed: float32 work fields, metrics and stencil / advection / hyperdiffusion /
tracer arithmetic; float64 tridiagonal elimination and its matrix, pressure
and density deviations, mass sums.  The float64 form equals the reference bit
for bit (test_gpu_parity, test_gpu_day), so its states stand for the
reference's here.  The errors below are relative L2 norms over interior cells
and levels kmin..kmax, per prognostic, and of the surface pressure
(``diagnostics.surface_pressure``, the reference's sl_ps); the bounds are the
north star's (surface pressure 1e-4 after one day) and, for the others, a
margin over the measured values written beside them.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# gl03 z10 golden case (dtl 1200 s, a sharp tracer): one and two steps; measured on
# B200 after step 1 (2): RHOG 5.0e-8 (6.1e-8), RHOGVX 1.6e-7 (2.6e-7), RHOGVZ 3.2e-6
# (2.7e-6), RHOGW 1.7e-5 (1.3e-5), RHOGE 4.5e-8 (4.5e-8), RHOGQ1 7.1e-8 (8.6e-8)
GL03_TOL = {"RHOG": 1e-6, "RHOGVX": 1e-5, "RHOGVY": 1e-5, "RHOGVZ": 1e-4, "RHOGW": 1e-3, "RHOGE": 1e-6,
            "RHOGQ1": 1e-6}
# gl05 z40 one day (144 steps of 600 s); measured on B200 after 1 / 36 / 144 steps:
# ps 4.4e-8 / 6.2e-8 / 8.8e-8, RHOG 4.7e-8 / 1.4e-7 / 2.1e-7, RHOGE 4.0e-8 / 5.9e-8 / 8.7e-8,
# RHOGVX 5.3e-7 / 6.1e-6 / 1.1e-5, RHOGVZ 1.7e-4 / 4.1e-4 / 6.3e-4, RHOGW 3.8e-5 / 6.8e-4 /
# 7.3e-4, RHOGQ1 9.7e-8 / 3.7e-6 / 1.9e-5; mass drift over the day 5.5e-11 (air), 2.7e-9
# (tracer)
DAY_PS_TOL = 1e-4


def _errs(dg, geo, a, b):
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    x, y = a[1:-1, 1:-1, kmin:kmax + 1], b[1:-1, 1:-1, kmin:kmax + 1]
    return {nm: dg.rel_l2(x[..., v], y[..., v]) for v, nm in enumerate(dg.PROG_NAMES + ("RHOGQ1",))}


@pytest.fixture(scope="module")
def dg():
    import importlib
    return importlib.import_module("pynicam-dc_b200.diagnostics")


def test_mixed_gl03_two_steps_near_reference(pkg, golden, dg):
    geo, st = golden
    c = pkg.NicamCuda(geo, graph=True, precision="mixed")
    try:
        c.upload(st["state0"], st["state0_pl"])
        for n in (1, 2):
            c.step(1)
            s, sp = c.download()
            e = _errs(dg, geo, s, st[f"state{n}"])
            for nm, tol in GL03_TOL.items():
                assert e[nm] <= tol, (n, nm, e)
            assert np.all(np.isfinite(sp))
    finally:
        c.close()


def test_mixed_graph_equals_eager(pkg, golden):
    geo, st = golden
    out = []
    for graph in (True, False):
        c = pkg.NicamCuda(geo, graph=graph, precision="mixed")
        try:
            c.upload(st["state0"], st["state0_pl"])
            c.step(2)
            out.append(c.download())
        finally:
            c.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_mixed_refuses_float64_only_calls(pkg, golden):
    geo, st = golden
    c = pkg.NicamCuda(geo, graph=False, precision="mixed")
    try:
        c.upload(st["state0"], st["state0_pl"])
        with pytest.raises(pkg.NicamError, match="mixed-precision"):
            c.forcing_step()
        with pytest.raises(pkg.NicamError, match="mixed-precision"):
            c.restart_pack(0, np.empty(c.shape[0] * c.shape[1] * c.shape[2] * c.shape[3]))
        c.check_finite()
        reg, pl = c.field("RHOGVX")          # float32 fields come back as float64
        assert reg.shape == c.shape[:4] and np.isfinite(reg).all()
    finally:
        c.close()


@pytest.fixture(scope="module")
def day(pkg):
    """gl05 z40 one day in both forms from the same state: states after 1,
    36 (6 h) and 144 (1 day) steps, and the mixed form's mass sums"""
    import make_day as M
    from oracle import nicam_step as O
    geo, s, s_pl = M.build_case()
    O.comm(O.Geo(geo), s, s_pl)
    states, mass = {}, {}
    for prec in ("float64", "mixed"):
        c = pkg.NicamCuda(geo, graph=True, precision=prec)
        try:
            c.upload(s, s_pl)
            m = [c.mass_sums()]
            for n in range(1, M.NSTEPS + 1):
                c.step(1)
                if n in M.RECORD:
                    states[(prec, n)] = c.download()
            m.append(c.mass_sums())
            mass[prec] = np.array(m)
        finally:
            c.close()
    return geo, states, mass


@pytest.mark.parametrize("step", [1, 36, 144])
def test_mixed_day_error_vs_float64(day, dg, step):
    geo, states, _ = day
    e = dg.state_errors(geo, states[("mixed", step)], states[("float64", step)])
    print("mixed vs float64 after", step, "steps:", e)
    assert e["ps"] <= DAY_PS_TOL, e
    for nm in ("RHOG", "RHOGE"):
        assert e[nm] <= 1e-5, e
    for nm in ("RHOGVX", "RHOGVY", "RHOGQ1"):
        assert e[nm] <= 1e-3, e
    for nm in ("RHOGVZ", "RHOGW"):
        assert e[nm] <= 1e-2, e


def test_mixed_day_mass(day):
    _, _, mass = day
    m = mass["mixed"]
    drift = np.abs(m[1] - m[0]) / np.abs(m[0])
    print("mixed mass drift over the day:", drift)
    assert drift[0] <= 1e-8 and drift[1] <= 1e-7, drift

"""CUDA step vs the reference's own golden states and vs the oracle.

The golden fixture is two large steps of the reference (gl03 z10, JW wave
with a sharp injected tracer).  FP64 bit-for-bit equality is required: the
kernels keep the reference's association order and are built without FMA
contraction.  Graph replay must equal eager launches exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core(pkg, golden):
    geo, _ = golden
    c = pkg.NicamCuda(geo, graph=False)
    yield c
    c.close()


def _steps(core, st, n):
    core.upload(st["state0"], st["state0_pl"])
    outs = []
    for _ in range(n):
        core.step(1)
        outs.append(core.download())
    return outs


def test_two_steps_bit_exact_vs_reference(core, golden):
    _, st = golden
    for s, (out, out_pl) in enumerate(_steps(core, st, 2), start=1):
        assert np.array_equal(out, st[f"state{s}"]), f"regional state after step {s}"
        assert np.array_equal(out_pl, st[f"state{s}_pl"]), f"pole state after step {s}"


def test_warm_rain_two_steps_bit_exact_vs_reference(pkg, golden_warm):
    """RAIN_TYPE WARM: the thermodynamics over three water tracers, bit for
    bit with the reference's two steps; the mixed form stays within 2e-3 of
    them (relative L2 per prognostic; the float32 arithmetic moves the small
    vertical momentum most, as in the dry case)"""
    geo, st = golden_warm
    for prec in ("float64", "mixed"):
        c = pkg.NicamCuda(geo, graph=True, precision=prec)
        try:
            outs = _steps(c, st, 2)
        finally:
            c.close()
        for s, (out, out_pl) in enumerate(outs, start=1):
            if prec == "float64":
                assert np.array_equal(out, st[f"state{s}"]) and np.array_equal(out_pl, st[f"state{s}_pl"]), s
            else:
                for v in range(out.shape[-1]):
                    ref = st[f"state{s}"][..., v]
                    den = np.sqrt(np.sum(ref * ref))
                    assert np.sqrt(np.sum((out[..., v] - ref) ** 2)) <= 2e-3 * den, (s, v)


@pytest.mark.parametrize("case", ["golden_nlhdiff", "golden_rayleigh"])
def test_numfilter_options_two_steps_bit_exact_vs_reference(pkg, case, request):
    """the NONLINEAR1 hyperdiffusion (per-cell Kh from the first pass's
    temperature Laplacian, its half-level average for w) and the Rayleigh
    sponge: bit for bit with the reference's two steps in float64, graph
    replayed; the mixed form within 2e-3 (relative L2 per prognostic)"""
    geo, st = request.getfixturevalue(case)
    for prec in ("float64", "mixed"):
        c = pkg.NicamCuda(geo, graph=True, precision=prec)
        try:
            outs = _steps(c, st, 2)
        finally:
            c.close()
        for s, (out, out_pl) in enumerate(outs, start=1):
            if prec == "float64":
                assert np.array_equal(out, st[f"state{s}"]) and np.array_equal(out_pl, st[f"state{s}_pl"]), s
            else:
                for v in range(out.shape[-1]):
                    ref = st[f"state{s}"][..., v]
                    den = np.sqrt(np.sum(ref * ref))
                    assert np.sqrt(np.sum((out[..., v] - ref) ** 2)) <= 2e-3 * den, (s, v)


def test_graph_replay_equals_eager(pkg, golden):
    geo, st = golden
    c = pkg.NicamCuda(geo, graph=True)
    try:
        c.upload(st["state0"], st["state0_pl"])
        c.step(2)
        out, out_pl = c.download()
        assert np.array_equal(out, st["state2"]) and np.array_equal(out_pl, st["state2_pl"])
        assert c.kernel_launches() > 0
    finally:
        c.close()


def test_step_from_perturbed_state_vs_oracle(core, golden):
    """a state the fixture never saw: oracle and device from the same input"""
    from oracle import nicam_step as O
    geo, st = golden
    rng = np.random.default_rng(11)
    s, sp = st["state1"].copy(), st["state1_pl"].copy()
    s[..., 1:4] *= 1.0 + 1e-3 * rng.standard_normal(s[..., 1:4].shape)
    s[..., 6] = np.abs(s[..., 6] * (1.0 + 0.1 * rng.standard_normal(s[..., 6].shape)))
    O.comm(O.Geo(geo), s, sp)
    want, want_pl = O.dynamics_step(O.Geo(geo), s, sp)
    core.upload(s, sp)
    core.step(1)
    got, got_pl = core.download()
    assert np.array_equal(got, want) and np.array_equal(got_pl, want_pl)


def test_mass_sums_match_host(core, golden):
    geo, st = golden
    core.upload(st["state2"], st["state2_pl"])
    m = core.mass_sums()
    s, sp = st["state2"], st["state2_pl"]
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    ks = slice(kmin, kmax + 1)
    rho = s[1:-1, 1:-1, ks, :, 0] / geo["VMTR_GSGAM2"][1:-1, 1:-1, ks]
    vol = geo["VMTR_VOLUME"][1:-1, 1:-1, ks]
    rho_p = sp[0, ks, :, 0] / geo["VMTR_GSGAM2_pl"][0, ks]
    vol_p = geo["VMTR_VOLUME_pl"][0, ks]
    want = np.sum(rho * vol) + np.sum(rho_p * vol_p)
    assert abs(m[0] - want) <= 1e-12 * abs(want)
    q = s[1:-1, 1:-1, ks, :, 6] / s[1:-1, 1:-1, ks, :, 0]
    qp = sp[0, ks, :, 6] / sp[0, ks, :, 0]
    wq = np.sum(rho * q * vol) + np.sum(rho_p * qp * vol_p)
    assert abs(m[1] - wq) <= 1e-12 * abs(wq)


def test_non_unit_gamma_factors_vs_oracle(pkg, golden):
    """a deep-atmosphere-like setup (gamma factors not all 1) takes the loaded
    path of the gamma factors; device and oracle agree bit for bit"""
    from oracle import nicam_step as O
    geo, st = golden
    g = dict(geo)
    rng = np.random.default_rng(5)
    for k in ("VMTR_RGAM", "VMTR_RGAMH", "VMTR_GAM2H"):
        g[k] = geo[k] * (1.0 + 1e-6 * rng.random(geo[k].shape))
    s, sp = st["state0"], st["state0_pl"]
    want, want_pl = O.dynamics_step(O.Geo(g), s, sp)
    c = pkg.NicamCuda(g, graph=False)
    try:
        c.upload(s, sp)
        c.step(1)
        out, out_pl = c.download()
    finally:
        c.close()
    assert np.array_equal(out, want) and np.array_equal(out_pl, want_pl)

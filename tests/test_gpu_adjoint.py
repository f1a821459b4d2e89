"""Tangent-linear and adjoint operators (adjoint.py, nc_vsolve / nc_vadv_lin /
nc_laplacian / nc_divergence / nc_gradient / nc_diffusion) on the device,
float64.

The operators' inputs come from a real step: the balanced-jet case at grid
level 4 with 40 layers is stepped once and the handle's implicit matrix
(Mc, Mu, Ml), tracer vertical mass flux and the tracer step's density
tendency are read back (non-finite values set to zero,
unused columns given an identity matrix); the density is the prognostic
density at the start of the step.  The tracer mass is a smooth
positive field with seeded noise (no ties for the limiter's min / max).

* forward parity: the vertical advection step equals the oracle's
  (mod_src_tracer.py:389-533 with the limiter of 1909-2074) bit for bit, the
  exchange + Laplacian / divergence / gradient equal the oracle's comm +
  laplacian / divergence / gradient bit for bit, and
  the tridiagonal solve equals a banded solve to 1e-12;
* dot-product tests <TL x, y> = <x, AD y> to 1e-12 (relative to the
  magnitudes of the products) for every operator, regional and pole;
* the exchange + Kh-weighted diffusion equals the oracle's comm + diffusion
  bit for bit, and the hyperdiffusion tendency composed from the Laplacian
  and diffusion operators (adjoint.hyperdiffusion, at the case's state) equals
  the oracle's hdiffusion to 1e-12 and passes the dot-product test;
* the HEVI vertical implicit step (adjoint.hevi_matrix / hevi_solve around
  the hand-written solve) equals the oracle's rhow_matrix / rhow_solver bit
  for bit and passes the dot-product test in all nine field arguments;
* central finite differences along seeded random directions against the
  tangent-linear, to 1e-6 relative (relative steps of 1e-9 / 1e-8; the
  errors at 1e-6 are reported: the limiter is piecewise linear);
* a multi-step chain through torch.autograd (vertical advection with the
  limiter, then diffusion by the Laplacian): the gradient of a box loss with
  per-step checkpointing equals the one without, and matches central finite
  differences along 16 seeded directions to 1e-6.
* the chain at grid level 6 with 40 layers, 36 steps: the time of the
  gradient against the forward run and the peak device memory with and
  without checkpointing are reported (NC_REPORT_DIR/adjoint_report.json).

The whole tracer advection step (nc_trc_step_lin: vertical step, horizontal
step with the horizontal Thuburn limiter, vertical step with the clamp, the
closing exchange), on the offline-advection case (DCMIP 2012 test 1-1 winds,
60 even layers to 12 km, its four tracers):

* its forward equals the handle's own step, bit for bit, for every tracer;
* the dot-product test, 1e-12, at the test's tracers and at a tie-free field;
* central differences (relative step 1e-9) against the tangent-linear;
* the gradient of a box loss over several steps (TracerTransport, all four
  tracers) checkpointed every step equals the one checkpointed every third
  step and matches central differences along 16 seeded directions to 1e-6
  and the run's tangent-linear to 1e-10 (grid level 4, 6 steps);
* grid level 6, 36 steps of 300 s: the run's tangent-linear (each step's
  tangent-linear in turn) against the adjoint along 16 seeded directions to
  1e-10; central differences at relative steps 1e-6, 1e-8 and 1e-10 are
  reported (over 36 steps the limiters switch branches inside a small step
  in enough cells that the differences do not reach 1e-6); the gradient's
  time against the forward run's and the peak device memory with a
  checkpoint every step and every sixth step are reported.

jax.vjp of the reference's jax backend is not available (jax is not
installed in this environment), so the reference-gradient comparison is not
made here.
"""
import importlib
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    return (importlib.import_module("pynicam-dc_b200.icogrid"), importlib.import_module("pynicam-dc_b200.adjoint"))


def _case(pkg, glevel, vlayer=40):
    import torch
    ig, adj = _mods()
    dtl = {4: 900.0, 5: 600.0, 6: 300.0}[glevel]
    gamma = {4: 9.6e16, 5: 1.2e16, 6: 1.5e15}[glevel]
    g = ig.Grid(glevel, vlayer=vlayer, ztop=30000.0, device="cuda")
    geo = g.setup(dtl=dtl, gamma=gamma, nq=1)
    s, sp = g.jw_state(nq=1)
    core = pkg.NicamCuda(geo, graph=False)
    core.upload(s, sp)
    core.step(1)
    f = {}
    for name in ("Mc", "Mu", "Ml", "flx_v", "frhog"):
        r, p = core.field(name)
        r, p = np.nan_to_num(r), np.nan_to_num(np.ascontiguousarray(p))
        f[name] = adj.to_device_layout(r)
        f[name + "_pl"] = torch.as_tensor(p).cuda()
    # columns the step leaves without a matrix (unused halo corners): identity
    for sfx in ("", "_pl"):
        bad = f["Mc" + sfx] == 0
        f["Mc" + sfx][bad] = 1.0
        f["Mu" + sfx][bad] = 0.0
        f["Ml" + sfx][bad] = 0.0
    # the density of the first vertical step: the prognostic density at the step's start
    f["den"] = adj.to_device_layout(s[..., 0])
    f["den_pl"] = torch.as_tensor(np.ascontiguousarray(sp[..., 0])).cuda()
    for sfx in ("", "_pl"):
        f["den" + sfx][~(f["den" + sfx] > 0)] = 1.0
    rng = np.random.default_rng(11)
    rho = s[..., 0]
    q = 1e-3 * (1.2 + 0.5 * np.sin(np.arange(rho.size).reshape(rho.shape) * 0.37)) * (1 + 0.1 * rng.random(rho.shape))
    f["rhogq"] = adj.to_device_layout(rho * q)
    f["rhogq_pl"] = torch.as_tensor(sp[..., 0] * 1.3e-3 * (1 + 0.1 * rng.random(sp.shape[:3]))).cuda()
    f["state"], f["state_pl"] = s, sp
    return geo, core, f


@pytest.fixture(scope="module")
def gl04(pkg):
    geo, core, f = _case(pkg, 4)
    yield geo, core, f
    core.close()


def _rand_like(t, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(t.shape, generator=g, dtype=t.dtype, device=t.device)


def _dot(a, b):
    return float((a * b).sum())


def _dot_rel(lhs, rhs, scale):
    return abs(lhs - rhs) / scale


# ---------------------------------------------------------------- forward parity
def test_vertical_advection_equals_oracle(gl04):
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    G = O.Geo(geo)
    dt = float(geo["dtl"])
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        out = torch.empty_like(f["rhogq" + sfx])
        core.vadv_lin(0, f["rhogq" + sfx], f["den" + sfx], f["flx_v" + sfx], f["frhog" + sfx], None, out, dt, 0.0,
                      True, pole)
        conv = (lambda t: t.cpu().numpy()) if pole else adj.from_device_layout
        rhogq, den, flx = conv(f["rhogq" + sfx]), conv(f["den" + sfx]), conv(f["flx_v" + sfx])
        kmin, kmax = G.kmin, G.kmax
        rdz = G.GRD_rdgz
        ck = np.zeros(rhogq.shape + (2,))
        sl = (slice(None),) if pole else (slice(None), slice(None))
        for k in range(kmin, kmax + 1):
            ck[sl + (k, slice(None), 0)] = -flx[sl + (k,)] / den[sl + (k,)] * rdz[k]
            ck[sl + (k, slice(None), 1)] = flx[sl + (k + 1,)] / den[sl + (k,)] * rdz[k]
        want = rhogq.copy()
        O._vertical_advection(G, want, den, flx, ck, np.zeros_like(den), pole, clamp=True)
        got = conv(out)
        assert np.array_equal(got, want), (pole, np.abs(got - want).max())


def test_laplacian_equals_oracle(gl04):
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    G = O.Geo(geo)
    q, q_pl = f["rhogq"], f["rhogq_pl"]
    y, y_pl = torch.empty_like(q), torch.empty_like(q_pl)
    core.laplacian(q, q_pl, y, y_pl)
    a, a_pl = adj.from_device_layout(q), q_pl.cpu().numpy()
    O.comm1(G, a, a_pl)
    assert np.array_equal(adj.from_device_layout(y), O.laplacian(G, a))
    assert np.array_equal(y_pl.cpu().numpy(), O.laplacian_pl(G, a_pl))


def test_vertical_solve_equals_banded_solve(gl04):
    from scipy.linalg import solve_banded
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    b = _rand_like(f["Mc"], 3)
    x = torch.empty_like(b)
    core.vsolve(f["Mc"], f["Mu"], f["Ml"], b, x)
    Mc, Mu, Ml = (adj.from_device_layout(f[k]) for k in ("Mc", "Mu", "Ml"))
    bb, xx = adj.from_device_layout(b), adj.from_device_layout(x)
    rows = slice(kmin + 1, kmax + 1)
    for (i, j, l) in ((3, 4, 0), (1, 1, 5), (8, 2, 9)):
        ab = np.zeros((3, kmax - kmin))
        ab[0, 1:] = Mu[i, j, rows, l][:-1]
        ab[1] = Mc[i, j, rows, l]
        ab[2, :-1] = Ml[i, j, rows, l][1:]
        want = solve_banded((1, 1), ab, bb[i, j, rows, l])
        assert np.allclose(xx[i, j, rows, l], want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
        assert np.all(xx[i, j, :kmin + 1, l] == 0) and np.all(xx[i, j, kmax + 1:, l] == 0)


def _three(f, seed):
    import torch
    v = torch.stack([f["rhogq"] * (1.0 + 0.1 * n) + 1e-4 * _rand_like(f["rhogq"], seed + n) for n in range(3)])
    v_pl = torch.stack([f["rhogq_pl"] * (1.0 + 0.1 * n) for n in range(3)])
    return v.contiguous(), v_pl.contiguous()


def test_divergence_and_gradient_equal_oracle(gl04):
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    G = O.Geo(geo)
    v, v_pl = _three(f, 30)
    y = torch.empty(core.field_shape, dtype=torch.float64, device="cuda")
    y_pl = torch.empty(core.field_shape_pl, dtype=torch.float64, device="cuda")
    core.divergence(v, v_pl, y, y_pl)
    comps = []
    for n in range(3):
        a, a_pl = adj.from_device_layout(v[n]), v_pl[n].cpu().numpy()
        O.comm1(G, a, a_pl)
        comps.append((a, a_pl))
    assert np.array_equal(adj.from_device_layout(y), O.divergence(G, *[c[0] for c in comps]))
    assert np.array_equal(y_pl.cpu().numpy(), O.divergence_pl(G, *[c[1] for c in comps]))
    q, q_pl = f["rhogq"], f["rhogq_pl"]
    g = torch.empty((3,) + core.field_shape, dtype=torch.float64, device="cuda")
    g_pl = torch.empty((3,) + core.field_shape_pl, dtype=torch.float64, device="cuda")
    core.gradient(q, q_pl, g, g_pl)
    a, a_pl = adj.from_device_layout(q), q_pl.cpu().numpy()
    O.comm1(G, a, a_pl)
    want, want_pl = O.gradient(G, a), O.gradient_pl(G, a_pl)
    for d in range(3):
        assert np.array_equal(adj.from_device_layout(g[d]), want[..., d]), d
        assert np.array_equal(g_pl[d].cpu().numpy(), want_pl[..., d]), d


def _hevi_case(geo, seed):
    """the HEVI matrix and solve inputs at gl04: metrics with their unused
    halo corners set to one (a zero there would divide), half-level enthalpy
    and gz near their atmospheric values, prognostic deviations and tendencies
    of plausible sizes, regional (reference layout) and pole"""
    g = dict(geo)
    for k in ("RGSGAM2", "GAM2H", "RGAMH", "RGSQRTH", "RGAM", "RGSGAM2H", "GSGAM2H"):
        for sfx in ("", "_pl"):
            a = np.array(geo["VMTR_" + k + sfx], np.float64)
            a[a == 0] = 1.0
            g["VMTR_" + k + sfx] = a
    rng = np.random.default_rng(seed)
    z = np.asarray(geo["GRD_gzh"], np.float64)
    out = {}
    for sfx, shp in (("", np.shape(geo["VMTR_RGAMH"])), ("_pl", np.shape(geo["VMTR_RGAMH_pl"]))):
        kax = 2 if sfx == "" else 1
        zz = z.reshape([-1 if d == kax else 1 for d in range(len(shp))])
        r = lambda scale: scale * (1.0 + 0.1 * rng.standard_normal(shp))
        out["eth_h" + sfx] = 3.0e5 * (1.0 + 0.01 * rng.standard_normal(shp))
        out["gz" + sfx] = 9.80616 * zz * (1.0 + 1e-3 * rng.standard_normal(shp))
        for k, sc in (("rhogw", 1e-2), ("rhogw0", 1e-2), ("preg0", 1e3), ("rhog0", 1.0), ("Srho", 1e-5),
                      ("Sw", 1e-3), ("Spre", 1.0)):
            out[k + sfx] = r(sc)
    return g, out


HEVI_ARGS = ("rhogw", "rhogw0", "preg0", "rhog0", "Srho", "Sw", "Spre")


def _hevi_dev(x, pole):
    import torch
    _, adj = _mods()
    return torch.as_tensor(np.ascontiguousarray(x)).cuda() if pole else adj.to_device_layout(x)


def test_hevi_matrix_and_solve_equal_oracle(gl04):
    from oracle import nicam_step as O
    _, adj = _mods()
    geo, core, _ = gl04
    g, a = _hevi_case(geo, 40)
    G, m = O.Geo(g), adj.hevi_metrics(g)
    dt = float(geo["dts"])
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    ks = slice(kmin + 1, kmax + 1)
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        back = (lambda t: t.cpu().numpy()) if pole else adj.from_device_layout
        want = O.rhow_matrix(G, a["eth_h" + sfx], a["gz" + sfx], dt, pole)
        got = adj.hevi_matrix(m, _hevi_dev(a["eth_h" + sfx], pole), _hevi_dev(a["gz" + sfx], pole), dt, pole)
        for w, t in zip(want, got):
            x = back(t)
            assert np.array_equal(x[:, ks] if pole else x[:, :, ks], w), pole
        want_x = O.rhow_solver(G, *(a[k + sfx] for k in HEVI_ARGS), *want, dt, pole)
        got_x = adj.hevi_solve(core, m, *(_hevi_dev(a[k + sfx], pole) for k in HEVI_ARGS), *got, dt, pole)
        assert np.array_equal(back(got_x), want_x), (pole, np.abs(back(got_x) - want_x).max())


def test_dot_product_hevi(gl04):
    """forward-mode against reverse-mode through the matrix assembly, the
    source assembly and the tridiagonal solve, in every field argument"""
    import torch
    import torch.autograd.forward_ad as fwAD
    _, adj = _mods()
    geo, core, _ = gl04
    g, a = _hevi_case(geo, 41)
    m = adj.hevi_metrics(g)
    dt = float(geo["dts"])
    names = ("eth_h", "gz") + HEVI_ARGS
    for pole in (False, True):
        sfx = "_pl" if pole else ""
        xs = [_hevi_dev(a[k + sfx], pole) for k in names]
        ds = [_rand_like(x, 50 + n) * x * 1e-3 for n, x in enumerate(xs)]

        def f(*v):
            M = adj.hevi_matrix(m, v[0], v[1], dt, pole)
            return adj.hevi_solve(core, m, *v[2:], *M, dt, pole)
        with fwAD.dual_level():
            tl = fwAD.unpack_dual(f(*[fwAD.make_dual(x, d) for x, d in zip(xs, ds)])).tangent
        leaves = [x.clone().requires_grad_(True) for x in xs]
        y = f(*leaves)
        w = _rand_like(y, 60)
        grads = torch.autograd.grad(y, leaves, w)
        lhs = _dot(tl, w)
        rhs = sum(_dot(d, gr) for d, gr in zip(ds, grads))
        scale = float((tl * w).abs().sum())
        assert _dot_rel(lhs, rhs, scale) <= 1e-12, (pole, lhs, rhs)


# ---------------------------------------------------------------- dot-product tests
@pytest.mark.parametrize("pole", [False, True])
def test_dot_product_vertical_advection(gl04, pole):
    import torch
    geo, core, f = gl04
    sfx = "_pl" if pole else ""
    args = (f["rhogq" + sfx], f["den" + sfx], f["flx_v" + sfx], f["frhog" + sfx])
    dt = float(geo["dtl"])
    x, y = _rand_like(args[0], 5), _rand_like(args[0], 6)
    tl, ad = torch.empty_like(x), torch.empty_like(x)
    core.vadv_lin(1, *args, x, tl, dt, 0.0, True, pole)
    core.vadv_lin(2, *args, y, ad, dt, 0.0, True, pole)
    lhs, rhs = _dot(tl, y), _dot(x, ad)
    scale = float((tl * y).abs().sum())
    assert _dot_rel(lhs, rhs, scale) <= 1e-12, (lhs, rhs)


def test_dot_product_laplacian(gl04):
    import torch
    _, core, f = gl04
    x, x_pl = _rand_like(f["rhogq"], 7), _rand_like(f["rhogq_pl"], 8)
    y, y_pl = _rand_like(f["rhogq"], 9), _rand_like(f["rhogq_pl"], 10)
    tl, tl_pl = torch.empty_like(x), torch.empty_like(x_pl)
    ad, ad_pl = torch.empty_like(x), torch.empty_like(x_pl)
    core.laplacian(x, x_pl, tl, tl_pl)
    core.laplacian(y, y_pl, ad, ad_pl, transpose=True)
    lhs = _dot(tl, y) + _dot(tl_pl, y_pl)
    rhs = _dot(x, ad) + _dot(x_pl, ad_pl)
    scale = float((tl * y).abs().sum() + (tl_pl * y_pl).abs().sum())
    assert _dot_rel(lhs, rhs, scale) <= 1e-12, (lhs, rhs)


def _kh(f, seed):
    """a positive coefficient field of the size the step uses (rhog x CVdry x Kh)"""
    import torch
    rg, rg_pl = f["den"], f["den_pl"]
    return (rg * 717.5 * 9.6e16 * (1.0 + 0.1 * _rand_like(rg, seed).abs()),
            rg_pl * 717.5 * 9.6e16 * (1.0 + 0.1 * _rand_like(rg_pl, seed + 1).abs()))


def test_diffusion_equals_oracle(gl04):
    """exchange + kh-weighted diffusion against the oracle's comm + diffusion
    (the hyperdiffusion's scalar pass, same expressions: bit for bit)"""
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    G = O.Geo(geo)
    q, q_pl = f["rhogq"], f["rhogq_pl"]
    kh, kh_pl = _kh(f, 21)
    y, y_pl = torch.empty_like(q), torch.empty_like(q_pl)
    core.diffusion(kh, kh_pl, q, q_pl, y, y_pl)
    a, a_pl = adj.from_device_layout(q), q_pl.cpu().numpy()
    O.comm1(G, a, a_pl)
    want = O.diffusion(G, a, adj.from_device_layout(kh))
    want_pl = O.diffusion_pl(G, a_pl, kh_pl.cpu().numpy())
    got, got_pl = adj.from_device_layout(y), y_pl.cpu().numpy()
    ins = (slice(1, -1), slice(1, -1))
    assert np.array_equal(got[ins], want[ins]) and np.array_equal(got_pl[0], want_pl[0])


def test_dot_product_diffusion(gl04):
    import torch
    _, core, f = gl04
    kh, kh_pl = _kh(f, 31)
    x, x_pl = _rand_like(f["rhogq"], 32), _rand_like(f["rhogq_pl"], 33)
    y, y_pl = _rand_like(f["rhogq"], 34), _rand_like(f["rhogq_pl"], 35)
    tl, tl_pl = torch.empty_like(x), torch.empty_like(x_pl)
    ad, ad_pl = torch.empty_like(x), torch.empty_like(x_pl)
    core.diffusion(kh, kh_pl, x, x_pl, tl, tl_pl)
    core.diffusion(kh, kh_pl, ad, ad_pl, y, y_pl, transpose=True)
    lhs = _dot(tl, y) + _dot(tl_pl, y_pl)
    rhs = _dot(x, ad) + _dot(x_pl, ad_pl)
    scale = float((tl * y).abs().sum() + (tl_pl * y_pl).abs().sum())
    assert _dot_rel(lhs, rhs, scale) <= 1e-12, (lhs, rhs)


def test_dot_product_diffusion_kh(gl04):
    """<Dk'(C(s)) y> for a coefficient direction dk (the forward operator with
    kh = dk) against <dk, nc_diffusion_kh(s, y)>: the coefficient cotangent"""
    import torch
    _, core, f = gl04
    s, s_pl = _rand_like(f["rhogq"], 81), _rand_like(f["rhogq_pl"], 82)
    dk, dk_pl = _kh(f, 83)
    y, y_pl = _rand_like(f["rhogq"], 84), _rand_like(f["rhogq_pl"], 85)
    tl, tl_pl = torch.empty_like(s), torch.empty_like(s_pl)
    gk, gk_pl = torch.empty_like(s), torch.empty_like(s_pl)
    core.diffusion(dk, dk_pl, s, s_pl, tl, tl_pl)
    core.diffusion_kh(s, s_pl, y, y_pl, gk, gk_pl)
    lhs = _dot(tl, y) + _dot(tl_pl, y_pl)
    rhs = _dot(dk, gk) + _dot(dk_pl, gk_pl)
    scale = float((tl * y).abs().sum() + (tl_pl * y_pl).abs().sum())
    assert _dot_rel(lhs, rhs, scale) <= 1e-12, (lhs, rhs)


def _hdiff_inputs(geo, f):
    """the six fields of the hyperdiffusion (vx, vy, vz, w, tem - tem_bs,
    rho - rho_bs) of the case's state from the oracle's diagnostics, in the
    device layout, with rhog"""
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    G = O.Geo(geo)
    s, sp = f["state"].copy(), f["state_pl"].copy()
    O.comm(G, s, sp)
    P, Pq, P_pl, Pq_pl = s[..., :6].copy(), s[..., 6:].copy(), sp[..., :6].copy(), sp[..., 6:].copy()
    D, D_pl = np.zeros(P.shape), np.zeros(P_pl.shape)
    rho, _, _, rho_pl, _, _ = O.diagnostics(G, P, Pq, D, P_pl, Pq_pl, D_pl)
    fields = [D[..., O.I_vx], D[..., O.I_vy], D[..., O.I_vz], D[..., O.I_w], D[..., O.I_tem] - G.tem_bs,
              rho - G.rho_bs]
    fields_pl = [D_pl[..., O.I_vx], D_pl[..., O.I_vy], D_pl[..., O.I_vz], D_pl[..., O.I_w],
                 D_pl[..., O.I_tem] - G.tem_bs_pl, rho_pl - G.rho_bs_pl]
    x = torch.stack([adj.to_device_layout(a) for a in fields])
    x_pl = torch.stack([torch.as_tensor(np.ascontiguousarray(a)) for a in fields_pl]).cuda()
    oracle_args = (P[..., 0], rho, D, P_pl[..., 0], rho_pl, D_pl)
    return x, x_pl, adj.to_device_layout(P[..., 0]), torch.as_tensor(np.ascontiguousarray(P_pl[..., 0])).cuda(), \
        oracle_args


def test_hyperdiffusion_equals_oracle(gl04):
    """the hyperdiffusion tendency composed from the differentiable
    operators against the oracle's hdiffusion (mod_numfilter.py:845-1578) on
    interior cells and the pole point: relative max difference <= 1e-12"""
    from oracle import nicam_step as O
    _, adj = _mods()
    geo, core, f = gl04
    x, x_pl, rg, rg_pl, oargs = _hdiff_inputs(geo, f)
    got, got_pl = adj.hyperdiffusion(core, x, x_pl, rg, rg_pl, adj.hdiff_setup(geo))
    want, want_pl = O.hdiffusion(O.Geo(geo), *oargs)
    for v in range(6):
        a = adj.from_device_layout(got[v])[1:-1, 1:-1]
        b = want[1:-1, 1:-1, :, :, v]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), v
        ap, bp = got_pl[v][0].cpu().numpy(), want_pl[0, :, :, v]
        assert np.abs(ap - bp).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), v


def test_dot_product_hyperdiffusion(gl04):
    """<H dx, dy> = <dx, H^T dy> for the hyperdiffusion tendency at a fixed
    density, H^T through torch.autograd and the operators' adjoint kernels"""
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    x, x_pl, rg, rg_pl, _ = _hdiff_inputs(geo, f)
    fixed = adj.hdiff_setup(geo)
    dx = (_rand_like(x, 41) * x.abs().mean(dim=(1, 2, 3, 4), keepdim=True)).requires_grad_(True)
    dx_pl = (_rand_like(x_pl, 42) * x_pl.abs().mean(dim=(1, 2, 3), keepdim=True)).requires_grad_(True)
    y, y_pl = adj.hyperdiffusion(core, dx, dx_pl, rg, rg_pl, fixed)
    wy, wy_pl = _rand_like(y, 43), _rand_like(y_pl, 44)
    lhs = float((y * wy).sum().detach() + (y_pl * wy_pl).sum().detach())
    gx, gx_pl = torch.autograd.grad((y * wy).sum() + (y_pl * wy_pl).sum(), (dx, dx_pl))
    rhs = float((dx * gx).sum() + (dx_pl * gx_pl).sum())
    scale = float((y * wy).abs().sum() + (y_pl * wy_pl).abs().sum())
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)


def _momenta(geo, f):
    """the four momenta (rhogvx, rhogvy, rhogvz, rhogw) of the case's state,
    exchanged, in the reference layout and the device layout"""
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    G = O.Geo(geo)
    s, sp = f["state"].copy(), f["state_pl"].copy()
    O.comm(G, s, sp)
    ref = [s[..., n] for n in range(1, 5)], [sp[..., n] for n in range(1, 5)]
    v = torch.stack([adj.to_device_layout(a) for a in ref[0]])
    v_pl = torch.stack([torch.as_tensor(np.ascontiguousarray(a)) for a in ref[1]]).cuda()
    return G, ref, v, v_pl


def test_divdamp_operators_equal_oracle(gl04):
    """exchange + the 3-D divergence damping operator of the four momenta, and
    exchange + the 2-D operator of three components, against the oracle's
    comm + divdamp3d / divdamp (same expressions: bit for bit)"""
    from oracle import nicam_step as O
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    G, (r, r_pl), v, v_pl = _momenta(geo, f)
    y, y_pl = torch.empty_like(v[:3]), torch.empty_like(v_pl[:3])
    core.divdamp3d(v, v_pl, y, y_pl)
    want, want_pl = O.divdamp3d(G, *r), O.divdamp3d_pl(G, *r_pl)
    for d in range(3):
        assert np.array_equal(adj.from_device_layout(y[d]), want[d]), d
        assert np.array_equal(y_pl[d].cpu().numpy(), want_pl[d]), d
    w, w_pl = _three(f, 51)
    core.divdamp2d(w, w_pl, y, y_pl)
    a = np.stack([adj.from_device_layout(t) for t in w], -1)
    a_pl = np.ascontiguousarray(np.moveaxis(w_pl.cpu().numpy(), 0, -1))
    O.comm(G, a, a_pl)
    want = O.divdamp(G, a[..., 0], a[..., 1], a[..., 2])
    want_pl = O.divdamp_pl(G, a_pl[..., 0], a_pl[..., 1], a_pl[..., 2])
    for d in range(3):
        assert np.array_equal(adj.from_device_layout(y[d]), want[d]), d
        assert np.array_equal(y_pl[d].cpu().numpy(), want_pl[d]), d


def test_divergence_damping_equals_oracle(gl04):
    """the divergence damping tendency composed from the differentiable
    operators against the oracle's numfilter_divdamp (mod_numfilter.py:
    2032-2268) on interior cells and the pole point: relative max difference
    <= 1e-12"""
    from oracle import nicam_step as O
    _, adj = _mods()
    geo, core, f = gl04
    G, (r, r_pl), v, v_pl = _momenta(geo, f)
    got, got_pl = adj.divergence_damping(core, v, v_pl, adj.hdiff_setup(geo))
    want, want_pl = O.numfilter_divdamp(G, *r, *r_pl)
    for d in range(3):
        a, b = adj.from_device_layout(got[d])[1:-1, 1:-1], want[d][1:-1, 1:-1]
        tol = 1e-12 * max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= tol, d
        assert np.abs(got_pl[d][0].cpu().numpy() - want_pl[d][0]).max() <= tol, d


def test_dot_product_divdamp(gl04):
    """<D dx, dy> = <dx, D^T dy> for both operators (their transposes with
    the exchange's adjoint) and for the whole tendency through autograd"""
    import torch
    _, adj = _mods()
    geo, core, f = gl04
    _, _, v, v_pl = _momenta(geo, f)
    sc = v.abs().mean(dim=(1, 2, 3, 4), keepdim=True)
    sc_pl = v_pl.abs().mean(dim=(1, 2, 3), keepdim=True)
    for three in (True, False):
        nc = 4 if three else 3
        op = core.divdamp3d if three else core.divdamp2d
        x, x_pl = _rand_like(v[:nc], 61) * sc[:nc], _rand_like(v_pl[:nc], 62) * sc_pl[:nc]
        y, y_pl = _rand_like(v[:3], 63), _rand_like(v_pl[:3], 64)
        tl, tl_pl = torch.empty_like(y), torch.empty_like(y_pl)
        ad, ad_pl = torch.empty_like(x), torch.empty_like(x_pl)
        op(x, x_pl, tl, tl_pl)
        op(ad, ad_pl, y, y_pl, transpose=True)
        lhs = _dot(tl, y) + _dot(tl_pl, y_pl)
        rhs = _dot(x, ad) + _dot(x_pl, ad_pl)
        scale = float((tl * y).abs().sum() + (tl_pl * y_pl).abs().sum())
        assert _dot_rel(lhs, rhs, scale) <= 1e-12, (three, lhs, rhs)
    dx = (_rand_like(v, 65) * sc).requires_grad_(True)
    dx_pl = (_rand_like(v_pl, 66) * sc_pl).requires_grad_(True)
    y, y_pl = adj.divergence_damping(core, dx, dx_pl, adj.hdiff_setup(geo))
    wy, wy_pl = _rand_like(y, 67), _rand_like(y_pl, 68)
    lhs = float((y * wy).sum().detach() + (y_pl * wy_pl).sum().detach())
    gx, gx_pl = torch.autograd.grad((y * wy).sum() + (y_pl * wy_pl).sum(), (dx, dx_pl))
    rhs = float((dx * gx).sum() + (dx_pl * gx_pl).sum())
    scale = float((y * wy).abs().sum() + (y_pl * wy_pl).abs().sum())
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)


def test_dot_product_divergence_and_gradient(gl04):
    """through autograd: forward-mode (the forward stencil on the tangent)
    against reverse-mode (the transposed stencil and the exchange's adjoint)"""
    import torch
    import torch.autograd.forward_ad as fwAD
    _, adj = _mods()
    _, core, f = gl04
    v, v_pl = _three(f, 31)
    dv, dv_pl = _rand_like(v, 32), _rand_like(v_pl, 33)
    q, q_pl = f["rhogq"], f["rhogq_pl"]
    dq, dq_pl = _rand_like(q, 34), _rand_like(q_pl, 35)
    for op, x, x_pl, d, d_pl in ((adj.divergence, v, v_pl, dv, dv_pl), (adj.gradient, q, q_pl, dq, dq_pl)):
        with fwAD.dual_level():
            y, y_pl = op(core, fwAD.make_dual(x, d), fwAD.make_dual(x_pl, d_pl))
            tl, tl_pl = fwAD.unpack_dual(y).tangent, fwAD.unpack_dual(y_pl).tangent
        xs, xs_pl = x.clone().requires_grad_(True), x_pl.clone().requires_grad_(True)
        y, y_pl = op(core, xs, xs_pl)
        w, w_pl = _rand_like(y, 36), _rand_like(y_pl, 37)
        gx, gx_pl = torch.autograd.grad((y, y_pl), (xs, xs_pl), (w, w_pl))
        lhs = _dot(tl, w) + _dot(tl_pl, w_pl)
        rhs = _dot(d, gx) + _dot(d_pl, gx_pl)
        scale = float((tl * w).abs().sum() + (tl_pl * w_pl).abs().sum())
        assert _dot_rel(lhs, rhs, scale) <= 1e-12, (op.__name__, lhs, rhs)


@pytest.mark.parametrize("pole", [False, True])
def test_dot_product_vertical_solve(gl04, pole):
    """b -> x and (Mc, Mu, Ml, b) -> x through autograd: forward-mode (jvp)
    against reverse-mode (vjp)"""
    import torch
    import torch.autograd.forward_ad as fwAD
    _, adj = _mods()
    _, core, f = gl04
    sfx = "_pl" if pole else ""
    M = [f[k + sfx] for k in ("Mc", "Mu", "Ml")]
    b = _rand_like(M[0], 12)
    dM = [1e-3 * _rand_like(m, 20 + n) * m for n, m in enumerate(M)]
    db = _rand_like(b, 13)
    with fwAD.dual_level():
        duals = [fwAD.make_dual(m, d) for m, d in zip(M, dM)] + [fwAD.make_dual(b, db)]
        out = adj.vertical_solve(core, *duals, pole=pole)
        tl = fwAD.unpack_dual(out).tangent
    leaves = [t.clone().requires_grad_(True) for t in M + [b]]
    x = adj.vertical_solve(core, *leaves, pole=pole)
    y = _rand_like(x, 14)
    grads = torch.autograd.grad(x, leaves, y)
    lhs = _dot(tl, y)
    rhs = sum(_dot(d, g) for d, g in zip(dM + [db], grads))
    scale = float((tl * y).abs().sum())
    assert _dot_rel(lhs, rhs, scale) <= 1e-12, (lhs, rhs)


# ---------------------------------------------------------------- finite differences
def test_finite_differences_vertical_advection(gl04):
    """central differences with a relative step of 1e-9 (asserted) and 1e-6
    (reported): the limiter is piecewise linear, and a larger step crosses
    the kink of a min / max in a few cells where two compared values lie
    that close"""
    import torch
    geo, core, f = gl04
    dt = float(geo["dtl"])
    args = (f["den"], f["flx_v"], f["frhog"])
    x0 = f["rhogq"]
    worst = {1e-9: 0.0, 1e-6: 0.0}
    for seed in range(4):
        d = _rand_like(x0, 100 + seed) * x0
        tl = torch.empty_like(x0)
        core.vadv_lin(1, x0, *args, d, tl, dt, 0.0, True, False)
        for eps in worst:
            fp, fm = torch.empty_like(x0), torch.empty_like(x0)
            core.vadv_lin(0, x0 + eps * d, *args, None, fp, dt, 0.0, True, False)
            core.vadv_lin(0, x0 - eps * d, *args, None, fm, dt, 0.0, True, False)
            fd = (fp - fm) / (2 * eps)
            worst[eps] = max(worst[eps], float((fd - tl).norm() / tl.norm()))
    print("vertical advection: finite differences vs tangent-linear, worst relative L2 by step:", worst)
    assert worst[1e-9] <= 1e-6


def _box(geo, lon0, lat0, half=10.0):
    x = np.asarray(geo["GRD_x"])[:, :, 0, :, :]
    lat = np.degrees(np.arcsin(x[..., 2] / np.linalg.norm(x, axis=-1)))
    lon = np.degrees(np.arctan2(x[..., 1], x[..., 0])) % 360.0
    m = (np.abs(lat - lat0) <= half) & (np.abs(((lon - lon0 + 180.0) % 360.0) - 180.0) <= half)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    return m                                              # (i, j, l)


def _chain(pkg, geo, core, f, nsteps):
    import torch
    _, adj = _mods()
    L, K, Gd = core.field_shape[0], core.field_shape[1], core.field_shape[2]
    ncell = int(geo["lall"]) * (Gd - 2) ** 2 + 2
    area = 4 * np.pi * float(geo["RADIUS"]) ** 2 / ncell
    model = adj.ColumnTransport(core, {k: f[k] for k in ("den", "flx_v", "frhog", "den_pl", "flx_v_pl", "frhog_pl")},
                                float(geo["dtl"]), 0.02 * area)
    m = _box(geo, 90.0, 45.0)
    mask = torch.as_tensor(np.ascontiguousarray(np.transpose(m, (2, 1, 0)))[:, None].astype(np.float64)).cuda()
    mask = mask.expand(L, K, Gd, Gd).clone()
    mask[:, :int(geo["kmin"])] = 0
    mask[:, int(geo["kmax"]) + 1:] = 0
    ref = f["rhogq"].clone()

    def loss(q, q_pl, checkpoint=False):
        a, _ = model.run(q, q_pl, nsteps, checkpoint=checkpoint)
        return ((a - ref) ** 2 * mask).sum()
    return model, loss


def test_chain_gradient_checkpointing_and_fd(pkg, gl04):
    import torch
    geo, core, f = gl04
    _, loss = _chain(pkg, geo, core, f, 6)
    grads = {}
    for ck in (False, True):
        q = f["rhogq"].clone().requires_grad_(True)
        q_pl = f["rhogq_pl"].clone().requires_grad_(True)
        L = loss(q, q_pl, ck)
        grads[ck] = torch.autograd.grad(L, (q, q_pl))
    for a, b in zip(grads[False], grads[True]):
        assert float((a - b).norm()) <= 1e-13 * float(a.norm())
    g, g_pl = grads[True]
    worst = {1e-8: 0.0, 1e-6: 0.0}
    for seed in range(16):
        d = _rand_like(f["rhogq"], 200 + seed) * f["rhogq"]
        d_pl = _rand_like(f["rhogq_pl"], 300 + seed) * f["rhogq_pl"]
        an = _dot(g, d) + _dot(g_pl, d_pl)
        for eps in worst:
            with torch.no_grad():
                lp = float(loss(f["rhogq"] + eps * d, f["rhogq_pl"] + eps * d_pl))
                lm = float(loss(f["rhogq"] - eps * d, f["rhogq_pl"] - eps * d_pl))
            worst[eps] = max(worst[eps], abs((lp - lm) / (2 * eps) - an) / abs(an))
    print("chain of 6 steps: central finite differences vs adjoint, worst relative error over 16 directions, "
          "by relative step:", worst)
    assert worst[1e-8] <= 1e-6


def test_chain_cost_and_memory_gl06(pkg):
    """36 steps at grid level 6: forward time, gradient time (forward +
    backward), their ratio, and peak device memory with and without
    checkpointing"""
    import torch
    geo, core, f = _case(pkg, 6)
    try:
        nsteps = 36
        _, loss = _chain(pkg, geo, core, f, nsteps)
        rep = {"grid": "gl06 z40", "steps": nsteps}

        def timed(fn):
            torch.cuda.synchronize()
            t = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            return time.perf_counter() - t

        with torch.no_grad():
            loss(f["rhogq"], f["rhogq_pl"])                  # warm-up
            rep["forward_s"] = min(timed(lambda: loss(f["rhogq"], f["rhogq_pl"])) for _ in range(3))
        for ck in (False, True):
            q = f["rhogq"].clone().requires_grad_(True)
            q_pl = f["rhogq_pl"].clone().requires_grad_(True)
            torch.autograd.grad(loss(q, q_pl, ck), (q, q_pl))
            torch.cuda.synchronize()
            torch.cuda.reset_peak_memory_stats()
            base = torch.cuda.memory_allocated()
            sec = min(timed(lambda: torch.autograd.grad(loss(q, q_pl, ck), (q, q_pl))) for _ in range(3))
            key = "checkpointed" if ck else "stored"
            rep[key] = {"gradient_s": sec, "gradient_over_forward": sec / rep["forward_s"],
                        "peak_extra_bytes": torch.cuda.max_memory_allocated() - base}
        print("adjoint chain:", rep)
        _report("chain", rep)
        # each operator keeps only its input tensor for the backward pass, so
        # checkpointing the steps saves no memory here: both hold about one
        # field per step
        field = 8 * int(np.prod(core.field_shape))
        assert rep["stored"]["peak_extra_bytes"] < 3 * nsteps * field
        assert rep["stored"]["gradient_over_forward"] < 10.0
    finally:
        core.close()


def _report(key, rep):
    out_dir = os.environ.get("NC_REPORT_DIR")
    if not out_dir:
        return
    path = os.path.join(out_dir, "adjoint_report.json")
    data = {}
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[key] = rep
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1)


# ---------------------------------------------------------------- the tracer advection step
def _trc_case(pkg, glevel):
    import torch
    ig, _ = _mods()
    dtl = {4: 600.0, 5: 600.0, 6: 300.0}[glevel]
    gamma = {4: 9.6e16, 5: 1.2e16, 6: 1.5e15}[glevel]
    g = ig.Grid(glevel, vlayer=60, ztop=12000.0, device="cuda", layer="EVEN", topo="NONE")
    geo = g.setup(dtl=dtl, gamma=gamma, nq=4, trcadv=True)
    s, sp = g.trcadv_state()
    core = pkg.NicamCuda(geo, graph=True)
    return geo, core, torch.as_tensor(s).cuda(), torch.as_tensor(sp).cuda()


def _noisy_tracers(s, sp, nq, seed):
    """tie-free positive tracer masses: the density times a smooth field with
    multiplicative noise"""
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    rho, rho_pl = s[..., 0], sp[..., 0]
    idx = torch.arange(rho.numel(), device="cuda", dtype=torch.float64).reshape(rho.shape)
    out, out_pl = [], []
    for n in range(nq):
        q = 1e-3 * (1.2 + 0.5 * torch.sin(idx * (0.37 + 0.05 * n))) * (
            1 + 0.1 * torch.rand(rho.shape, generator=gen, dtype=torch.float64, device="cuda"))
        q_pl = 1.3e-3 * (1 + 0.1 * torch.rand(rho_pl.shape, generator=gen, dtype=torch.float64, device="cuda"))
        out.append((rho * q).permute(3, 2, 1, 0))
        out_pl.append(rho_pl * q_pl)
    return torch.stack(out).contiguous(), torch.stack(out_pl).contiguous()


@pytest.fixture(scope="module")
def trc4(pkg):
    geo, core, s, sp = _trc_case(pkg, 4)
    core.upload_tensor(s, sp)
    core.step(1)
    yield geo, core, s, sp
    core.close()


def test_tracer_step_forward_equals_step(trc4):
    import torch
    _, adj = _mods()
    geo, core, s, sp = trc4
    s1, sp1 = core.download_tensor()
    x, x_pl = adj._tracers(s, sp, 4)
    want, want_pl = adj._tracers(s1, sp1, 4)
    for iq in range(4):
        y, y_pl = torch.empty_like(x[iq]), torch.empty_like(x_pl[iq])
        core.trc_step_lin(0, x[iq], x_pl[iq], None, None, y, y_pl)
        assert torch.equal(y, want[iq]) and torch.equal(y_pl, want_pl[iq]), iq


@pytest.mark.parametrize("field", ["test", "tie-free"])
def test_tracer_step_dot_product(trc4, field):
    import torch
    _, adj = _mods()
    geo, core, s, sp = trc4
    if field == "test":
        x, x_pl = adj._tracers(s, sp, 4)
    else:
        x, x_pl = _noisy_tracers(s, sp, 4, 5)
    worst = 0.0
    for iq in range(4):
        d, d_pl = _rand_like(x[iq], 40 + iq), _rand_like(x_pl[iq], 50 + iq)
        w, w_pl = _rand_like(x[iq], 60 + iq), _rand_like(x_pl[iq], 70 + iq)
        tl, tl_pl, ad, ad_pl = (torch.empty_like(t) for t in (d, d_pl, d, d_pl))
        core.trc_step_lin(1, x[iq], x_pl[iq], d, d_pl, tl, tl_pl)
        core.trc_step_lin(2, x[iq], x_pl[iq], w, w_pl, ad, ad_pl)
        lhs = _dot(tl, w) + _dot(tl_pl, w_pl)
        rhs = _dot(d, ad) + _dot(d_pl, ad_pl)
        scale = float((tl * w).abs().sum() + (tl_pl * w_pl).abs().sum())
        worst = max(worst, _dot_rel(lhs, rhs, scale))
    print(f"tracer step dot-product test ({field} field): worst relative difference {worst:.2e}")
    assert worst <= 1e-12


def test_tracer_step_finite_differences(trc4):
    import torch
    geo, core, s, sp = trc4
    x, x_pl = _noisy_tracers(s, sp, 1, 6)
    x, x_pl = x[0], x_pl[0]
    worst = {1e-9: 0.0, 1e-6: 0.0}
    for seed in range(4):
        d, d_pl = _rand_like(x, 80 + seed) * x, _rand_like(x_pl, 90 + seed) * x_pl
        tl, tl_pl = torch.empty_like(x), torch.empty_like(x_pl)
        core.trc_step_lin(1, x, x_pl, d, d_pl, tl, tl_pl)
        for eps in worst:
            yp, yp_pl, ym, ym_pl = (torch.empty_like(t) for t in (x, x_pl, x, x_pl))
            core.trc_step_lin(0, x + eps * d, x_pl + eps * d_pl, None, None, yp, yp_pl)
            core.trc_step_lin(0, x - eps * d, x_pl - eps * d_pl, None, None, ym, ym_pl)
            fd = torch.cat([((yp - ym) / (2 * eps)).ravel(), ((yp_pl - ym_pl) / (2 * eps)).ravel()])
            t = torch.cat([tl.ravel(), tl_pl.ravel()])
            worst[eps] = max(worst[eps], float((fd - t).norm() / t.norm()))
    print("tracer step: finite differences vs tangent-linear, worst relative L2 by step:", worst)
    assert worst[1e-9] <= 1e-6


def _box_mask(geo, core, nq):
    import torch
    m = _box(geo, 90.0, 30.0)
    L, K, Gd = core.field_shape[0], core.field_shape[1], core.field_shape[2]
    mask = torch.as_tensor(np.ascontiguousarray(np.transpose(m, (2, 1, 0)))[:, None].astype(np.float64)).cuda()
    mask = mask.expand(L, K, Gd, Gd).clone()
    mask[:, :int(geo["kmin"])] = 0
    mask[:, int(geo["kmax"]) + 1:] = 0
    return mask.expand((nq,) + mask.shape)


def _transport_fd(adj, geo, core, s, sp, nsteps, ndir, eps=(1e-8,), every=1, chained=False):
    """gradient of the box loss by the adjoint; for each of ndir seeded
    directions the central differences at each step in eps and, with
    chained, the run's tangent-linear along the direction: worst relative
    differences against the adjoint's directional derivative"""
    import torch
    model = adj.TracerTransport(core, s, sp, checkpoint_every=every)
    x0, x0_pl = _noisy_tracers(s, sp, 4, 7)
    mask = _box_mask(geo, core, 4)

    def loss(x, x_pl):
        y, _ = model.run(x, x_pl, nsteps)
        return ((y - x0) ** 2 * mask).sum()
    x = x0.clone().requires_grad_(True)
    x_pl = x0_pl.clone().requires_grad_(True)
    g, g_pl = torch.autograd.grad(loss(x, x_pl), (x, x_pl))
    worst = {e: 0.0 for e in eps}
    worst_tl = 0.0
    for seed in range(ndir):
        d, d_pl = _rand_like(x0, 500 + seed) * x0, _rand_like(x0_pl, 600 + seed) * x0_pl
        an = _dot(g, d) + _dot(g_pl, d_pl)
        for e in eps:
            with torch.no_grad():
                lp = float(loss(x0 + e * d, x0_pl + e * d_pl))
                lm = float(loss(x0 - e * d, x0_pl - e * d_pl))
            worst[e] = max(worst[e], abs((lp - lm) / (2 * e) - an) / abs(an))
        if chained:
            (y, _), (dy, _) = model.directional(x0, x0_pl, d, d_pl, nsteps)
            tl = float((2.0 * (y - x0) * mask * dy).sum())
            worst_tl = max(worst_tl, abs(tl - an) / abs(an))
    return (g, g_pl), worst, worst_tl


def test_tracer_transport_gradient_gl04(pkg, trc4):
    geo, core, s, sp = trc4
    _, adj = _mods()
    (g1, g1_pl), worst, worst_tl = _transport_fd(adj, geo, core, s, sp, 6, 16, chained=True)
    (g3, g3_pl), _, _ = _transport_fd(adj, geo, core, s, sp, 6, 0, every=3)
    assert float((g1 - g3).norm()) <= 1e-12 * float(g1.norm())
    assert float((g1_pl - g3_pl).norm()) <= 1e-12 * max(float(g1_pl.norm()), 1e-300)
    print("tracer transport, 6 steps at gl04, worst over 16 directions: central differences (step 1e-8)",
          worst[1e-8], "chained tangent-linear", worst_tl)
    assert worst[1e-8] <= 1e-6 and worst_tl <= 1e-10


def test_tracer_transport_gl06(pkg):
    """36 steps of 300 s at grid level 6: finite differences along 16
    directions; the gradient's cost against the forward run and its peak
    memory with a checkpoint every step and every sixth step"""
    import torch
    _, adj = _mods()
    geo, core, s, sp = _trc_case(pkg, 6)
    try:
        nsteps = 36
        _, worst, worst_tl = _transport_fd(adj, geo, core, s, sp, nsteps, 16, eps=(1e-6, 1e-8, 1e-10),
                                           chained=True)
        rep = {"grid": "gl06 z60 trcadv, 4 tracers", "steps": nsteps,
               "fd_worst_rel_16_directions": {str(e): v for e, v in worst.items()},
               "tangent_linear_vs_adjoint_worst_rel_16_directions": worst_tl}

        def timed(fn):
            torch.cuda.synchronize()
            t = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            return time.perf_counter() - t

        def forward():
            core.set_time(0.0)
            core.upload_tensor(s, sp)
            core.step(nsteps)
        forward()
        rep["forward_s"] = min(timed(forward) for _ in range(3))
        mask = _box_mask(geo, core, 4)
        for every in (1, 6):
            model = adj.TracerTransport(core, s, sp, checkpoint_every=every)
            x0, x0_pl = model.initial_tracers()

            def grad():
                x = x0.clone().requires_grad_(True)
                x_pl = x0_pl.clone().requires_grad_(True)
                y, _ = model.run(x, x_pl, nsteps)
                return torch.autograd.grad(((y - x0) ** 2 * mask).sum(), (x, x_pl))
            grad()
            torch.cuda.synchronize()
            torch.cuda.reset_peak_memory_stats()
            base = torch.cuda.memory_allocated()
            sec = min(timed(grad) for _ in range(2))
            rep[f"checkpoint_every_{every}"] = {"gradient_s": sec, "gradient_over_forward": sec / rep["forward_s"],
                                                "peak_extra_bytes": torch.cuda.max_memory_allocated() - base}
        print("tracer transport adjoint:", rep)
        _report("tracer_transport", rep)
        # the run's tangent-linear against its adjoint, along the same 16
        # directions: exact up to rounding.  The central differences are
        # reported: over 36 steps both limiters switch branches within a
        # relative perturbation of 1e-8 in enough cells to show at 1e-3
        assert worst_tl <= 1e-10
        assert rep["checkpoint_every_6"]["peak_extra_bytes"] < rep["checkpoint_every_1"]["peak_extra_bytes"]
    finally:
        core.close()

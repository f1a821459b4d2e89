"""The differentiable dynamics step (dynstep.py) on a B200, float64:

* one large step of the torch composition over the library's operators
  against the oracle's dynamics_step and against the handle's own step
  (gl03 z10 fixtures: DIRECT and NONLINEAR1 hyperdiffusion, the Rayleigh
  sponge): relative max difference <= 1e-12;
* dot-product test of one step, the tangent-linear by forward-mode AD (the
  operators' forward kernels on the tangent) against the adjoint by
  reverse-mode AD (their transposed kernels): 1e-12;
* the Held-Suarez forcing step against the oracle's, and the dot-product
  test of a step followed by it;
* the adjoint configuration: grid level 6, 40 layers, the balanced jet plus
  seeded Gaussian temperature noise (0.1 K), 36 steps of 300 s, loss the sum
  over a 20 x 20 degree box of the squared deviation of the surface pressure
  after the last step from the initial one; the gradient with respect to the
  six initial prognostic fields with a checkpoint every large step, checked
  against the run's tangent-linear along 2 directions and against central
  differences of the handle's own model (nc_step) along 16 seeded directions
  (relative step 1e-6); times and peak memory reported.
"""
import importlib
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    return importlib.import_module("pynicam-dc_b200.dynstep"), importlib.import_module("pynicam-dc_b200.adjoint")


def _dev_state(s, sp):
    import torch
    _, adj = _mods()
    x = torch.stack([adj.to_device_layout(s[..., n]) for n in range(6)])
    x_pl = torch.as_tensor(np.ascontiguousarray(np.moveaxis(sp[..., :6], -1, 0))).cuda()
    nq = s.shape[-1] - 6
    q = torch.stack([adj.to_device_layout(s[..., 6 + n]) for n in range(nq)])
    q_pl = torch.as_tensor(np.ascontiguousarray(np.moveaxis(sp[..., 6:], -1, 0))).cuda()
    return x, x_pl, q, q_pl


def _ref_state(x, x_pl, q, q_pl):
    """device-layout tensors -> reference-layout numpy state"""
    _, adj = _mods()
    s = np.stack([adj.from_device_layout(t) for t in x] + [adj.from_device_layout(t) for t in q], -1)
    sp = np.concatenate([np.moveaxis(x_pl.detach().cpu().numpy(), 0, -1),
                         np.moveaxis(q_pl.detach().cpu().numpy(), 0, -1)], -1)
    return s, sp


def _rel_check(y, y_pl, want, want_pl, tol=1e-12):
    _, adj = _mods()
    for n in range(6):
        a, b = adj.from_device_layout(y[n])[1:-1, 1:-1], want[1:-1, 1:-1, :, :, n]
        t = tol * np.abs(b).max()
        assert np.abs(a - b).max() <= t, (n, np.abs(a - b).max() / np.abs(b).max())
        assert np.abs(y_pl[n][0].detach().cpu().numpy() - want_pl[0, :, :, n]).max() <= t, n


@pytest.mark.parametrize("case", ["golden", "golden_nlhdiff", "golden_rayleigh"])
def test_step_equals_oracle_and_handle(pkg, case, request):
    """DIRECT and NONLINEAR1 hyperdiffusion, the Rayleigh sponge"""
    from oracle import nicam_step as O
    import torch
    ds, _ = _mods()
    geo, st = request.getfixturevalue(case)
    core = pkg.NicamCuda(geo, graph=False)
    try:
        s, sp = st["state0"], st["state0_pl"]
        stepper = ds.DynamicsStep(core, geo)
        with torch.no_grad():
            y, y_pl = stepper.step(*_dev_state(s, sp))
        want, want_pl = O.dynamics_step(O.Geo(geo), s, sp)
        _rel_check(y, y_pl, want, want_pl)
        core.upload(s, sp)
        core.step(1)
        got, got_pl = core.download()
        _rel_check(y, y_pl, got, got_pl)
    finally:
        core.close()


def _rand_like(t, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(t.shape, generator=g, dtype=t.dtype, device=t.device)


def _scaled(x, x_pl, seed):
    """a direction per prognostic field at the field's magnitude"""
    sc = x.abs().mean(dim=(1, 2, 3, 4), keepdim=True)
    return _rand_like(x, seed) * sc, _rand_like(x_pl, seed + 1) * sc.view(6, 1, 1, 1)


@pytest.mark.parametrize("case", ["golden", "golden_nlhdiff"])
def test_dot_product_step(pkg, case, request):
    """<J dx, w> = <dx, J^T w> for one large step"""
    import torch
    import torch.autograd.forward_ad as fwAD
    ds, _ = _mods()
    geo, st = request.getfixturevalue(case)
    core = pkg.NicamCuda(geo, graph=False)
    x, x_pl, q, q_pl = _dev_state(st["state0"], st["state0_pl"])
    stepper = ds.DynamicsStep(core, geo)
    dx, dx_pl = _scaled(x, x_pl, 71)
    with fwAD.dual_level():
        y, y_pl = stepper.step(fwAD.make_dual(x, dx), fwAD.make_dual(x_pl, dx_pl), q, q_pl)
        ty, ty_pl = fwAD.unpack_dual(y).tangent, fwAD.unpack_dual(y_pl).tangent
    w, w_pl = _rand_like(ty, 73), _rand_like(ty_pl, 74)
    xr, xr_pl = x.clone().requires_grad_(True), x_pl.clone().requires_grad_(True)
    y, y_pl = stepper.step(xr, xr_pl, q, q_pl)
    g, g_pl = torch.autograd.grad((y * w).sum() + (y_pl * w_pl).sum(), (xr, xr_pl))
    lhs = float((ty * w).sum() + (ty_pl * w_pl).sum())
    rhs = float((dx * g).sum() + (dx_pl * g_pl).sum())
    scale = float((ty * w).abs().sum() + (ty_pl * w_pl).abs().sum())
    core.close()
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)


def test_held_suarez_step(pkg, golden_hs):
    """the Held-Suarez forcing step on the device against the oracle's
    forcing_step_hs (1e-12), and the dot-product test of a large step
    followed by it (1e-12)"""
    from oracle import nicam_step as O
    import torch
    import torch.autograd.forward_ad as fwAD
    ds, adj = _mods()
    geo, lat, st = golden_hs
    core = pkg.NicamCuda(geo, graph=False)
    try:
        s, sp = st["state1"], st["state1_pl"]
        x, x_pl, q, q_pl = _dev_state(s, sp)
        m = ds.Metrics(geo)
        latt = torch.as_tensor(np.ascontiguousarray(np.transpose(np.asarray(lat, np.float64), (2, 1, 0)))[:, None]).cuda()
        Q = [ds.F(q[n], q_pl[n]) for n in range(q.shape[0])]
        with torch.no_grad():
            y, y_pl = ds.stack(ds.held_suarez(m, core, ds.unstack(x, x_pl), latt, Q))
        _rel_check(y, y_pl, *O.forcing_step_hs(O.Geo(geo), s, sp, lat))
        stepper = ds.DynamicsStep(core, geo, hs_lat=lat)
        dx, dx_pl = _scaled(x, x_pl, 91)
        with fwAD.dual_level():
            y, y_pl = stepper.step(fwAD.make_dual(x, dx), fwAD.make_dual(x_pl, dx_pl), q, q_pl)
            ty, ty_pl = fwAD.unpack_dual(y).tangent, fwAD.unpack_dual(y_pl).tangent
        w, w_pl = _rand_like(ty, 93), _rand_like(ty_pl, 94)
        xr, xr_pl = x.clone().requires_grad_(True), x_pl.clone().requires_grad_(True)
        y, y_pl = stepper.step(xr, xr_pl, q, q_pl)
        g, g_pl = torch.autograd.grad((y * w).sum() + (y_pl * w_pl).sum(), (xr, xr_pl))
        lhs = float((ty * w).sum() + (ty_pl * w_pl).sum())
        rhs = float((dx * g).sum() + (dx_pl * g_pl).sum())
        scale = float((ty * w).abs().sum() + (ty_pl * w_pl).abs().sum())
        assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)
    finally:
        core.close()


def _report(key, rep):
    out_dir = os.environ.get("NC_REPORT_DIR")
    if not out_dir:
        return
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "dynstep_report.json")
    data = {}
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[key] = rep
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1)


def _box(geo, lon0, lat0, half=10.0):
    x = np.asarray(geo["GRD_x"])[:, :, 0, :, :]
    lat = np.degrees(np.arcsin(x[..., 2] / np.linalg.norm(x, axis=-1)))
    lon = np.degrees(np.arctan2(x[..., 1], x[..., 0])) % 360.0
    m = (np.abs(lat - lat0) <= half) & (np.abs(((lon - lon0 + 180.0) % 360.0) - 180.0) <= half)
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    return m                                              # (i, j, l)


def test_adjoint_gl06(pkg):
    from oracle import nicam_step as O
    import torch
    import torch.autograd.forward_ad as fwAD
    ds, _ = _mods()
    ig = importlib.import_module("pynicam-dc_b200.icogrid")
    nsteps = 36
    g = ig.Grid(6, vlayer=40, ztop=30000.0, device="cuda")
    geo = g.setup(dtl=300.0, gamma=1.5e15, nq=1)
    s, sp = g.jw_state(nq=1)
    kmin, kmax = int(geo["kmin"]), int(geo["kmax"])
    cv = float(np.asarray(geo["CVdry"]).reshape(-1)[0])
    rng = np.random.default_rng(2012)
    dT = rng.normal(0.0, 0.1, s.shape[:4])
    dT_pl = rng.normal(0.0, 0.1, sp.shape[:3])
    dT[:, :, :kmin], dT[:, :, kmax + 1:] = 0.0, 0.0
    dT_pl[:, :kmin], dT_pl[:, kmax + 1:] = 0.0, 0.0
    s[..., 5] += s[..., 0] * cv * dT
    sp[..., 5] += sp[..., 0] * cv * dT_pl
    O.comm(O.Geo(geo), s, sp)
    core = pkg.NicamCuda(geo, graph=False)
    try:
        stepper = ds.DynamicsStep(core, geo)
        x0, x0_pl, q, q_pl = _dev_state(s, sp)
        L, K, Gd = core.field_shape[0], core.field_shape[1], core.field_shape[2]
        zk_val = float(np.asarray(geo["GRD_gz"])[kmin])      # flat surface: the level's height
        zk = torch.full((L, 1, Gd, Gd), zk_val, dtype=torch.float64, device="cuda")
        zk_pl = torch.full((x0_pl.shape[1], 1, x0_pl.shape[3]), zk_val, dtype=torch.float64, device="cuda")
        mask = torch.as_tensor(np.ascontiguousarray(np.transpose(_box(geo, 20.0, 40.0), (2, 1, 0)))[:, None]
                               .astype(np.float64)).cuda()
        ps0 = stepper.surface_pressure(x0, x0_pl, zk, zk_pl)[0].detach()

        def loss_of(x, x_pl):
            ps, _ = stepper.surface_pressure(x, x_pl, zk, zk_pl)
            return (((ps - ps0) ** 2) * mask).sum()

        def timed(fn):
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            return time.perf_counter() - t, r

        def fwd():
            with torch.no_grad():
                return loss_of(*stepper.run(x0, x0_pl, nsteps, checkpoint=False, tracers=q, tracers_pl=q_pl))
        t_fwd, loss0 = timed(fwd)

        def grad():
            xr, xr_pl = x0.clone().requires_grad_(True), x0_pl.clone().requires_grad_(True)
            y, y_pl = stepper.run(xr, xr_pl, nsteps, checkpoint=True, tracers=q, tracers_pl=q_pl)
            return torch.autograd.grad(loss_of(y, y_pl), (xr, xr_pl))
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        base = torch.cuda.memory_allocated()
        t_grad, (gx, gx_pl) = timed(grad)
        peak = torch.cuda.max_memory_allocated() - base

        def handle_loss(x, x_pl):
            core.upload(*_ref_state(x, x_pl, q, q_pl))
            core.step(nsteps)
            out, out_pl = core.download()
            y, y_pl, _, _ = _dev_state(out, out_pl)
            with torch.no_grad():
                return float(loss_of(y, y_pl))
        t_handle, _ = timed(lambda: handle_loss(x0, x0_pl))

        def direction(seed):
            d, d_pl = _scaled(x0, x0_pl, seed)
            core.exchange(d, d_pl)                      # a halo-consistent direction
            return d, d_pl

        worst_tl, worst_fd, eps = 0.0, 0.0, 1e-6
        for n in range(16):
            d, d_pl = direction(300 + 2 * n)
            adj_dd = float((gx * d).sum() + (gx_pl * d_pl).sum())
            if n < 2:
                with fwAD.dual_level(), torch.no_grad():
                    y, y_pl = stepper.run(fwAD.make_dual(x0, d), fwAD.make_dual(x0_pl, d_pl), nsteps,
                                          checkpoint=False, tracers=q, tracers_pl=q_pl)
                    tl = float(fwAD.unpack_dual(loss_of(y, y_pl)).tangent)
                worst_tl = max(worst_tl, abs(tl - adj_dd) / abs(adj_dd))
            fd = (handle_loss(x0 + eps * d, x0_pl + eps * d_pl) - handle_loss(x0 - eps * d, x0_pl - eps * d_pl)) \
                / (2 * eps)
            worst_fd = max(worst_fd, abs(fd - adj_dd) / abs(adj_dd))
        rep = {"grid": "gl06 z40 JW + 0.1 K noise", "steps": nsteps, "loss": float(loss0),
               "forward_restatement_s": t_fwd, "gradient_s": t_grad, "gradient_over_forward": t_grad / t_fwd,
               "handle_forward_s": t_handle, "gradient_peak_extra_bytes": peak,
               "tangent_linear_vs_adjoint_worst_rel_2_directions": worst_tl,
               "fd_handle_vs_adjoint_worst_rel_16_directions_eps_1e-6": worst_fd}
        print("dynamics adjoint:", rep)
        _report("dynamics_adjoint_gl06", rep)
        assert worst_tl <= 1e-9
        assert worst_fd <= 1e-4
    finally:
        core.close()

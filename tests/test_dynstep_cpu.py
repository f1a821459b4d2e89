"""The differentiable restatement of the dynamics step (dynstep.py) on the
CPU: its torch composition, with the library's operators replaced by
stand-ins that call the oracle's stencils (forward only), against the
oracle's own dynamics_step on the gl03 z10 fixture."""
import importlib

import numpy as np
import pytest
import torch


def _mods():
    return importlib.import_module("pynicam-dc_b200.dynstep"), importlib.import_module("pynicam-dc_b200.adjoint")


class OracleOps:
    """the operator surface of a handle (field shapes, levels, the stencils
    the autograd wrappers call), computed by the oracle on CPU tensors"""

    def __init__(self, geo):
        from oracle import nicam_step as O
        self.O, self.G = O, O.Geo(geo)
        g = self.G
        self.field_shape = (g.lall, g.kall, g.gall_1d, g.gall_1d)
        self.field_shape_pl = tuple(np.asarray(geo["VMTR_GSGAM2_pl"]).shape)
        self.kmin, self.kmax = g.kmin, g.kmax

    @staticmethod
    def _r(t):
        return t.detach().permute(3, 2, 1, 0).numpy().copy()

    @staticmethod
    def _put(dst, a):
        dst.copy_(torch.as_tensor(np.ascontiguousarray(np.moveaxis(a, (0, 1, 2, 3), (3, 2, 1, 0)))))

    def _comm(self, v, v_pl):
        """v (n,) + field shape -> exchanged (i,j,k,l,n) and (g,k,l,n)"""
        a = np.stack([self._r(t) for t in v], -1)
        ap = np.ascontiguousarray(np.moveaxis(v_pl.detach().numpy(), 0, -1))
        self.O.comm(self.G, a, ap)
        return a, ap

    def _no_t(self, transpose):
        if transpose:
            raise NotImplementedError("forward only")

    def exchange(self, x, x_pl, transpose=False):
        self._no_t(transpose)
        one = x.dim() == len(self.field_shape)
        xs, xps = (x[None], x_pl[None]) if one else (x, x_pl)
        a, ap = self._comm(xs, xps)
        for n in range(xs.shape[0]):
            self._put(xs[n], a[..., n])
            xps[n].copy_(torch.as_tensor(ap[..., n]))

    def laplacian(self, q, q_pl, y, y_pl, transpose=False):
        self._no_t(transpose)
        a, ap = self._comm(q[None], q_pl[None])
        self._put(y, self.O.laplacian(self.G, a[..., 0]))
        y_pl.copy_(torch.as_tensor(self.O.laplacian_pl(self.G, ap[..., 0])))

    def divergence(self, v, v_pl, y, y_pl, transpose=False):
        self._no_t(transpose)
        a, ap = self._comm(v, v_pl)
        self._put(y, self.O.divergence(self.G, a[..., 0], a[..., 1], a[..., 2]))
        y_pl.copy_(torch.as_tensor(self.O.divergence_pl(self.G, ap[..., 0], ap[..., 1], ap[..., 2])))

    def gradient(self, q, q_pl, g, g_pl, transpose=False):
        self._no_t(transpose)
        a, ap = self._comm(q[None], q_pl[None])
        r, p = self.O.gradient(self.G, a[..., 0]), self.O.gradient_pl(self.G, ap[..., 0])
        for d in range(3):
            self._put(g[d], r[..., d])
            g_pl[d].copy_(torch.as_tensor(p[..., d]))

    def diffusion(self, kh, kh_pl, s, s_pl, y, y_pl, transpose=False):
        self._no_t(transpose)
        a, ap = self._comm(s[None], s_pl[None])
        self._put(y, self.O.diffusion(self.G, a[..., 0], self._r(kh)))
        y_pl.copy_(torch.as_tensor(self.O.diffusion_pl(self.G, ap[..., 0], kh_pl.detach().numpy())))

    def _dd(self, v, v_pl, y, y_pl, transpose, f, fp):
        self._no_t(transpose)
        a, ap = self._comm(v, v_pl)
        r = f(self.G, *[a[..., n] for n in range(a.shape[-1])])
        p = fp(self.G, *[ap[..., n] for n in range(ap.shape[-1])])
        for d in range(3):
            self._put(y[d], r[d])
            y_pl[d].copy_(torch.as_tensor(p[d]))

    def divdamp3d(self, v, v_pl, y, y_pl, transpose=False):
        self._dd(v, v_pl, y, y_pl, transpose, self.O.divdamp3d, self.O.divdamp3d_pl)

    def divdamp2d(self, v, v_pl, y, y_pl, transpose=False):
        self._dd(v, v_pl, y, y_pl, transpose, self.O.divdamp, self.O.divdamp_pl)

    def vsolve(self, Mc, Mu, Ml, b, x, pole=False, transpose=False, x_fwd=None, gM=None):
        """the Thomas solve on rows kmin+1..kmax of the level axis (the
        oracle's rhow_solver recurrence)"""
        self._no_t(transpose)
        k0, k1 = self.kmin + 1, self.kmax
        C, U, L, S = (t.detach()[:, k0:k1 + 1] for t in (Mc, Mu, Ml, b))
        N = k1 - k0 + 1
        beta = C[:, 0]
        u, gam = [S[:, 0] / beta], [None] * N
        for n in range(1, N):
            gg = U[:, n - 1] / beta
            beta = C[:, n] - L[:, n] * gg
            u.append((S[:, n] - L[:, n] * u[n - 1]) / beta)
            gam[n] = gg
        xs = [None] * N
        xs[N - 1] = u[N - 1]
        for n in range(N - 2, -1, -1):
            xs[n] = u[n] - gam[n + 1] * xs[n + 1]
        x.zero_()
        x[:, k0:k1 + 1] = torch.stack(xs, 1)


@pytest.mark.parametrize("case", ["golden", "golden_nlhdiff", "golden_rayleigh"])
def test_step_equals_oracle(case, request):
    """one large step of the torch composition against the oracle's
    dynamics_step (DIRECT and NONLINEAR1 hyperdiffusion, the Rayleigh
    sponge): relative max difference <= 1e-12 per prognostic"""
    from oracle import nicam_step as O
    ds, adj = _mods()
    geo, st = request.getfixturevalue(case)
    ops = OracleOps(geo)
    stepper = ds.DynamicsStep(ops, geo, device="cpu")
    s, sp = st["state0"], st["state0_pl"]
    x = torch.stack([adj.to_device_layout(s[..., n], "cpu") for n in range(6)])
    x_pl = torch.as_tensor(np.ascontiguousarray(np.moveaxis(sp[..., :6], -1, 0)))
    nq = s.shape[-1] - 6
    q = torch.stack([adj.to_device_layout(s[..., 6 + n], "cpu") for n in range(nq)])
    q_pl = torch.as_tensor(np.ascontiguousarray(np.moveaxis(sp[..., 6:], -1, 0)))
    with torch.no_grad():
        y, y_pl = stepper.step(x, x_pl, q, q_pl)
    want, want_pl = O.dynamics_step(O.Geo(geo), s, sp)
    for n in range(6):
        a, b = adj.from_device_layout(y[n])[1:-1, 1:-1], want[1:-1, 1:-1, :, :, n]
        tol = 1e-12 * np.abs(b).max()
        assert np.abs(a - b).max() <= tol, (n, np.abs(a - b).max() / np.abs(b).max())
        assert np.abs(y_pl[n][0].numpy() - want_pl[0, :, :, n]).max() <= tol, n


def test_held_suarez_equals_oracle(golden_hs):
    """the Held-Suarez forcing step (diagnostics, tendencies, update,
    exchange) from the fixture's states against the oracle's
    forcing_step_hs: relative max difference <= 1e-12 per prognostic"""
    from oracle import nicam_step as O
    ds, adj = _mods()
    geo, lat, st = golden_hs
    ops = OracleOps(geo)
    m = ds.Metrics(geo, device="cpu")
    latt = torch.as_tensor(np.ascontiguousarray(np.transpose(np.asarray(lat, np.float64), (2, 1, 0)))[:, None])
    G = O.Geo(geo)
    for name in ("state0", "state1"):
        s, sp = st[name], st[name + "_pl"]
        x = torch.stack([adj.to_device_layout(s[..., n], "cpu") for n in range(6)])
        x_pl = torch.as_tensor(np.ascontiguousarray(np.moveaxis(sp[..., :6], -1, 0)))
        Q = [ds.F(adj.to_device_layout(s[..., 6 + n], "cpu"), torch.as_tensor(np.ascontiguousarray(sp[..., 6 + n])))
             for n in range(s.shape[-1] - 6)]
        with torch.no_grad():
            y, y_pl = ds.stack(ds.held_suarez(m, ops, ds.unstack(x, x_pl), latt, Q))
        want, want_pl = O.forcing_step_hs(G, s, sp, lat)
        for n in range(6):
            a, b = adj.from_device_layout(y[n])[1:-1, 1:-1], want[1:-1, 1:-1, :, :, n]
            tol = 1e-12 * np.abs(b).max()
            assert np.abs(a - b).max() <= tol, (name, n, np.abs(a - b).max() / np.abs(b).max())
            assert np.abs(y_pl[n][0].numpy() - want_pl[0, :, :, n]).max() <= tol, (name, n)

"""Differentiation of step operators through PyTorch autograd.

Each operator is a ``torch.autograd.Function`` whose forward, tangent-linear
(``jvp``, forward-mode AD) and adjoint (``backward``, reverse-mode AD) are the
library's hand-written float64 kernels (``nc_vsolve``, ``nc_vadv_lin``,
``nc_laplacian``), on CUDA tensors in the handle's device layout: regional
fields of shape (lall, kall, gall_1d, gall_1d), pole fields (6, kall, 2).

* ``VerticalSolve`` -- the HEVI tridiagonal system of
  kernels/virhowsolver.py:67-122; the adjoint is the transposed solve plus
  the matrix cotangents, differentiable in the matrix and the right-hand side.
* ``VerticalAdvection`` -- one vertical tracer advection step with the
  vertical Thuburn limiter (mod_src_tracer.py:389-533, 1909-2074),
  differentiable in the tracer mass; the limiter's branches are those of the
  forward evaluation (active-branch linearisation); density, vertical mass
  flux and density tendency are held fixed (passing one that requires a
  gradient is an error).
* ``Laplacian`` -- halo exchange then the hexagonal Laplacian
  (kernels/oprtlaplacian.py:41-70), linear; the adjoint runs the transposed
  stencil and adds each halo value back into its exchange source.
* ``hevi_matrix`` / ``hevi_solve`` -- the HEVI vertical implicit step
  (kernels/vimatrix.py:67-164, kernels/virhowsolver.py:42-172): the matrix
  and source assembly as torch expressions in the reference's operation
  order around ``VerticalSolve``, differentiable in every field.
* ``Divergence`` / ``Gradient`` -- halo exchange then OPRT_divergence
  (kernels/fluxconv.py:52-108) / OPRT_gradient (kernels/oprtgradient.py:
  45-88), linear, adjoints as for the Laplacian (``nc_divergence``,
  ``nc_gradient``).

* ``Diffusion`` -- halo exchange then the Kh-weighted diffusion of the
  hyperdiffusion's scalar pass (kernels/oprtdiffusion.py), bilinear in the
  field and the coefficient field: adjoints ``nc_diffusion`` (transposed)
  and ``nc_diffusion_kh`` (the coefficient's cotangent).
* ``divdamp3d`` / ``divdamp2d`` -- halo exchange then the divergence
  damping's 3-D / 2-D operator (kernels/oprt3ddivdamp.py, oprtdivdamp.py),
  linear (``nc_divdamp3d``, ``nc_divdamp2d``); ``hyperdiffusion`` and
  ``divergence_damping`` compose the two filters' tendencies.
* ``Exchange`` -- the halo exchange alone (share/mod_comm.py:1563-1644),
  linear (``nc_exchange``).

The whole dynamics step built from these operators is ``dynstep.DynamicsStep``.

* ``TracerStep`` -- the whole tracer advection of a step
  (mod_src_tracer.py:83-1228: vertical step, horizontal step with the
  horizontal Thuburn limiter of 2190-2605, vertical step with the clamp, the
  closing exchange) for the winds and densities of the handle's last step,
  differentiable in the tracer mass (``nc_trc_step_lin``).

``ColumnTransport`` chains the operators into a multi-step tracer model
(vertical advection with the limiter, then horizontal diffusion by the
Laplacian) whose steps can be checkpointed with ``torch.utils.checkpoint``.

``TracerTransport`` differentiates a run of the handle's own steps with
respect to the initial tracer masses of all tracers (the winds do not depend
on the tracers: the offline advection, or passive tracers): the forward pass
stores the full state every ``checkpoint_every`` steps; the backward pass
re-runs each segment from its stored state, keeping the segment's per-step
states, and walks back through it, re-running each step to put its winds and
densities on the handle before applying the step's adjoint.

The reference obtains gradients with jax.vjp of its jax backend; jax is not
part of this build's environment, so the checks here are the dot-product
test (tangent-linear against adjoint) and central finite differences.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.utils.checkpoint

from .runtime import _scalar


def to_device_layout(field, device="cuda"):
    """(gall_1d, gall_1d, kall, lall) array -> (lall, kall, gall_1d, gall_1d) tensor"""
    t = torch.as_tensor(np.asarray(field, np.float64) if not torch.is_tensor(field) else field)
    return t.permute(3, 2, 1, 0).contiguous().to(device)


def from_device_layout(t):
    """inverse of ``to_device_layout`` (returns a numpy array)"""
    return t.detach().permute(3, 2, 1, 0).contiguous().cpu().numpy()


def _c(t):
    return t.contiguous()


def _fixed(name, *ts):
    for t in ts:
        if t is not None and t.requires_grad:
            raise ValueError(f"{name}: density, fluxes and tendencies are held fixed; detach them")


class VerticalSolve(torch.autograd.Function):
    """x = M^-1 b per column, M tridiagonal (Mc, Mu, Ml)"""

    @staticmethod
    def forward(ctx, core, pole, Mc, Mu, Ml, b):
        Mc, Mu, Ml, b = _c(Mc), _c(Mu), _c(Ml), _c(b)
        x = torch.empty_like(b)
        core.vsolve(Mc, Mu, Ml, b, x, pole=pole)
        ctx.core, ctx.pole = core, pole
        ctx.save_for_backward(Mc, Mu, Ml, x)
        ctx.save_for_forward(Mc, Mu, Ml, x)
        return x

    @staticmethod
    def backward(ctx, gx):
        Mc, Mu, Ml, x = ctx.saved_tensors
        gb = torch.empty_like(x)
        gM = tuple(torch.empty_like(x) for _ in range(3))
        ctx.core.vsolve(Mc, Mu, Ml, _c(gx), gb, pole=ctx.pole, transpose=True, x_fwd=x, gM=gM)
        return None, None, gM[0], gM[1], gM[2], gb

    @staticmethod
    def jvp(ctx, _core, _pole, dMc, dMu, dMl, db):
        # dx = M^-1 (db - dM x) on the system rows kmin+1..kmax
        Mc, Mu, Ml, x = ctx.saved_tensors
        k0, k1 = ctx.core.kmin + 1, ctx.core.kmax
        r = torch.zeros_like(x) if db is None else db.clone()
        rs = r[:, k0:k1 + 1]
        if dMc is not None:
            rs -= dMc[:, k0:k1 + 1] * x[:, k0:k1 + 1]
        if dMu is not None:
            rs[:, :-1] -= dMu[:, k0:k1] * x[:, k0 + 1:k1 + 1]
        if dMl is not None:
            rs[:, 1:] -= dMl[:, k0 + 1:k1 + 1] * x[:, k0:k1]
        dx = torch.empty_like(x)
        ctx.core.vsolve(Mc, Mu, Ml, _c(r), dx, pole=ctx.pole)
        return dx


class VerticalAdvection(torch.autograd.Function):
    """one vertical tracer advection step of rhogq (den, flx_v, frhog fixed)"""

    @staticmethod
    def forward(ctx, core, pole, rhogq, den, flx_v, frhog, dt, bcoef, clamp):
        _fixed("VerticalAdvection", den, flx_v, frhog)
        rhogq, den, flx_v, frhog = _c(rhogq), _c(den), _c(flx_v), _c(frhog)
        out = torch.empty_like(rhogq)
        core.vadv_lin(0, rhogq, den, flx_v, frhog, None, out, dt, bcoef, clamp, pole)
        ctx.core, ctx.args = core, (pole, dt, bcoef, clamp)
        ctx.save_for_backward(rhogq, den, flx_v, frhog)
        ctx.save_for_forward(rhogq, den, flx_v, frhog)
        return out

    @staticmethod
    def backward(ctx, g):
        rhogq, den, flx_v, frhog = ctx.saved_tensors
        pole, dt, bcoef, clamp = ctx.args
        gq = torch.empty_like(rhogq)
        ctx.core.vadv_lin(2, rhogq, den, flx_v, frhog, _c(g), gq, dt, bcoef, clamp, pole)
        return None, None, gq, None, None, None, None, None, None

    @staticmethod
    def jvp(ctx, _core, _pole, drhogq, *_rest):
        rhogq, den, flx_v, frhog = ctx.saved_tensors
        pole, dt, bcoef, clamp = ctx.args
        out = torch.empty_like(rhogq)
        if drhogq is None:
            return out.zero_()
        ctx.core.vadv_lin(1, rhogq, den, flx_v, frhog, _c(drhogq), out, dt, bcoef, clamp, pole)
        return out


class Laplacian(torch.autograd.Function):
    """(y, y_pl) = L(C(q, q_pl)): halo exchange then the hexagonal Laplacian"""

    @staticmethod
    def forward(ctx, core, q, q_pl):
        y, y_pl = torch.empty_like(q), torch.empty_like(q_pl)
        core.laplacian(_c(q), _c(q_pl), y, y_pl)
        ctx.core = core
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        core = ctx.core
        gy = torch.zeros(core.field_shape, dtype=torch.float64, device="cuda") if gy is None else _c(gy)
        gy_pl = torch.zeros(core.field_shape_pl, dtype=torch.float64, device=gy.device) if gy_pl is None else _c(gy_pl)
        g, g_pl = torch.empty_like(gy), torch.empty_like(gy_pl)
        core.laplacian(gy, gy_pl, g, g_pl, transpose=True)
        return None, g, g_pl

    @staticmethod
    def jvp(ctx, _core, dq, dq_pl):
        core = ctx.core
        dq = torch.zeros(core.field_shape, dtype=torch.float64, device="cuda") if dq is None else _c(dq)
        dq_pl = torch.zeros(core.field_shape_pl, dtype=torch.float64, device=dq.device) if dq_pl is None else _c(dq_pl)
        y, y_pl = torch.empty_like(dq), torch.empty_like(dq_pl)
        core.laplacian(dq, dq_pl, y, y_pl)
        return y, y_pl


class Divergence(torch.autograd.Function):
    """(y, y_pl) = D(C(v, v_pl)): halo exchange of the three components then
    the divergence (kernels/fluxconv.py:52-108); v of shape (3, lall, kall,
    g, g), v_pl (3, 6, kall, LP)"""

    @staticmethod
    def forward(ctx, core, v, v_pl):
        v, v_pl = _c(v), _c(v_pl)
        y = torch.empty(core.field_shape, dtype=torch.float64, device=v.device)
        y_pl = torch.empty(core.field_shape_pl, dtype=torch.float64, device=v.device)
        core.divergence(v, v_pl, y, y_pl)
        ctx.core = core
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        core = ctx.core
        gy = torch.zeros(core.field_shape, dtype=torch.float64, device="cuda") if gy is None else _c(gy)
        gy_pl = torch.zeros(core.field_shape_pl, dtype=torch.float64, device="cuda") if gy_pl is None else _c(gy_pl)
        gv = torch.empty((3,) + core.field_shape, dtype=torch.float64, device=gy.device)
        gv_pl = torch.empty((3,) + core.field_shape_pl, dtype=torch.float64, device=gy.device)
        core.divergence(gv, gv_pl, gy, gy_pl, transpose=True)
        return None, gv, gv_pl

    @staticmethod
    def jvp(ctx, _core, dv, dv_pl):
        return Divergence.forward(ctx, ctx.core, dv, dv_pl)


class Gradient(torch.autograd.Function):
    """(g, g_pl) = Grad(C(q, q_pl)): halo exchange then the gradient
    (kernels/oprtgradient.py:45-88); g of shape (3, lall, kall, g, g)"""

    @staticmethod
    def forward(ctx, core, q, q_pl):
        q, q_pl = _c(q), _c(q_pl)
        g = torch.empty((3,) + core.field_shape, dtype=torch.float64, device=q.device)
        g_pl = torch.empty((3,) + core.field_shape_pl, dtype=torch.float64, device=q.device)
        core.gradient(q, q_pl, g, g_pl)
        ctx.core = core
        return g, g_pl

    @staticmethod
    def backward(ctx, gg, gg_pl):
        core = ctx.core
        gg = torch.zeros((3,) + core.field_shape, dtype=torch.float64, device="cuda") if gg is None else _c(gg)
        gg_pl = (torch.zeros((3,) + core.field_shape_pl, dtype=torch.float64, device="cuda") if gg_pl is None
                 else _c(gg_pl))
        gq = torch.empty(core.field_shape, dtype=torch.float64, device=gg.device)
        gq_pl = torch.empty(core.field_shape_pl, dtype=torch.float64, device=gg.device)
        core.gradient(gq, gq_pl, gg, gg_pl, transpose=True)
        return None, gq, gq_pl

    @staticmethod
    def jvp(ctx, _core, dq, dq_pl):
        return Gradient.forward(ctx, ctx.core, dq, dq_pl)


class Diffusion(torch.autograd.Function):
    """(y, y_pl) = Dk(C(s, s_pl)): halo exchange then the kh-weighted
    diffusion of the hyperdiffusion's scalar pass (kernels/oprtdiffusion.py);
    bilinear in s and the coefficient field (kh, kh_pl): the s cotangent is
    the transposed operator, the kh cotangent ``nc_diffusion_kh``"""

    @staticmethod
    def forward(ctx, core, s, s_pl, kh, kh_pl):
        s, s_pl, kh, kh_pl = _c(s), _c(s_pl), _c(kh), _c(kh_pl)
        y, y_pl = torch.empty_like(s), torch.empty_like(s_pl)
        core.diffusion(kh, kh_pl, s, s_pl, y, y_pl)
        ctx.core = core
        ctx.save_for_backward(s, s_pl, kh, kh_pl)
        ctx.save_for_forward(s, s_pl, kh, kh_pl)
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        core = ctx.core
        s, s_pl, kh, kh_pl = ctx.saved_tensors
        gy = torch.zeros_like(kh) if gy is None else _c(gy)
        gy_pl = torch.zeros_like(kh_pl) if gy_pl is None else _c(gy_pl)
        g = g_pl = gk = gk_pl = None
        if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
            g, g_pl = torch.empty_like(gy), torch.empty_like(gy_pl)
            core.diffusion(kh, kh_pl, g, g_pl, gy, gy_pl, transpose=True)
        if ctx.needs_input_grad[3] or ctx.needs_input_grad[4]:
            gk, gk_pl = torch.empty_like(gy), torch.empty_like(gy_pl)
            core.diffusion_kh(s, s_pl, gy, gy_pl, gk, gk_pl)
        return None, g, g_pl, gk, gk_pl

    @staticmethod
    def jvp(ctx, _core, ds, ds_pl, dkh, dkh_pl):
        core = ctx.core
        s, s_pl, kh, kh_pl = ctx.saved_tensors
        y, y_pl = torch.zeros_like(s), torch.zeros_like(s_pl)
        t, t_pl = torch.empty_like(s), torch.empty_like(s_pl)
        if ds is not None or ds_pl is not None:
            ds = torch.zeros_like(s) if ds is None else _c(ds)
            ds_pl = torch.zeros_like(s_pl) if ds_pl is None else _c(ds_pl)
            core.diffusion(kh, kh_pl, ds, ds_pl, t, t_pl)
            y, y_pl = y + t, y_pl + t_pl
        if dkh is not None or dkh_pl is not None:
            dkh = torch.zeros_like(kh) if dkh is None else _c(dkh)
            dkh_pl = torch.zeros_like(kh_pl) if dkh_pl is None else _c(dkh_pl)
            core.diffusion(dkh, dkh_pl, s, s_pl, t, t_pl)
            y, y_pl = y + t, y_pl + t_pl
        return y, y_pl


class Exchange(torch.autograd.Function):
    """(y, y_pl) = C(x, x_pl): the halo exchange (share/mod_comm.py:1563-1644)
    of one field or of (nf,) stacked fields, out of place; linear"""

    @staticmethod
    def forward(ctx, core, x, x_pl):
        y, y_pl = x.detach().clone(memory_format=torch.contiguous_format), \
            x_pl.detach().clone(memory_format=torch.contiguous_format)
        core.exchange(y, y_pl)
        ctx.core = core
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        g, g_pl = gy.clone(memory_format=torch.contiguous_format), gy_pl.clone(memory_format=torch.contiguous_format)
        ctx.core.exchange(g, g_pl, transpose=True)
        return None, g, g_pl

    @staticmethod
    def jvp(ctx, _core, dx, dx_pl):
        y, y_pl = dx.clone(memory_format=torch.contiguous_format), dx_pl.clone(memory_format=torch.contiguous_format)
        ctx.core.exchange(y, y_pl)
        return y, y_pl


def exchange(core, x, x_pl):
    return Exchange.apply(core, x, x_pl)


def diffusion(core, s, s_pl, kh, kh_pl):
    return Diffusion.apply(core, s, s_pl, kh, kh_pl)


class _DivDamp(torch.autograd.Function):
    """(y, y_pl) = D(C(v, v_pl)): halo exchange then one of the divergence
    damping's operators (three = True: the 3-D OPRT3D_divdamp of the four
    momenta, kernels/oprt3ddivdamp.py; else the 2-D OPRT_divdamp of three
    components, kernels/oprtdivdamp.py); linear in v"""

    @staticmethod
    def forward(ctx, core, three, v, v_pl):
        op = core.divdamp3d if three else core.divdamp2d
        y = torch.empty((3,) + tuple(v.shape[1:]), dtype=v.dtype, device=v.device)
        y_pl = torch.empty((3,) + tuple(v_pl.shape[1:]), dtype=v_pl.dtype, device=v_pl.device)
        op(_c(v), _c(v_pl), y, y_pl)
        ctx.core, ctx.three, ctx.shapes = core, three, (tuple(v.shape), tuple(v_pl.shape))
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        op = ctx.core.divdamp3d if ctx.three else ctx.core.divdamp2d
        sv, sv_pl = ctx.shapes
        dev = (gy if gy is not None else gy_pl).device
        z = lambda shp: torch.zeros(shp, dtype=torch.float64, device=dev)
        gy = z((3,) + sv[1:]) if gy is None else _c(gy)
        gy_pl = z((3,) + sv_pl[1:]) if gy_pl is None else _c(gy_pl)
        g, g_pl = z(sv), z(sv_pl)
        op(g, g_pl, gy, gy_pl, transpose=True)
        return None, None, g, g_pl

    @staticmethod
    def jvp(ctx, _core, _three, dv, dv_pl):
        return _DivDamp.forward(ctx, ctx.core, ctx.three, dv, dv_pl)


def divdamp3d(core, v, v_pl):
    """the 3-D divergence damping operator of the four momenta (4, ...) -> (3, ...)"""
    return _DivDamp.apply(core, True, v, v_pl)


def divdamp2d(core, v, v_pl):
    """the 2-D divergence damping operator of three components (3, ...) -> (3, ...)"""
    return _DivDamp.apply(core, False, v, v_pl)


def divergence_damping(core, v, v_pl, fixed: dict):
    """The divergence damping tendency of the large step (mod_numfilter.py:
    2032-2268, lap_order 2): the 3-D operator on the four momenta
    v = (rhogvx, rhogvy, rhogvz, rhogw) (4, lall, kall, g, g) and v_pl
    (4, 6, kall, LP), the exchange, the 2-D operator on its negation, the
    coefficient, the result made horizontal (kernels/horizontalizevec.py;
    the pole rows with the per-term division of its pole form).  Returns
    (gd, gd_pl) of shape (3, ...), differentiable through the operators'
    hand-written transposes."""
    r, coef = fixed["rscale"], fixed["divdamp_coef"]
    d, d_pl = divdamp3d(core, v, v_pl)
    o, o_pl = divdamp2d(core, -d, -d_pl)
    out = []
    for pole, t in ((0, o), (1, o_pl)):
        fx, fy, fz = coef * t[0], coef * t[1], coef * t[2]
        gx = fixed["gx_pl"] if pole else fixed["gx"]
        if pole:
            prd = fx * gx[0] / r + fy * gx[1] / r + fz * gx[2] / r
        else:
            prd = (fx * gx[0] + fy * gx[1] + fz * gx[2]) / r
        out.append(torch.stack([fx - prd * gx[0] / r, fy - prd * gx[1] / r, fz - prd * gx[2] / r]))
    return out[0], out[1]


def hdiff_setup(geo: dict, device="cuda") -> dict:
    """the fixed inputs of ``hyperdiffusion`` and ``divergence_damping`` from a
    setup dict (DIRECT Kh): Kh, divdamp_coef, CVdry, hdiff_fact_rho, the C2W
    weights (device layout, two components) and the unit-radius position
    vectors GRD_x / rscale of the regional points and pole points"""
    sc = lambda k: float(np.asarray(geo[k]).reshape(-1)[0])
    c2w = np.asarray(geo["VMTR_C2Wfact"], np.float64)
    c2w_pl = np.asarray(geo["VMTR_C2Wfact_pl"], np.float64)
    gx = np.asarray(geo["GRD_x"], np.float64)[:, :, 0, :, :]               # (i, j, l, 3)
    gx_pl = np.asarray(geo["GRD_x_pl"], np.float64)[:, 0, :, :]            # (g, l, 3)
    f = {"Kh": sc("Kh_coef"), "divdamp_coef": sc("divdamp_coef"), "CVdry": sc("CVdry"),
         "hfr": sc("hdiff_fact_rho"), "rscale": sc("rscale"), "kmin": int(sc("kmin"))}
    f["c2w"] = torch.stack([to_device_layout(c2w[..., c], device) for c in range(2)])
    f["c2w_pl"] = torch.as_tensor(np.ascontiguousarray(np.moveaxis(c2w_pl, -1, 0))).to(device)
    f["gx"] = torch.as_tensor(np.ascontiguousarray(np.moveaxis(gx, (2, 1, 0, 3), (1, 2, 3, 0))))[:, :, None].to(device)
    f["gx_pl"] = torch.as_tensor(np.ascontiguousarray(np.moveaxis(gx_pl, -1, 0)))[:, :, None, :].to(device)
    return f


def hyperdiffusion(core, x, x_pl, rhog, rhog_pl, fixed: dict):
    """The hyperdiffusion tendency of the large step (mod_numfilter.py:845-1469,
    DIRECT Kh, lap_order 2; _hdiff_tendency_host :1519-1578 and the final
    horizontalize) as a differentiable function of the six fields
    x = (vx, vy, vz, w, tem - tem_bs, rho - rho_bs) (6, lall, kall, g, g) and
    x_pl (6, 6, kall, LP), at a fixed density (rhog, rhog_pl): two
    Laplacian passes (the second a kh-weighted diffusion for the two scalars),
    the tendencies scaled by Kh and rhog (rhog at half levels for w), the
    momentum made horizontal.  Returns (f, f_pl) in prognostic order (RHOG,
    RHOGVX, RHOGVY, RHOGVZ, RHOGW, RHOGE) on interior cells and the pole
    point; the adjoint follows from the operators' hand-written transposes."""
    Kh, r = fixed["Kh"], fixed["rscale"]
    rhog, rhog_pl = rhog.detach(), rhog_pl.detach()
    v1 = [laplacian(core, x[n], x_pl[n]) for n in range(6)]
    v1 = [(-a, -b) for a, b in v1]
    v2 = [laplacian(core, *v1[n]) for n in range(4)]
    v2.append(diffusion(core, *v1[4], rhog * fixed["CVdry"] * Kh, rhog_pl * fixed["CVdry"] * Kh))
    v2.append(diffusion(core, *v1[5], rhog * fixed["hfr"] * Kh, rhog_pl * fixed["hfr"] * Kh))
    v2 = [(-a, -b) for a, b in v2]
    kmin = fixed["kmin"]
    out = []
    for pole in (0, 1):
        rg = rhog_pl if pole else rhog
        c2w = fixed["c2w_pl"] if pole else fixed["c2w"]
        kax = 1   # the level axis of (lall, kall, g, g) and of (6, kall, LP)
        below = torch.zeros_like(rg)
        below.narrow(kax, 1, rg.shape[kax] - 1).copy_(rg.narrow(kax, 0, rg.shape[kax] - 1))
        rgh = c2w[0] * rg + c2w[1] * below
        rgh.narrow(kax, 0, kmin).zero_()
        v = [t[pole] for t in v2]
        fx, fy, fz = (-(v[n] * Kh) * rg for n in range(3))
        fw = -(v[3] * Kh) * rgh
        gx = fixed["gx_pl"] if pole else fixed["gx"]
        prd = (fx * gx[0] + fy * gx[1] + fz * gx[2]) / r
        fx, fy, fz = fx - prd * gx[0] / r, fy - prd * gx[1] / r, fz - prd * gx[2] / r
        out.append(torch.stack([-v[5], fx, fy, fz, fw, -v[4]]))
    return out[0], out[1]


def divergence(core, v, v_pl):
    return Divergence.apply(core, v, v_pl)


def gradient(core, q, q_pl):
    return Gradient.apply(core, q, q_pl)


class TracerStep(torch.autograd.Function):
    """(y, y_pl) = T(x, x_pl): one tracer advection step with the winds and
    densities of the handle's last step (they must still be the ones the
    forward used when the backward runs)"""

    @staticmethod
    def forward(ctx, core, x, x_pl):
        x, x_pl = _c(x), _c(x_pl)
        y, y_pl = torch.empty_like(x), torch.empty_like(x_pl)
        core.trc_step_lin(0, x, x_pl, None, None, y, y_pl)
        ctx.core = core
        ctx.save_for_backward(x, x_pl)
        ctx.save_for_forward(x, x_pl)
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        x, x_pl = ctx.saved_tensors
        gy = torch.zeros_like(x) if gy is None else _c(gy)
        gy_pl = torch.zeros_like(x_pl) if gy_pl is None else _c(gy_pl)
        g, g_pl = torch.empty_like(x), torch.empty_like(x_pl)
        ctx.core.trc_step_lin(2, x, x_pl, gy, gy_pl, g, g_pl)
        return None, g, g_pl

    @staticmethod
    def jvp(ctx, _core, dx, dx_pl):
        x, x_pl = ctx.saved_tensors
        dx = torch.zeros_like(x) if dx is None else _c(dx)
        dx_pl = torch.zeros_like(x_pl) if dx_pl is None else _c(dx_pl)
        y, y_pl = torch.empty_like(x), torch.empty_like(x_pl)
        ctx.core.trc_step_lin(1, x, x_pl, dx, dx_pl, y, y_pl)
        return y, y_pl


def tracer_step(core, x, x_pl):
    return TracerStep.apply(core, x, x_pl)


def _tracers(prg, prg_pl, nq):
    """device-layout tracer masses (nq, lall, kall, g, g) / (nq, 6, kall, LP)
    of a reference-layout state tensor"""
    x = prg[..., 6:6 + nq].permute(4, 3, 2, 1, 0).contiguous()
    x_pl = prg_pl[..., 6:6 + nq].permute(3, 0, 1, 2).contiguous()
    return x, x_pl


def _with_tracers(prg, prg_pl, x, x_pl):
    s, sp = prg.clone(), prg_pl.clone()
    nq = x.shape[0]
    s[..., 6:6 + nq] = x.permute(4, 3, 2, 1, 0)
    sp[..., 6:6 + nq] = x_pl.permute(1, 2, 3, 0)
    return s.contiguous(), sp.contiguous()


class _TracerRun(torch.autograd.Function):
    @staticmethod
    def forward(ctx, model, nsteps, x, x_pl):
        core = model.core
        s, sp = _with_tracers(model.prg, model.prg_pl, x.detach(), x_pl.detach())
        model.clock(0)
        core.upload_tensor(s, sp)
        stored = {}
        for n in range(nsteps):
            if n % model.every == 0:
                stored[n] = core.download_tensor()
            core.step(1)
        y, y_pl = _tracers(*core.download_tensor(), x.shape[0])
        ctx.model, ctx.nsteps, ctx.stored = model, nsteps, stored
        return y, y_pl

    @staticmethod
    def backward(ctx, gy, gy_pl):
        model, core, nq = ctx.model, ctx.model.core, ctx.model.nq
        g = torch.zeros((nq,) + core.field_shape, dtype=torch.float64, device="cuda") if gy is None else gy.clone()
        g_pl = (torch.zeros((nq,) + core.field_shape_pl, dtype=torch.float64, device="cuda") if gy_pl is None
                else gy_pl.clone())
        out, out_pl = torch.empty_like(g[0]), torch.empty_like(g_pl[0])
        starts = sorted(ctx.stored)
        for seg, n0 in reversed(list(enumerate(starts))):
            n1 = starts[seg + 1] if seg + 1 < len(starts) else ctx.nsteps
            states = [ctx.stored[n0]]                      # the segment's per-step states, re-run
            model.clock(n0)
            core.upload_tensor(*states[0])
            for _ in range(n0, n1 - 1):
                core.step(1)
                states.append(core.download_tensor())
            for m, (s, sp) in reversed(list(enumerate(states))):
                model.clock(n0 + m)
                core.upload_tensor(s, sp)
                model.coefficients()                       # the step's winds and densities onto the handle
                x, x_pl = _tracers(s, sp, nq)
                for iq in range(nq):
                    core.trc_step_lin(2, x[iq], x_pl[iq], g[iq], g_pl[iq], out, out_pl)
                    g[iq].copy_(out)
                    g_pl[iq].copy_(out_pl)
            del states
        return None, None, g, g_pl


class TracerTransport:
    """Runs of the handle's own steps from the state (prg, prg_pl) (device
    tensors, reference layout) as a differentiable function of the initial
    tracer masses of its nq tracers: ``run(x, x_pl, nsteps)`` with x of shape
    (nq, lall, kall, gall_1d, gall_1d) and x_pl (nq, 6, kall, LP) returns the
    tracer masses after nsteps steps, the full state stored every
    ``checkpoint_every`` steps for the backward pass"""

    def __init__(self, core, prg, prg_pl, checkpoint_every: int = 1, time0: float = 0.0):
        self.core, self.prg, self.prg_pl = core, prg, prg_pl
        self.nq = prg.shape[-1] - 6
        self.every = max(1, int(checkpoint_every))
        self.time0 = float(time0)

    def coefficients(self):
        """the winds and densities of the step from the uploaded state onto
        the handle: the offline advection reads them straight from the state
        (nc_trc_prepare); otherwise the step is re-run"""
        if self.core.trcadv:
            self.core.trc_prepare()
        else:
            self.core.step(1)

    def directional(self, x, x_pl, d, d_pl, nsteps: int):
        """the run and its tangent-linear along (d, d_pl): the tracer masses
        after nsteps steps and their derivative along the direction, each
        step's tangent-linear applied while the step's winds are on the
        handle"""
        core = self.core
        s, sp = _with_tracers(self.prg, self.prg_pl, x, x_pl)
        self.clock(0)
        core.upload_tensor(s, sp)
        d, d_pl = d.clone(), d_pl.clone()
        out, out_pl = torch.empty_like(d[0]), torch.empty_like(d_pl[0])
        for _ in range(nsteps):
            xs, xs_pl = _tracers(*core.download_tensor(), self.nq)
            core.step(1)
            for iq in range(self.nq):
                core.trc_step_lin(1, xs[iq], xs_pl[iq], d[iq], d_pl[iq], out, out_pl)
                d[iq].copy_(out)
                d_pl[iq].copy_(out_pl)
        y, y_pl = _tracers(*core.download_tensor(), self.nq)
        return (y, y_pl), (d, d_pl)

    def clock(self, n: int):
        """an offline-advection handle's prescribed-wind time at step n"""
        if self.core.trcadv:
            self.core.set_time(self.time0 + n * float(_scalar(self.core._tab["dtl"])))

    def initial_tracers(self):
        return _tracers(self.prg, self.prg_pl, self.nq)

    def run(self, x, x_pl, nsteps: int):
        return _TracerRun.apply(self, nsteps, x, x_pl)


def vertical_solve(core, Mc, Mu, Ml, b, pole=False):
    return VerticalSolve.apply(core, pole, Mc, Mu, Ml, b)


# ---------------------------------------------------------------------------
# the HEVI vertical implicit step: the matrix of kernels/vimatrix.py:67-164 and
# the source assembly + solve of kernels/virhowsolver.py:42-172, as torch
# expressions in the reference's operation order around the hand-written
# tridiagonal solve (VerticalSolve); differentiable in every field argument.
# Fields in device layout: the level axis is axis 1 for regional and pole
# tensors alike.
# ---------------------------------------------------------------------------
def hevi_metrics(geo: dict, device="cuda") -> dict:
    """device tensors of the metrics and vertical factors the HEVI matrix and
    solve read (VMTR_* regional and pole, GRD_* 1-D), and the constants"""
    m = {}
    for k in ("RGSGAM2", "GAM2H", "RGAMH", "RGSQRTH", "RGAM", "RGSGAM2H", "GSGAM2H"):
        m[k] = to_device_layout(geo["VMTR_" + k], device)
        m[k + "_pl"] = torch.as_tensor(np.ascontiguousarray(geo["VMTR_" + k + "_pl"], np.float64)).to(device)
    for k in ("rdgz", "rdgzh", "afact", "bfact", "cfact", "dfact"):
        m[k] = torch.as_tensor(np.asarray(geo["GRD_" + k], np.float64)).to(device)
    for k in ("GRAV", "CVdry", "Rdry", "alpha"):
        m[k] = float(_scalar(geo[k]))
    m["kmin"], m["kmax"] = int(_scalar(geo["kmin"])), int(_scalar(geo["kmax"]))
    return m


def _lev(v, sl, nd):
    """a 1-D level vector sliced and shaped to broadcast along axis 1"""
    shape = [1] * nd
    shape[1] = -1
    return v[sl].view(shape)


def _pad_levels(x, kmin, kmax, kall):
    """interior rows kmin+1..kmax -> all kall levels, zero elsewhere"""
    lo = x.new_zeros(x.shape[:1] + (kmin + 1,) + x.shape[2:])
    hi = x.new_zeros(x.shape[:1] + (kall - kmax - 1,) + x.shape[2:])
    return torch.cat([lo, x, hi], dim=1)


def hevi_matrix(m: dict, eth_h, gz, dt: float, pole: bool = False):
    """(Mc, Mu, Ml) on all levels (rows kmin+1..kmax, zero elsewhere) from the
    half-level enthalpy eth_h and gz (kernels/vimatrix.py:67-164)"""
    sfx = "_pl" if pole else ""
    kmin, kmax, nd, kall = m["kmin"], m["kmax"], eth_h.dim(), eth_h.shape[1]
    ks, ksp, ksm = slice(kmin + 1, kmax + 1), slice(kmin + 2, kmax + 2), slice(kmin, kmax)
    K = lambda a, sl: a[:, sl]
    RGSGAM2, GAM2H, RGAMH, RGSQRTH = (m[k + sfx] for k in ("RGSGAM2", "GAM2H", "RGAMH", "RGSQRTH"))
    GCVovR = m["GRAV"] * m["CVdry"] / m["Rdry"]
    ACVovRt2 = m["alpha"] * m["CVdry"] / m["Rdry"] / (dt * dt)
    rg, rgm = _lev(m["rdgz"], ks, nd), _lev(m["rdgz"], ksm, nd)
    Ca = (K(RGSGAM2, ks) * rg + K(RGSGAM2, ksm) * rgm) * K(GAM2H, ks)
    Cb = (m["dfact"][ks] - m["cfact"][ksm]).view([1, -1] + [1] * (nd - 2))
    Cu1 = K(RGSGAM2, ks) * rg * K(GAM2H, ksp)
    Cu2 = K(GAM2H, ksp) * K(RGAMH, ks) ** 2 * GCVovR
    Cl1 = K(RGSGAM2, ks) * rg * K(GAM2H, ksm)
    Cl2 = K(GAM2H, ksm) * K(RGAMH, ks) ** 2 * GCVovR
    rgh, cf, dfm = _lev(m["rdgzh"], ks, nd), _lev(m["cfact"], ks, nd), _lev(m["dfact"], ksm, nd)
    Mc = ACVovRt2 / K(RGSQRTH, ks) + rgh * (Ca * K(eth_h, ks) - Cb * (K(gz, ks) + GCVovR))
    Mu = -rgh * (Cu1 * K(eth_h, ksp) + cf * (K(gz, ksp) + Cu2))
    Ml = -rgh * (Cl1 * K(eth_h, ksm) - dfm * (K(gz, ksm) + Cl2))
    return tuple(_pad_levels(x, kmin, kmax, kall).contiguous() for x in (Mc, Mu, Ml))


def hevi_solve(core, m: dict, rhogw, rhogw0, preg0, rhog0, Srho, Sw, Spre, Mc, Mu, Ml, dt: float,
               pole: bool = False):
    """the new rhogw of the vertical implicit step (kernels/virhowsolver.py:
    42-172): source assembly on rows kmin+1..kmax, the boundary rows of rhogw
    (kmin, kmax+1) moved into the sources, the tridiagonal solve, the result
    scaled by GSGAM2H; levels outside kmin..kmax+1 keep rhogw"""
    sfx = "_pl" if pole else ""
    kmin, kmax, nd, kall = m["kmin"], m["kmax"], rhogw.dim(), rhogw.shape[1]
    ks, ksm = slice(kmin + 1, kmax + 1), slice(kmin, kmax)
    K = lambda a, sl: a[:, sl]
    RGAMH, RGSGAM2, RGAM, RGSGAM2H, GSGAM2H = (m[k + sfx] for k in ("RGAMH", "RGSGAM2", "RGAM", "RGSGAM2H",
                                                                      "GSGAM2H"))
    CVovRt2 = m["CVdry"] / m["Rdry"] / (dt * dt)
    rgh, af, bf = _lev(m["rdgzh"], ks, nd), _lev(m["afact"], ks, nd), _lev(m["bfact"], ks, nd)
    Sall = ((K(rhogw0, ks) * m["alpha"] + dt * K(Sw, ks)) * K(RGAMH, ks) ** 2
            - ((K(preg0, ks) + dt * K(Spre, ks)) * K(RGSGAM2, ks)
               - (K(preg0, ksm) + dt * K(Spre, ksm)) * K(RGSGAM2, ksm)) * dt * rgh
            - ((K(rhog0, ks) + dt * K(Srho, ks)) * K(RGAM, ks) ** 2 * af
               + (K(rhog0, ksm) + dt * K(Srho, ksm)) * K(RGAM, ksm) ** 2 * bf) * dt * m["GRAV"]
            ) * CVovRt2
    rw_kmin = rhogw[:, kmin] * RGSGAM2H[:, kmin]
    rw_kmaxp1 = rhogw[:, kmax + 1] * RGSGAM2H[:, kmax + 1]
    rows = list(Sall.unbind(1))
    rows[0] = rows[0] - Ml[:, kmin + 1] * rw_kmin
    rows[-1] = rows[-1] - Mu[:, kmax] * rw_kmaxp1
    b = _pad_levels(torch.stack(rows, 1), kmin, kmax, kall).contiguous()
    x = VerticalSolve.apply(core, pole, Mc, Mu, Ml, b)
    return torch.cat([rhogw[:, :kmin], (rw_kmin * GSGAM2H[:, kmin]).unsqueeze(1), K(x, ks) * K(GSGAM2H, ks),
                      (rw_kmaxp1 * GSGAM2H[:, kmax + 1]).unsqueeze(1), rhogw[:, kmax + 2:]], dim=1)


def vertical_advection(core, rhogq, den, flx_v, frhog, dt, bcoef=0.0, clamp=True, pole=False):
    return VerticalAdvection.apply(core, pole, rhogq, den, flx_v, frhog, dt, bcoef, clamp)


def laplacian(core, q, q_pl):
    return Laplacian.apply(core, q, q_pl)


class ColumnTransport:
    """A tracer model built from the differentiable operators: each step is
    one vertical advection step (limiter, clamp) of the regional and pole
    columns, then horizontal diffusion rhogq += kappa * L(C(rhogq)).

    ``fields``: dict of device-layout tensors den, flx_v, frhog and their
    ``_pl`` pole counterparts (held fixed); ``dt`` the advection step."""

    def __init__(self, core, fields: dict, dt: float, kappa: float, clamp: bool = True):
        self.core, self.f, self.dt, self.kappa, self.clamp = core, fields, dt, kappa, clamp

    def step(self, q, q_pl):
        f, c = self.f, self.core
        q = vertical_advection(c, q, f["den"], f["flx_v"], f["frhog"], self.dt, 0.0, self.clamp)
        q_pl = vertical_advection(c, q_pl, f["den_pl"], f["flx_v_pl"], f["frhog_pl"], self.dt, 0.0, self.clamp,
                                  pole=True)
        y, y_pl = laplacian(c, q, q_pl)
        return q + self.kappa * y, q_pl + self.kappa * y_pl

    def run(self, q, q_pl, nsteps: int, checkpoint: bool = False):
        for _ in range(nsteps):
            if checkpoint:
                q, q_pl = torch.utils.checkpoint.checkpoint(self.step, q, q_pl, use_reentrant=False)
            else:
                q, q_pl = self.step(q, q_pl)
        return q, q_pl

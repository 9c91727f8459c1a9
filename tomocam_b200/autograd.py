"""torch.autograd forms of the MBIR path.

* ``Radon``: forward projection; its backward is the hand-written adjoint
  (back-projection without the ramp, ``tc_iradon``), so <A x, y> = <x, A^T y>
  holds to rounding.
* ``MBIRObjective``: F(x) = 1/2 ||A x - y||^2 + beta U(x; sigma, p), with the
  data term in the reference's Toeplitz form 1/2 (x.Hx - 2 x.A^T y + ||y||^2)
  (src/error2.cpp:41-63) and U the qGGMRF potential whose gradient is the
  reference's clamped 26-neighbour stencil (src/gpu/cuTV2.cu:33-76).  Its
  backward is the hand-written gradient kernels: dF/dx = H x - A^T y +
  beta grad U (tc_toeplitz_grad + tc_qggmrf_grad, src/mbir2.cpp:122-129),
  dF/dbeta = U, dF/dsigma = beta dU/dsigma (tc_qggmrf_value).
* ``MBIRGrad``: g(x) = H x - A^T y + beta grad U(x), differentiable in x,
  A^T y, beta and sigma; its backward uses H (symmetric) and the prior's
  Hessian-vector product (tc_qggmrf_hvp).
* ``unrolled_mbir``: K fixed-step iterations built from ``MBIRGrad``,
  optionally activation-checkpointed per iteration, differentiable with
  respect to beta, sigma, the initial image and A^T y.

All tensors are float32 CUDA tensors on the library's kernels; the scalar
parameters beta and sigma may be Python floats or 0-d tensors (their
gradients are returned in their dtype).  No CPU path exists.
"""
from __future__ import annotations

import math

import torch
from torch.utils.checkpoint import checkpoint

from .plan import Plan, qggmrf_grad, qggmrf_hvp, qggmrf_value


def _scalar(v) -> float:
    return float(v.detach().item()) if isinstance(v, torch.Tensor) else float(v)


def _like(v, value: float):
    """value as a 0-d tensor matching v's dtype/device (or float64 CPU)."""
    if isinstance(v, torch.Tensor):
        return torch.as_tensor(value, dtype=v.dtype, device=v.device)
    return None


# ---------------------------------------------------------------------------
class Radon(torch.autograd.Function):
    """y = A x on [S, N, N] -> [S, P, N]; backward x-grad = A^T dy."""

    @staticmethod
    def forward(ctx, x, plan: Plan):
        ctx.plan = plan
        return plan.radon(x.contiguous())

    @staticmethod
    def backward(ctx, gy):
        gx = ctx.plan.iradon(gy.contiguous(), ramp=False) if ctx.needs_input_grad[0] else None
        return gx, None


def radon(x, plan: Plan):
    return Radon.apply(x, plan)


# ---------------------------------------------------------------------------
class MBIRObjective(torch.autograd.Function):
    """Scalar F(x; beta, sigma) as a 0-d float64 tensor on x's device."""

    @staticmethod
    def forward(ctx, x, beta, sigma, plan: Plan, aty, sino_sq: float, p: float):
        b, s = _scalar(beta), _scalar(sigma)
        x = x.contiguous()
        g, xhx, xaty = plan.toeplitz_grad(x, aty.contiguous(), dots=True)
        u, du = qggmrf_value(x, s, p)
        if ctx.needs_input_grad[0]:
            qggmrf_grad(x, g, s, p, b)  # g = H x - A^T y + beta grad U
            ctx.save_for_backward(g)
        ctx.u, ctx.du, ctx.b = u, du, b
        ctx.beta_t, ctx.sigma_t = beta, sigma
        f = 0.5 * (xhx - 2.0 * xaty + float(sino_sq)) + b * u
        return torch.tensor(f, dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx, gf):
        gfv = float(gf.item())
        gx = gbeta = gsigma = None
        if ctx.needs_input_grad[0]:
            (g,) = ctx.saved_tensors
            gx = g * gfv
        if ctx.needs_input_grad[1]:
            gbeta = _like(ctx.beta_t, gfv * ctx.u)
        if ctx.needs_input_grad[2]:
            gsigma = _like(ctx.sigma_t, gfv * ctx.b * ctx.du)
        return gx, gbeta, gsigma, None, None, None, None


def mbir_objective(x, plan: Plan, aty, sino_sq: float, beta=1.0, sigma=1.0, p: float = 1.2):
    """F(x) = 1/2 ||A x - y||^2 + beta U(x; sigma, p) (0-d float64 tensor)."""
    return MBIRObjective.apply(x, beta, sigma, plan, aty, sino_sq, p)


# ---------------------------------------------------------------------------
class MBIRGrad(torch.autograd.Function):
    """g = H x - A^T y + beta grad U(x; sigma); vector-Jacobian products:
    x: H v + beta Hess U v;  A^T y: -v;  beta: v.grad U;  sigma: beta v.dgradU/dsigma."""

    @staticmethod
    def forward(ctx, x, aty, beta, sigma, plan: Plan, p: float):
        b, s = _scalar(beta), _scalar(sigma)
        x = x.contiguous()
        g = plan.toeplitz_grad(x, aty.contiguous())
        qggmrf_grad(x, g, s, p, b)
        ctx.save_for_backward(x)
        ctx.plan, ctx.p, ctx.b, ctx.s = plan, p, b, s
        ctx.beta_t, ctx.sigma_t = beta, sigma
        return g

    @staticmethod
    def backward(ctx, v):
        (x,) = ctx.saved_tensors
        v = v.contiguous()
        need_x, need_aty, need_b, need_s = ctx.needs_input_grad[:4]
        gx = gaty = gbeta = gsigma = None
        dots = need_b or need_s
        hp, vg, vgs = qggmrf_hvp(x, v, ctx.s, ctx.p, ctx.b, dots=dots)
        if need_x:
            gx = ctx.plan.toeplitz_grad(v)  # H v (H = A^T A is symmetric)
            gx.add_(hp)
        if need_aty:
            gaty = -v
        if need_b:
            gbeta = _like(ctx.beta_t, vg)
        if need_s:
            gsigma = _like(ctx.sigma_t, ctx.b * vgs)
        return gx, gaty, gbeta, gsigma, None, None


def mbir_grad(x, plan: Plan, aty, beta=1.0, sigma=1.0, p: float = 1.2):
    return MBIRGrad.apply(x, aty, beta, sigma, plan, p)


# ---------------------------------------------------------------------------
def unrolled_mbir(x0, plan: Plan, aty, num_iters: int, step: float, beta=1.0, sigma=1.0,
                  p: float = 1.2, nesterov: bool = False, checkpoint_every: int = 1):
    """x_K of K fixed-step iterations x <- y - step g(y).

    nesterov=False follows Optimizer::run2's accepted-step path
    (src/optimize.h:117-146), where x = sol after every accepted step so
    y = sol and the iteration is a gradient step; nesterov=True applies the
    FISTA extrapolation y = s + (t_k - 1)/t_{k+1} (s - s_prev).
    checkpoint_every > 0 recomputes each group of that many iterations in
    the backward pass instead of keeping its activations (0: keep all)."""
    step = float(step)

    def block(s, prev, t0, n):
        t = t0
        for _ in range(n):
            if nesterov:
                tn = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t))
                y = s + ((t - 1.0) / tn) * (s - prev)
                t = tn
            else:
                y = s
            prev = s
            s = y - step * MBIRGrad.apply(y, aty, beta, sigma, plan, p)
        return s, prev

    s, prev, t = x0, x0, 1.0
    k = 0
    group = checkpoint_every if checkpoint_every > 0 else num_iters
    while k < num_iters:
        n = min(group, num_iters - k)
        if checkpoint_every > 0 and torch.is_grad_enabled():
            s, prev = checkpoint(block, s, prev, t, n, use_reentrant=False)
        else:
            s, prev = block(s, prev, t, n)
        for _ in range(n):
            t = 0.5 * (1.0 + math.sqrt(1.0 + 4.0 * t * t)) if nesterov else t
        k += n
    return s

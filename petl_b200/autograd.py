"""torch.autograd.Function wrappers over the CUDA operators.

* ``project(f, geom)``: g = P f; its backward is the exact transpose P^T
  (the PETL_BP_ADJOINT backprojector), so gradients through the projector
  are exact to float rounding (inner-product test < 1e-6).
* ``backproject(g, geom)``: f = P^T g; its backward is P.
* ``poisson_nll(Pf, g)``: sum over Pf > 0 of (Pf - g log Pf), reduced in
  FP64 on the device; backward (1 - g/Pf) on those bins, 0 elsewhere.
* ``rd_penalty(f, delta, beta)`` and ``tv_penalty(f, delta, beta, p, nn)``:
  the relative-difference and Huber-TV penalties as the reference's cost
  kernels sum them (every neighbour pair from both sides;
  src/relative_differences.cu:107-173, src/total_variation.cu:434-586).  The
  reference gradient kernels return half the gradient of that sum
  (src/relative_differences.cu:13-28, src/total_variation.cu:588-660), so
  the backward is 2 x the hand-written gradient kernel.

Every wrapper accepts a leading batch dimension: a [B, Z, Y, X] volume (or
[B, v1, v0, u1, u0] planogram) is B independent problems on one geometry,
each reduced to its own value ([B] costs).  All tensors are CUDA float32
(costs are float64); there is no CPU path.
"""
import torch

from . import ops


def _each(t, nd):
    """Iterate the problems of a possibly batched tensor with nd problem dims."""
    if t.dim() == nd:
        return [t]
    if t.dim() == nd + 1:
        return list(t.unbind(0))
    raise ValueError(f"expected a tensor with {nd} or {nd + 1} dims, got shape {tuple(t.shape)}")


def _stack(parts, like, nd):
    return parts[0] if like.dim() == nd else torch.stack(parts)


class Project(torch.autograd.Function):
    """g = P f with backward P^T (exact adjoint)."""

    @staticmethod
    def forward(ctx, f, geom):
        ctx.geom = geom
        outs = [ops.project(geom, x.contiguous()) for x in _each(f, 3)]
        return _stack(outs, f, 3)

    @staticmethod
    def backward(ctx, grad_g):
        geom = ctx.geom
        outs = [ops.backproject(geom, y.contiguous(), mode="adjoint") for y in _each(grad_g, 4)]
        return _stack(outs, grad_g, 4), None


class Backproject(torch.autograd.Function):
    """f = P^T g (exact adjoint) with backward P."""

    @staticmethod
    def forward(ctx, g, geom):
        ctx.geom = geom
        outs = [ops.backproject(geom, y.contiguous(), mode="adjoint") for y in _each(g, 4)]
        return _stack(outs, g, 4)

    @staticmethod
    def backward(ctx, grad_f):
        geom = ctx.geom
        outs = [ops.project(geom, x.contiguous()) for x in _each(grad_f, 3)]
        return _stack(outs, grad_f, 3), None


class PoissonNLL(torch.autograd.Function):
    """sum over Pf > 0 of (Pf - g log Pf) per problem, FP64; g is data (no grad)."""

    @staticmethod
    def forward(ctx, Pf, g):
        ctx.save_for_backward(Pf, g)
        vals = [-ops.loglik(y.contiguous(), x.contiguous()) for x, y in zip(_each(Pf, 4), _each(g, 4))]
        return vals[0] if Pf.dim() == 4 else torch.stack(vals)

    @staticmethod
    def backward(ctx, grad_out):
        Pf, g = ctx.saved_tensors
        parts = []
        for i, (x, y) in enumerate(zip(_each(Pf, 4), _each(g, 4))):
            d = ops.poisson_grad_(x.contiguous().clone(), y.contiguous())
            s = grad_out if grad_out.dim() == 0 else grad_out[i]
            parts.append(d * s.to(d.dtype))
        return _stack(parts, Pf, 4), None


class RDPenalty(torch.autograd.Function):
    """Relative-difference penalty (26 neighbours), FP64 cost per problem."""

    @staticmethod
    def forward(ctx, f, delta, beta):
        ctx.save_for_backward(f)
        ctx.args = (float(delta), float(beta))
        vals = [ops.rd_cost(x.contiguous(), *ctx.args) for x in _each(f, 3)]
        return vals[0] if f.dim() == 3 else torch.stack(vals)

    @staticmethod
    def backward(ctx, grad_out):
        (f,) = ctx.saved_tensors
        parts = []
        for i, x in enumerate(_each(f, 3)):
            d = ops.rd_gradient(x.contiguous(), *ctx.args)
            s = grad_out if grad_out.dim() == 0 else grad_out[i]
            parts.append(d * (2.0 * s).to(d.dtype))
        return _stack(parts, f, 3), None, None


class TVPenalty(torch.autograd.Function):
    """Huber total variation (p-Huber, 6 or 26 neighbours), FP64 cost per problem."""

    @staticmethod
    def forward(ctx, f, delta, beta, p, num_neighbors):
        ctx.save_for_backward(f)
        ctx.args = (float(delta), float(beta), float(p), int(num_neighbors))
        vals = [ops.tv_cost(x.contiguous(), *ctx.args) for x in _each(f, 3)]
        return vals[0] if f.dim() == 3 else torch.stack(vals)

    @staticmethod
    def backward(ctx, grad_out):
        (f,) = ctx.saved_tensors
        parts = []
        for i, x in enumerate(_each(f, 3)):
            d = ops.tv_gradient(x.contiguous(), *ctx.args)
            s = grad_out if grad_out.dim() == 0 else grad_out[i]
            parts.append(d * (2.0 * s).to(d.dtype))
        return _stack(parts, f, 3), None, None, None, None


def project(f, geom):
    return Project.apply(f, geom)


def backproject(g, geom):
    return Backproject.apply(g, geom)


def poisson_nll(Pf, g):
    return PoissonNLL.apply(Pf, g)


def rd_penalty(f, delta=2.0, beta=0.01):
    return RDPenalty.apply(f, delta, beta)


def tv_penalty(f, delta=1e-4, beta=1.0, p=1.0, num_neighbors=26):
    return TVPenalty.apply(f, delta, beta, p, num_neighbors)


__all__ = ["Project", "Backproject", "PoissonNLL", "RDPenalty", "TVPenalty", "project", "backproject", "poisson_nll",
           "rd_penalty", "tv_penalty"]

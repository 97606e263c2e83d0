"""Differentiable penalized reconstruction on the autograd wrappers.

Objective per problem (one volume of a batch on a shared geometry):

    Phi(f) = sum_{Pf > 0} (Pf - g log Pf)          Poisson negative log-likelihood
           + RD(f; gamma, beta_rd)                 relative differences, 26 neighbours
           + TV(f; delta, beta_tv, p, neighbours)  Huber total variation

with the penalties summed as the reference's cost kernels sum them
(src/relative_differences.cu:107-173, src/total_variation.cu:434-586).  The
gradient comes from torch.autograd through petl_b200.autograd: the
projector's backward is its exact adjoint kernel, the penalties' backward the
hand-written gradient kernels.

``reconstruct`` runs EM-preconditioned gradient steps,
    d = -(f / P^T 1) * grad Phi(f),   f <- max(f + alpha d, 0),
with alpha from a backtracking (Armijo) line search whose objective values
are FP64 reductions on the device; the projection of d is computed once per
step, so the line search costs no further projections.

``fd_check`` compares the autograd gradient with central finite differences
of the FP64 objective at chosen voxels.
"""
import torch

from . import autograd as A
from . import ops


def objective(f, geom, g, rd=(2.0, 0.01), tv=(1e-4, 0.01, 1.0, 26), Pf=None):
    """Phi per problem ([B] float64, or 0-d for one volume)."""
    if Pf is None:
        Pf = A.project(f, geom)
    val = A.poisson_nll(Pf, g)
    if rd is not None:
        val = val + A.rd_penalty(f, *rd)
    if tv is not None:
        val = val + A.tv_penalty(f, *tv)
    return val


def gradient(f, geom, g, rd=(2.0, 0.01), tv=(1e-4, 0.01, 1.0, 26)):
    """(Phi, grad Phi) through autograd."""
    x = f.detach().requires_grad_(True)
    val = objective(x, geom, g, rd, tv)
    val.sum().backward()
    return val.detach(), x.grad.detach()


def fd_check(f, geom, g, voxels, h=1e-3, rd=(2.0, 0.01), tv=(1e-4, 0.01, 1.0, 26)):
    """Autograd gradient and central differences (Phi(f+h e) - Phi(f-h e)) / 2h
    at the flat voxel indices ``voxels`` of a single volume; both float64."""
    _, grad = gradient(f, geom, g, rd, tv)
    flat = f.detach().reshape(-1)
    fd = []
    with torch.no_grad():
        for i in voxels:
            i = int(i)
            old = float(flat[i])
            vals = []
            for s in (h, -h):
                flat[i] = old + s
                vals.append(float(objective(f.detach(), geom, g, rd, tv)))
            flat[i] = old
            fd.append((vals[0] - vals[1]) / (2.0 * h))
    return grad.reshape(-1)[torch.as_tensor(voxels, device=f.device)].double(), torch.tensor(fd, dtype=torch.float64)


def reconstruct(geom, g, iters=50, f0=None, rd=(2.0, 0.01), tv=(1e-4, 0.01, 1.0, 26), armijo=1e-4, max_backtrack=8):
    """EM-preconditioned gradient descent on Phi for a batch [B, ...] of data
    (or one planogram).  Returns (f, history of Phi per step as a [iters+1, B]
    float64 CPU tensor)."""
    batched = g.dim() == 5
    gb = g if batched else g.unsqueeze(0)
    B = gb.shape[0]
    dev = g.device
    ones = torch.ones(geom.shape, device=dev)
    sens = ops.backproject(geom, ones, mode="adjoint")
    sens[sens <= 0] = 1.0
    if f0 is None:
        # uniform image with the data's total counts
        scale = gb.reshape(B, -1).sum(1, dtype=torch.float64) / float(sens.double().sum())
        f = torch.ones((B,) + tuple(geom.vol_shape), device=dev) * scale.float().view(B, 1, 1, 1)
    else:
        f = (f0 if f0.dim() == 4 else f0.unsqueeze(0)).clone()
    hist = []
    for _ in range(iters):
        val, grad = gradient(f, geom, gb, rd, tv)
        hist.append(val.cpu())
        with torch.no_grad():
            d = -(f / sens) * grad
            Pf = A.project(f, geom)
            Pd = A.project(d, geom)
            for b in range(B):
                slope = float(ops.dot(grad[b], d[b]))  # directional derivative, FP64
                alpha = 1.0
                for _ in range(max_backtrack):
                    fa = torch.clamp(f[b] + alpha * d[b], min=0.0)
                    Pa = Pf[b] + alpha * Pd[b]
                    va = float(objective(fa, geom, gb[b], rd, tv, Pf=Pa))
                    if va <= float(val[b]) + armijo * alpha * slope:
                        break
                    alpha *= 0.5
                f[b] = torch.clamp(f[b] + alpha * d[b], min=0.0)
    val, _ = gradient(f, geom, gb, rd, tv)
    hist.append(val.cpu())
    out = f if batched else f[0]
    return out, torch.stack(hist)


__all__ = ["objective", "gradient", "fd_check", "reconstruct"]

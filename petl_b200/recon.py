"""Device-resident reconstruction drivers: MLEM, OSEM, one-step-late RD MLEM,
and penalized least squares by preconditioned conjugate gradient.

Every iteration stays on the GPU: the MLEM data ratio is computed inside the
forward projector (ops.project_ratio), the image update is one fused kernel,
and the log-likelihood and step-size reductions run in FP64 on the device.

* ``mlem`` follows the reference PETLserver.MLEM loop
  (src/petl_server.py:1534-1606): f starts at 1 (or is clipped at 0 when
  given), sensitivity = P^T 1 with zeros replaced by 1, d = P^T (g / P f),
  f *= d / sens, or with beta > 0 the one-step-late relative-difference
  update f *= d / max(0.1 sens, sens + grad R(f)).
* ``osem`` splits the views into S interleaved subsets (subset s holds
  iv0 = s, s+S, ...); with S = 1 it is ``mlem``.  The reference has no OSEM.
  A response R (planograms) makes the system model R P, as in the
  reference's MLEM once a response is set.
* ``rwls`` follows PETLserver.RWLS (src/petl_server.py:1691-1877): PCG with
  an optional SQS preconditioner 1/P^T W P 1, restarts every 50 iterations,
  step = <d,grad> / (<Pd, W Pd> + TV quadratic form), optional
  non-negativity.
"""
import torch

from . import ops
from .geometry import as_list


def _ones_like_list(gl):
    return [torch.ones_like(x) for x in gl]


def sensitivity(geoms, like, subset=None, mode="reference", response=None):
    """P^T 1 (src/petl_server.py:1257-1273), or P^T R with a response R,
    with zeros replaced by 1."""
    geoms = as_list(geoms)
    w = _ones_like_list(like) if response is None else as_list(response)
    s = ops.backproject(geoms, w, subset=subset, mode=mode)
    s[s == 0.0] = 1.0
    return s


def _response_masked(gl, response):
    """The data with zeros where the response is zero.  With a response R the
    reference's MLEM projects R P f and backprojects R (g / R P f)
    (src/petl_server.py:723-747 with include_response_with_projectors on
    during MLEM, src/petl_server.py:1566-1567); R (g / R P f) = g / P f
    wherever R != 0 and 0 elsewhere, so the iteration keeps the plain data
    ratio on this masked data and uses P^T R as its sensitivity."""
    return [torch.where(r != 0, x, torch.zeros_like(x)) for x, r in zip(gl, as_list(response))]


def _init_image(geoms, f, device):
    if f is None:
        return torch.ones(geoms[0].vol_shape, device=device, dtype=torch.float32)
    if not torch.any(f):
        f.fill_(1.0)
    else:
        f.clamp_(min=0.0)
    return f


def mlem(geoms, g, num_iter, f=None, delta=2.0, beta=0.0, sens=None, loglik_every=0, response=None):
    """MLEM / OSL-RD MLEM; returns (f, loglik history)."""
    return osem(geoms, g, num_iter, 1, f=f, delta=delta, beta=beta, sens=sens, loglik_every=loglik_every,
                response=response)


def osem(geoms, g, num_iter, num_subsets, f=None, delta=2.0, beta=0.0, sens=None, loglik_every=0,
         response=None):
    """OSEM with interleaved view subsets; returns (f, loglik history).

    ``sens`` may pass precomputed per-subset sensitivities (list of S
    volumes) so that repeated reconstructions on one geometry reuse them.
    ``response`` (planograms R) makes the system model R P, as the
    reference's MLEM does when a response is set."""
    single = not isinstance(geoms, (list, tuple))
    geoms = as_list(geoms)
    gl = as_list(g)
    device = gl[0].device
    f = _init_image(geoms, f, device)
    S = int(num_subsets)
    if response is not None:
        gl = _response_masked(gl, response)
    if sens is None:
        sens = [sensitivity(geoms, gl, subset=(s, S), response=response) for s in range(S)]
    ratio = [torch.empty_like(x) for x in gl]
    d = torch.empty_like(f)
    Df = torch.empty_like(f) if beta > 0.0 else None
    history = []
    for it in range(num_iter):
        for s in range(S):
            sub = (s, S)
            ops.project_ratio(geoms, f, gl, out=ratio, subset=sub)
            ops.backproject(geoms, ratio, f=d, subset=sub)
            if beta > 0.0:
                ops.rd_gradient(f, delta, beta, out=Df)
                ops.osl_update_(f, d, sens[s], Df)
            else:
                ops.mlem_update_(f, d, sens[s])
        if loglik_every and (it + 1) % loglik_every == 0:
            history.append(loglik(geoms, gl, f, response=response))
    del single
    return f, history


def osem_bf16(geom, g, num_iter, num_subsets, f=None, sens=None, image="fp32"):
    """OSEM with the planogram-sized arrays (measured data and data ratio) and
    the projector's volume input stored in bfloat16, footprints accumulated
    in FP32.  With image="fp32" (default) the image itself is kept in FP32
    and rounded to a bfloat16 copy for each forward projection, so bfloat16
    rounding never compounds through the multiplicative updates; with
    image="bf16" the image is stored and updated in bfloat16 as well.  One
    axis-aligned, equal-pitch geometry (the TMA path).  Returns the image
    (float32 or bfloat16)."""
    S = int(num_subsets)
    device = g.device
    if g.dtype != torch.bfloat16:
        raise ValueError("osem_bf16 expects bfloat16 data")
    if image not in ("fp32", "bf16"):
        raise ValueError("image must be 'fp32' or 'bf16'")
    if sens is None:
        ones = torch.ones(geom.shape, device=device, dtype=torch.bfloat16)
        sens = []
        for s in range(S):
            x = ops.backproject_bf16(geom, ones, subset=(s, S))
            x[x == 0.0] = 1.0
            sens.append(x)
    ratio = torch.empty_like(g)
    d = torch.empty(geom.vol_shape, device=device, dtype=torch.float32)
    if image == "bf16":
        if f is None:
            f = torch.ones(geom.vol_shape, device=device, dtype=torch.bfloat16)
        for _ in range(num_iter):
            for s in range(S):
                ops.project_ratio_bf16(geom, f, g, out=ratio, subset=(s, S))
                ops.backproject_bf16(geom, ratio, f=d, subset=(s, S))
                ops.mlem_update_bf16_(f, d, sens[s])
        return f
    if f is None:
        f = torch.ones(geom.vol_shape, device=device, dtype=torch.float32)
    f16 = torch.empty(geom.vol_shape, device=device, dtype=torch.bfloat16)
    for _ in range(num_iter):
        for s in range(S):
            ops.to_bf16(f, out=f16)
            ops.project_ratio_bf16(geom, f16, g, out=ratio, subset=(s, S))
            ops.backproject_bf16(geom, ratio, f=d, subset=(s, S))
            ops.mlem_update_(f, d, sens[s])
    return f


def loglik(geoms, g, f, response=None):
    """Poisson log-likelihood of f (FP64, device), under R P f with a
    response R."""
    geoms = as_list(geoms)
    gl = as_list(g)
    Pf = ops.project(geoms, f)
    Pf = as_list(Pf)
    if response is not None:
        for pi, r in zip(Pf, as_list(response)):
            ops.multiply_(pi, r)
    total = torch.zeros((), device=gl[0].device, dtype=torch.float64)
    for gi, pi in zip(gl, Pf):
        total = total + ops.loglik(gi, pi)
    return total


def auto_weights(gl):
    """The reference RWLS default weights 1 / max(gaussian(g, 3 bins), 7),
    per planogram, the Gaussian over (u1, u0) (src/petl_server.py:1739-1746)."""
    out = []
    for gi in as_list(gl):
        w = gi.clone()
        ops.gaussian_filter_(w.view(w.shape[0] * w.shape[1], w.shape[2], w.shape[3]), 3.0, 2)
        w.clamp_(min=7.0)
        ops.reciprocal_(w, 0.0)
        out.append(w)
    return out


def rwls(geoms, g, f, num_iter, delta=1.0, beta=0.0, W=None, preconditioner=None, nonnegativity=True, p=1.0,
         bp_mode="reference", response=None):
    """Regularized weighted least squares by PCG (PETLserver.RWLS,
    src/petl_server.py:1691-1877): restarts every 50 iterations, optional
    SQS preconditioner 1 / P^T W P 1, step <d, grad> / (<Pd, W Pd> + TV
    quadratic form), optional non-negativity.  W: planograms, "auto" for
    1 / max(gaussian(g, 3), 7) (src/petl_server.py:1739-1746), or None.
    ``response`` (planograms R) makes the model R P, as the reference's
    projectors with include_response_with_projectors."""
    geoms = as_list(geoms)
    gl = as_list(g)
    Rl = as_list(response) if response is not None else None
    restart = 50
    if isinstance(W, str) and W == "auto":
        W = auto_weights(gl)
    Wl = as_list(W) if W is not None else None

    def fwd(x, out=None):
        y = as_list(ops.project(geoms, x, out if out is None or len(out) > 1 else out[0]))
        if Rl is not None:
            for yi, r in zip(y, Rl):
                ops.multiply_(yi, r)
        return y

    def bwd(ys, out=None):
        if Rl is not None:
            ys = [y * r for y, r in zip(ys, Rl)]
        return ops.backproject(geoms, ys, f=out, mode=bp_mode)

    if torch.any(f):
        if nonnegativity:
            f.clamp_(min=0.0)
        Pf = fwd(f)
    else:
        Pf = [torch.zeros_like(x) for x in gl]
    resid = [p_ - g_ for p_, g_ in zip(Pf, gl)]
    grad = torch.empty_like(f)
    d = torch.zeros_like(f)
    grad_old = torch.zeros_like(f)
    Pd = [torch.empty_like(x) for x in gl]
    Q = None
    if preconditioner in (True, "SQS"):
        P1 = fwd(torch.ones_like(f))
        if Wl is not None:
            P1 = [a * w for a, w in zip(P1, Wl)]
        Q = bwd(P1)
        ops.reciprocal_(Q, 1.0)
    gog = 0.0
    for n in range(num_iter):
        WR = [r * w for r, w in zip(resid, Wl)] if Wl is not None else resid
        bwd(WR, out=grad)
        if beta > 0.0:
            grad += ops.tv_gradient(f, delta, beta, p)
        u = grad * Q if Q is not None else grad.clone()
        if n == 0 or n % restart == 0:
            d.copy_(u)
        else:
            gamma = (float(ops.dot(u, grad)) - float(ops.dot(u, grad_old))) / gog
            d.mul_(gamma).add_(u)
            if float(ops.dot(d, grad)) <= 0.0:
                d.copy_(u)
        gog = float(ops.dot(u, grad))
        grad_old.copy_(grad)
        Pd = fwd(d, Pd)
        num = float(ops.dot(d, grad))
        den = 0.0
        for pd, w in zip(Pd, Wl if Wl is not None else [None] * len(Pd)):
            den += float(ops.dot(pd, pd, w))
        if beta > 0.0:
            den += float(ops.tv_quadform(f, d, delta, beta, p))
        step = num / den if abs(den) > 1.0e-16 else 0.0
        if step <= 0.0:
            break
        f.add_(d, alpha=-step)
        if nonnegativity:
            f.clamp_(min=0.0)
            Pf = fwd(f)
            resid = [p_ - g_ for p_, g_ in zip(Pf, gl)]
        else:
            resid = [r - step * pd for r, pd in zip(resid, Pd)]
    return f

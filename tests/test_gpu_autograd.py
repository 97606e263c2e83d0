"""torch.autograd wrappers: the projector's backward is its exact adjoint, the
RD/TV penalties' backward is twice the hand-written gradient kernel (the
reference kernels return half the gradient of their cost sums), and the whole
penalized objective matches central finite differences (h = 1e-3) of its FP64
value.  The penalty gradients are also held against the reference's own
gradient outputs (tests/golden/regularizers.npz)."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

ARGS = (0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25)
VOL = (64, 64, 16, 2.0)
RD = (2.0, 0.01)          # gamma, beta (relative differences, 26 neighbours)
TV = (1e-4, 0.01, 1.0, 26)  # delta, beta, p, neighbours


def _problem(cuda, seed=0, counts=2e5, batch=None):
    import torch
    from petl_b200 import Geometry, ops
    G = Geometry(*ARGS, volume=VOL)
    rng = np.random.default_rng(seed)
    vols, data = [], []
    for b in range(batch or 1):
        f = ellipsoids(G.vol_shape, (VOL[3], VOL[3]), rng, 6) + 0.05
        ft = torch.from_numpy(f.astype(np.float32)).to(cuda)
        y = ops.project(G, ft)
        y = y * (counts / float(y.sum()))
        y = torch.poisson(y, generator=torch.Generator(device=cuda).manual_seed(seed + b))
        vols.append(ft)
        data.append(y)
    if batch is None:
        return G, vols[0], data[0]
    return G, torch.stack(vols), torch.stack(data)


def test_project_backward_is_the_adjoint(cuda):
    import torch
    from petl_b200 import autograd as A, ops
    G, f, _ = _problem(cuda)
    y = torch.rand(G.shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(1))
    x = f.clone().requires_grad_(True)
    (A.project(x, G) * y).sum().backward()
    want = ops.backproject(G, y, mode="adjoint")
    assert torch.equal(x.grad, want)
    # and the backprojector's backward is the projector
    z = y.clone().requires_grad_(True)
    (A.backproject(z, G) * f).sum().backward()
    assert torch.equal(z.grad, ops.project(G, f))


def test_penalty_gradients_against_reference(cuda):
    import torch
    from petl_b200 import autograd as A
    r = load_golden("regularizers.npz")
    f = torch.from_numpy(r["f_3d"]).to(cuda).requires_grad_(True)
    A.rd_penalty(f, 2.0, 0.01).backward()
    assert rel_l2(f.grad.cpu().numpy(), 2.0 * r["rd_grad_3d"]) < 1e-5
    for delta, p in ((0.05, 1.0), (0.3, 1.2)):
        x = torch.from_numpy(r["f_3d"]).to(cuda).requires_grad_(True)
        c = A.tv_penalty(x, delta, 0.7, p, 26)
        c.backward()
        assert abs(float(c.detach()) / r[f"tv_cost_3d_d{delta}_p{p}"] - 1) < 1e-5
        assert rel_l2(x.grad.cpu().numpy(), 2.0 * r[f"tv_grad_3d_d{delta}_p{p}"]) < 1e-5


def test_objective_gradient_matches_finite_differences(cuda):
    import torch
    from petl_b200 import penalized
    G, f, y = _problem(cuda)
    rng = np.random.default_rng(7)
    # interior voxels with activity, where the objective is smooth
    fz = f.cpu().numpy()
    cand = np.flatnonzero(fz.reshape(-1) > 0.2)
    vox = rng.choice(cand, 32, replace=False)
    got, fd = penalized.fd_check(f, G, y, vox, h=1e-3, rd=RD, tv=TV)
    got, fd = got.cpu().numpy(), fd.numpy()
    err = np.abs(got - fd) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    assert np.median(err) < 1e-3 and err.max() < 2e-2, (got[:8], fd[:8])


def test_batched_objective_equals_single(cuda):
    import torch
    from petl_b200 import penalized
    G, fb, yb = _problem(cuda, batch=2)
    vb = penalized.objective(fb, G, yb, RD, TV)
    for b in range(2):
        v = penalized.objective(fb[b], G, yb[b], RD, TV)
        assert abs(float(vb[b]) - float(v)) <= 1e-12 * abs(float(v))


def test_penalized_reconstruction_decreases_objective(cuda):
    import torch
    from petl_b200 import penalized
    G, fb, yb = _problem(cuda, batch=2)
    f, hist = penalized.reconstruct(G, yb, iters=8, rd=RD, tv=TV)
    assert f.shape == fb.shape and torch.isfinite(f).all() and (f >= 0).all()
    assert hist.shape == (9, 2)
    h = hist.numpy()
    assert (h[-1] < h[0]).all()
    assert (np.diff(h, axis=0) <= 1e-9 * np.abs(h[:-1])).mean() > 0.8

"""The shear-warp kernels (axis-aligned planograms, voxel pitch = bin pitch)
against the general kernels, the FP64 oracle and each other.

Both kernel families compute the same operator with different rounding, so
they agree to float accuracy (relative L2 < 1e-5); the shear forward and the
shear adjoint are exact transposes (inner-product test < 1e-6).
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

CASES = {
    # psi, D, L, H, T, v_m0, v_m1 ; volume
    "t2": ((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0)),
    "t1": ((0.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25), (128, 128, 32, 1.0)),
    # ragged sizes (not multiples of 32) and an off-centre volume
    "odd": ((0.0, 100.0, 50.0, 26.0, 1.5, 0.45, 0.2), (50, 58, 15, 1.5, 1.5, 3.0, -4.5, 1.5)),
}


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


def _setup(name, cuda, seed=0):
    from petl_b200 import Geometry
    args, vol = CASES[name]
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(seed)
    f = ellipsoids(G.vol_shape, (vol[3], vol[4] if len(vol) > 4 else vol[3]), rng, 8) + \
        0.1 * rng.random(G.vol_shape).astype(np.float32)
    return G, Go, f, rng


def _both(fn):
    """Run fn under the general kernels and under the default dispatch."""
    from petl_b200 import lib
    lib().petl_set_dispatch(1)
    try:
        a = fn()
    finally:
        lib().petl_set_dispatch(0)
    b = fn()
    return a, b


@pytest.mark.parametrize("name", list(CASES))
def test_shear_forward_matches_general_and_oracle(cuda, name):
    from petl_b200 import ops
    G, Go, f, _ = _setup(name, cuda)
    ft = _t(f, cuda)
    a, b = _both(lambda: _np(ops.project(G, ft)))
    assert rel_l2(b, a) < 1e-5
    if name != "t1":
        assert rel_l2(b, O.project(Go, f)[0]) < 1e-5


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("mode", ["reference", "adjoint"])
def test_shear_backward_matches_general(cuda, name, mode):
    from petl_b200 import ops
    G, Go, f, rng = _setup(name, cuda)
    y = _t(rng.random(G.shape), cuda)
    a, b = _both(lambda: _np(ops.backproject(G, y, mode=mode)))
    assert rel_l2(b, a) < 1e-5
    if mode == "reference" and name != "t1":
        assert rel_l2(b, O.backproject(Go, _np(y))) < 1e-5


@pytest.mark.parametrize("name", list(CASES))
def test_shear_pair_is_exact_adjoint(cuda, name):
    import torch
    from petl_b200 import ops
    G, _, f, rng = _setup(name, cuda)
    x = _t(rng.random(G.vol_shape), cuda)
    y = _t(rng.random(G.shape), cuda)
    Ax = ops.project(G, x)
    Aty = ops.backproject(G, y, mode="adjoint")
    lhs = float(torch.sum(Ax.double() * y.double()))
    rhs = float(torch.sum(x.double() * Aty.double()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_shear_subsets_slabs_ratio(cuda):
    import torch
    from petl_b200 import ops
    G, _, f, rng = _setup("t2", cuda)
    ft = _t(f, cuda)
    full = ops.project(G, ft)
    parts = torch.zeros_like(full)
    for s in range(4):
        ops.project(G, ft, parts, subset=(s, 4))
    assert torch.equal(full, parts)
    slabs = torch.zeros_like(full)
    ops.project(G, ft, slabs, v1_range=(0, 5))
    ops.project(G, ft, slabs, v1_range=(5, G.shape[0]))
    assert torch.equal(full, slabs)
    meas = torch.poisson(full * 20.0)
    ratio = ops.project_ratio(G, ft, meas)
    want = torch.where(full == 0, torch.zeros_like(full), meas / full)
    assert rel_l2(_np(ratio), _np(want)) < 1e-6
    y = _t(rng.random(G.shape), cuda)
    b = ops.backproject(G, y)
    b2 = ops.backproject(G, y, subset=(0, 3))
    for s in (1, 2):
        ops.backproject(G, y, f=b2, subset=(s, 3), accumulate=True)
    assert rel_l2(_np(b2), _np(b)) < 1e-6
    b3 = ops.backproject(G, y, v1_range=(0, 7))
    ops.backproject(G, y, f=b3, v1_range=(7, G.shape[0]), accumulate=True)
    assert rel_l2(_np(b3), _np(b)) < 1e-6
    b4 = ops.backproject(G, y, scale=2.5)
    assert rel_l2(_np(b4), 2.5 * _np(b)) < 1e-6

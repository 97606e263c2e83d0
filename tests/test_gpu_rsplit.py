"""The split backprojector with the reference's semantics for any psi (path
3 in reference mode: an in-plane pass per (v1, u1) slice, then a z pass)
against the general kernel (dispatch 1) and the FP64 oracle: y- and
x-dominant views, ragged and off-centre volumes, unequal voxel and u1
pitch (psi = 0, 30 and 90), four-tap extents, view subsets, slope ranges,
accumulate, scale and FBP.  Voxels wider than three u0 bins keep the
general kernel."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2
from helpers import ellipsoids
from test_gpu_gsplit import CASES as GCASES
from test_gpu_gsplit import _under

pytestmark = pytest.mark.gpu

CASES = dict(GCASES)
CASES.update({
    # unequal voxel height and u1 pitch (at psi = 0 and 90 too: the shear
    # kernels need equal pitch, so these take the split kernels)
    "p30pitch": ((30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (40, 40, 12, 1.5, 1.25)),
    "p0pitch": ((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (44, 40, 12, 1.0, 1.5, 0.5, -1.0, 0.0)),
    "p90pitch": ((90.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (40, 44, 12, 1.0, 1.5, -1.0, 0.5, 0.0)),
    # voxels 1.9 bins wide: extents of up to four u0 bins
    "p75wide": ((75.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25), (40, 44, 12, 1.9, 1.0, 1.0, -2.0, 0.5)),
})


def _setup(name, cuda, seed=0):
    import torch
    from petl_b200 import Geometry
    args, vol = CASES[name]
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(seed)
    y = rng.random(G.shape).astype(np.float32)
    return G, Go, y, torch.from_numpy(y).to(cuda), rng


@pytest.mark.parametrize("name", list(CASES))
def test_split_reference_backprojection(cuda, name):
    from petl_b200 import ops
    G, Go, y, yt, _ = _setup(name, cuda)
    a, pa = _under(0, lambda: ops.backproject(G, yt).cpu().numpy())
    b, pb = _under(1, lambda: ops.backproject(G, yt).cpu().numpy())
    assert (pa, pb) == (3, 0)
    assert rel_l2(a, b) < 1e-5
    assert rel_l2(a, O.backproject(Go, y)) < 1e-5


def test_split_reference_subsets_slopes_accumulate(cuda):
    import torch
    from petl_b200 import lib
    G, _, _, y, rng = _setup("p135rag", cuda)
    L = lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    f0 = torch.from_numpy(rng.random(G.vol_shape).astype(np.float32)).to(cuda)
    nv1 = G.shape[0]
    for first, step, v1b, v1e, acc, scale in ((1, 3, 0, nv1, 0, 1.0), (0, 1, 5, nv1 - 3, 1, 0.5),
                                              (2, 4, 3, nv1, 1, 2.0)):
        outs, paths = [], []
        for mode in (0, 1):
            f = f0.clone()
            assert L.petl_set_dispatch(mode) == 0
            try:
                rc = L.petl_backproject_range_dev(G.ptr, y.data_ptr(), f.data_ptr(), 0, acc, ctypes.c_float(scale),
                                                  v1b, v1e, first, step, st)
                torch.cuda.synchronize()
                paths.append(L.petl_last_projector_path())
            finally:
                L.petl_set_dispatch(0)
            assert rc == 0, (mode, first, step, v1b, v1e, L.petl_last_error().decode())
            assert L.petl_device_error_flag() == 0
            outs.append(f.cpu().numpy())
        assert paths == [3, 0]
        assert rel_l2(outs[0], outs[1]) < 1e-5


def test_split_reference_fbp(cuda):
    import torch
    from petl_b200 import Geometry, ops
    args, vol = CASES["p30"]
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(3)
    f = ellipsoids(G.vol_shape, (vol[3], vol[3]), rng, 6)
    g = O.project(Go, f)[0].astype(np.float32)
    gt = torch.from_numpy(g).to(cuda)
    a, pa = _under(0, lambda: ops.fbp(G, gt).cpu().numpy())
    b, pb = _under(1, lambda: ops.fbp(G, gt).cpu().numpy())
    assert (pa, pb) == (3, 0)
    assert rel_l2(a, b) < 1e-5


def test_wide_voxels_keep_the_general_kernel(cuda):
    import torch
    from petl_b200 import Geometry, lib, ops
    G = Geometry(30.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25, volume=(16, 16, 8, 4.0))
    ops.backproject(G, torch.rand(G.shape, device=cuda))
    torch.cuda.synchronize()
    assert lib().petl_last_projector_path() == 0

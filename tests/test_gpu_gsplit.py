"""The split forward projector for any psi (x pass and z pass through FP32
scratch, path 3) against the general kernels (dispatch 1) and the FP64
oracle: y-driven and x-driven views, ragged and off-centre volumes, view
subsets, slope ranges and the MLEM ratio epilogue.  Unequal voxel height and
u1 pitch keeps the general kernels."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

CASES = {
    # psi, D, L, H, T, v_m0, v_m1 ; volume
    "p30": ((30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0)),
    "p60": ((60.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0)),
    "p135rag": ((135.0, 100.0, 75.0, 27.0, 1.5, 0.45, 0.2), (52, 60, 18, 1.5, 1.5, 3.0, -4.5, 1.5)),
    "p17wide": ((17.0, 300.0, 128.0, 32.0, 1.0, 0.5, 0.25), (200, 96, 32, 1.0)),
    # psi = 180 (y-driven, cos = -1) and -45 degrees (ties |r_x| = |r_y| at v0 = 0)
    "p180": ((180.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 48, 16, 2.0)),
    "pm45": ((-45.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (48, 64, 16, 2.0, 2.0, -2.0, 3.0, 1.0)),
    # 33 and 21 slopes over 80 and 72 u1 rows: the last 1 and 5 slopes run in
    # the tail shape (8 slopes x 128 rows per CTA)
    "p30tail1": ((30.0, 128.0, 64.0, 80.0, 1.0, 0.5, 0.25), (64, 64, 80, 1.0)),
    "p60tail5": ((60.0, 96.0, 48.0, 72.0, 1.0, 0.5, 0.22), (48, 48, 72, 1.0)),
}


def _setup(name, cuda, seed=0):
    import torch
    from petl_b200 import Geometry
    args, vol = CASES[name]
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(seed)
    f = ellipsoids(G.vol_shape, (vol[3], vol[4] if len(vol) > 4 else vol[3]), rng, 8) + \
        0.1 * rng.random(G.vol_shape).astype(np.float32)
    return G, Go, f, torch.from_numpy(f).to(cuda), rng


def _under(mode, fn):
    import torch
    from petl_b200 import lib
    L = lib()
    assert L.petl_set_dispatch(mode) == 0
    try:
        out = fn()
        torch.cuda.synchronize()
        path = L.petl_last_projector_path()
    finally:
        L.petl_set_dispatch(0)
    assert L.petl_device_error_flag() == 0
    return out, path


@pytest.mark.parametrize("name", list(CASES))
def test_split_forward_any_psi(cuda, name):
    from petl_b200 import ops
    G, Go, f, ft, _ = _setup(name, cuda)
    a, pa = _under(0, lambda: ops.project(G, ft).cpu().numpy())
    b, pb = _under(1, lambda: ops.project(G, ft).cpu().numpy())
    assert (pa, pb) == (3, 0)
    assert rel_l2(a, b) < 1e-5
    assert rel_l2(a, O.project(Go, f)[0]) < 1e-5


def test_split_forward_subsets_slopes_ratio(cuda):
    import torch
    from petl_b200 import lib
    G, _, f, ft, rng = _setup("p30", cuda)
    L = lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    meas = torch.from_numpy(rng.poisson(5.0, size=G.shape).astype(np.float32)).to(cuda)
    nv1 = G.shape[0]
    for first, step, v1b, v1e, with_meas in ((1, 3, 0, nv1, False), (0, 1, 5, nv1 - 3, True),
                                             (2, 4, 3, nv1, True)):
        outs = []
        for mode in (0, 1):
            g = torch.full(G.shape, -7.0, device=cuda)
            assert L.petl_set_dispatch(mode) == 0
            try:
                if with_meas:
                    rc = L.petl_project_ratio_dev(G.ptr, ft.data_ptr(), meas.data_ptr(), g.data_ptr(), v1b, v1e,
                                                  first, step, st)
                else:
                    rc = L.petl_project_range_dev(G.ptr, ft.data_ptr(), g.data_ptr(), v1b, v1e, first, step, st)
                torch.cuda.synchronize()
            finally:
                L.petl_set_dispatch(0)
            assert rc == 0, (mode, first, step, v1b, v1e, with_meas, L.petl_last_error().decode())
            assert L.petl_device_error_flag() == 0
            outs.append(g.cpu().numpy())
        a, b = outs
        # untouched entries keep their value; computed ones agree
        assert np.array_equal(a == -7.0, b == -7.0)
        assert rel_l2(a, b) < 1e-5


def test_unequal_pitch_keeps_the_general_kernels(cuda):
    import torch
    from petl_b200 import Geometry, lib, ops
    G = Geometry(30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25, volume=(40, 40, 12, 1.5, 1.25))
    ops.project(G, torch.rand(G.vol_shape, device=cuda))
    torch.cuda.synchronize()
    assert lib().petl_last_projector_path() == 0

"""The split exact-adjoint backprojector for any psi (path 3 in adjoint mode:
h = g l_phi rs, a z gather over the slopes, an x gather over the u0
columns) against the general adjoint kernel (dispatch 1), the adjoint
identity with the split forward projector, and the FP64 oracle's forward
projector: y-driven and x-driven views, ragged and off-centre volumes, view
subsets, slope ranges, accumulate and scale."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import rel_l2
from test_gpu_gsplit import CASES, _setup, _under

pytestmark = pytest.mark.gpu


def _dot(a, b):
    return float(np.sum(a.astype(np.float64) * b.astype(np.float64)))


@pytest.mark.parametrize("name", list(CASES))
def test_split_adjoint_any_psi(cuda, name):
    import torch
    from petl_b200 import ops
    G, Go, f, ft, rng = _setup(name, cuda)
    y = rng.random(G.shape).astype(np.float32)
    yt = torch.from_numpy(y).to(cuda)
    a, pa = _under(0, lambda: ops.backproject(G, yt, mode="adjoint").cpu().numpy())
    b, pb = _under(1, lambda: ops.backproject(G, yt, mode="adjoint").cpu().numpy())
    assert (pa, pb) == (3, 0)
    assert rel_l2(a, b) < 1e-5
    # <A x, y> = <x, A^T y>: with the split forward (float rounding) and with
    # the oracle's FP64 forward
    Ax, _ = _under(0, lambda: ops.project(G, ft).cpu().numpy())
    lhs, rhs = _dot(Ax, y), _dot(f, a)
    assert abs(lhs - rhs) / abs(lhs) < 1e-6
    lhs_o = _dot(O.project(Go, f)[0], y)
    assert abs(lhs_o - rhs) / abs(lhs_o) < 1e-5


def test_split_adjoint_subsets_slopes_accumulate(cuda):
    import torch
    from petl_b200 import lib
    G, _, _, _, rng = _setup("p135rag", cuda)
    L = lib()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    y = torch.from_numpy(rng.random(G.shape).astype(np.float32)).to(cuda)
    f0 = torch.from_numpy(rng.random(G.vol_shape).astype(np.float32)).to(cuda)
    nv1 = G.shape[0]
    for first, step, v1b, v1e, acc, scale in ((1, 3, 0, nv1, 0, 1.0), (0, 1, 5, nv1 - 3, 1, 0.5),
                                              (2, 4, 3, nv1, 1, 2.0)):
        outs, paths = [], []
        for mode in (0, 1):
            f = f0.clone()
            assert L.petl_set_dispatch(mode) == 0
            try:
                rc = L.petl_backproject_range_dev(G.ptr, y.data_ptr(), f.data_ptr(), 1, acc, ctypes.c_float(scale),
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

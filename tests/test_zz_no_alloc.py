"""The allocation-free forward projection entry point.

petl_project_noalloc_dev serves callers that must not allocate device memory
while they run (a real-time acquisition thread that cannot block on the
allocator, or a program whose own memory pool owns the GPU).  It keeps its
scratch tables in a fixed device array instead of allocating them.  These
checks call it through the C ABI and compare it with the allocating entry
point petl_project_dev on two calls in a row (the second on another
geometry, so the shared array is rewritten), and check that a geometry whose
tables do not fit is refused with an error.  The file sorts last so that a
run stopping at the first failure has run every other test already; it also
passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_noalloc_projection_matches_allocating_entry_point(cuda):
    import torch
    from petl_b200 import Geometry, lib
    L = lib()
    cases = [((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0)),
             ((0.0, 100.0, 50.0, 26.0, 1.5, 0.45, 0.2), (50, 58, 15, 1.5, 1.5, 3.0, -4.5, 1.5))]
    rng = np.random.default_rng(11)
    for args, vol in cases:  # two calls in a row, different geometries
        G = Geometry(*args, volume=vol)
        f = torch.from_numpy(rng.random(G.vol_shape).astype(np.float32)).to(cuda)
        want = torch.full(G.shape, -1.0, device=cuda)
        got = torch.full(G.shape, -2.0, device=cuda)
        assert L.petl_project_dev(G.ptr, _vp(f), _vp(want), 0, 1, _stream()) == 0
        assert L.petl_project_noalloc_dev(G.ptr, _vp(f), _vp(got), _stream()) == 0, L.petl_last_error()
        # the shear kernel ran, so its tables went through the fixed array
        assert L.petl_last_projector_path() == 1
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-5


def test_noalloc_projection_follows_forced_general_dispatch(cuda):
    import torch
    from petl_b200 import Geometry, lib
    L = lib()
    G = Geometry(0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25, volume=(64, 64, 16, 2.0))
    f = torch.from_numpy(np.random.default_rng(12).random(G.vol_shape).astype(np.float32)).to(cuda)
    want = torch.zeros(G.shape, device=cuda)
    got = torch.zeros(G.shape, device=cuda)
    assert L.petl_project_dev(G.ptr, _vp(f), _vp(want), 0, 1, _stream()) == 0
    assert L.petl_set_dispatch(1) == 0
    try:
        assert L.petl_project_noalloc_dev(G.ptr, _vp(f), _vp(got), _stream()) == 0, L.petl_last_error()
        assert L.petl_last_projector_path() == 0
    finally:
        L.petl_set_dispatch(0)
    torch.cuda.synchronize()
    assert rel_l2(got.cpu().numpy(), want.cpu().numpy()) < 1e-5


def test_noalloc_projection_refuses_oversized_tables(cuda):
    import torch
    from petl_b200 import Geometry, lib
    L = lib()
    # 129 slopes x 4096 planes of shift tables: more than the 4 MiB array
    G = Geometry(0.0, 64.0, 32.0, 2.0, 0.25, 0.5, 0.25, volume=(8, 4096, 4, 0.25))
    assert G.shape[1] == 129
    f = torch.zeros(G.vol_shape, device=cuda)
    g = torch.zeros(G.shape, device=cuda)
    rc = L.petl_project_noalloc_dev(G.ptr, _vp(f), _vp(g), _stream())
    assert rc != 0
    assert b"at most" in L.petl_last_error()

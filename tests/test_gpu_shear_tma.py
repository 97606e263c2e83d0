"""The TMA-staged shear-warp kernels against the first-generation shear
kernels, the general kernels and the FP64 oracle.

Dispatch 0 runs the TMA-staged kernels wherever their layout rules hold
(volume rows a multiple of 4 floats for the forward copy; for the backward
N_u0 a multiple of 4 and at most 256 with a tensor map, else any even N_u0
up to 512 with bulk copies of row pairs), with the split forward (x-shift
pass into scratch, then the z-tap kernel); dispatch 3 the same with the
single-kernel TMA forward and single-pass TMA backprojection; dispatch 2
runs the first-generation shear kernels; dispatch 1 the general kernels.
The split and single-kernel forms (forward, and backward where the planogram
rows are multiples of 16 bytes) do the same float operations in the same
order and agree bit for bit; the forward TMA kernels and the first-generation one agree to rounding
of the final scale; the backward kernels sum in a different order and agree
to float accuracy.  Every case also checks that no
bounded wait gave up (petl_device_error_flag) and which kernels ran.
"""
import numpy as np
import pytest

import oracle as O
from conftest import rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

CASES = {
    # psi, D, L, H, T, v_m0, v_m1 ; volume ; single-kernel TMA forward, TMA
    # backward expected (the split forward applies to every case: it stages
    # its own padded scratch rows, not the volume's)
    "t2": ((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0), True, True),
    "t1": ((0.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25), (128, 128, 32, 1.0), True, True),
    # the dual-panel geometry of the 128x128x64 / 2 mm recon: planogram (33, 65, 64, 128)
    "panel2mm": ((0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0), True, True),
    # ragged sizes, off-centre volume, rows a multiple of 4
    "rag4": ((0.0, 100.0, 75.0, 27.0, 1.5, 0.45, 0.2), (52, 60, 18, 1.5, 1.5, 3.0, -4.5, 1.5), True, True),
    # volume rows not a multiple of 4 floats: no single-kernel TMA forward; the
    # backward stages planogram rows (62 columns) by bulk copies of row pairs
    "odd": ((0.0, 100.0, 50.0, 26.0, 1.5, 0.45, 0.2), (50, 58, 15, 1.5, 1.5, 3.0, -4.5, 1.5), False, True),
    # N_u0 = 278 (> 256, not a multiple of 4): bulk-copy backward, one plane group
    "wide": ((0.0, 300.0, 128.0, 32.0, 1.0, 0.5, 0.25), (256, 64, 32, 1.0), True, True),
    # and numX = 320 > 256
    "wide2": ((0.0, 300.0, 128.0, 32.0, 1.0, 0.5, 0.25), (320, 48, 16, 1.0), True, True),
    # psi = 90 degrees (x-driven rays): the same kernels on the volume with x and
    # y exchanged (y' = -x); square, and ragged with offsets (numX != numY)
    "p90": ((90.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0), True, True),
    "p90rag": ((90.0, 100.0, 75.0, 27.0, 1.5, 0.45, 0.2), (52, 60, 18, 1.5, 1.5, 3.0, -4.5, 1.5), True, True),
}


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


def _np(t):
    return t.detach().cpu().numpy()


def _setup(name, cuda, seed=0):
    from petl_b200 import Geometry
    args, vol, _, _ = CASES[name]
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(seed)
    f = ellipsoids(G.vol_shape, (vol[3], vol[4] if len(vol) > 4 else vol[3]), rng, 8) + \
        0.1 * rng.random(G.vol_shape).astype(np.float32)
    return G, Go, f, rng


def _under(mode, fn):
    """fn() under dispatch mode, and the kernel path it took."""
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
def test_tma_forward(cuda, name):
    from petl_b200 import ops
    G, Go, f, _ = _setup(name, cuda)
    ft = _t(f, cuda)
    a, pa = _under(0, lambda: _np(ops.project(G, ft)))
    b, pb = _under(2, lambda: _np(ops.project(G, ft)))
    c, pc = _under(1, lambda: _np(ops.project(G, ft)))
    d, pd = _under(3, lambda: _np(ops.project(G, ft)))
    assert (pa, pb, pc, pd) == (2, 1, 0, 2 if CASES[name][2] else 1)
    if CASES[name][2]:
        assert np.array_equal(a, d)
    assert rel_l2(a, b) < 1e-6
    assert rel_l2(a, c) < 1e-5
    assert rel_l2(a, O.project(Go, f)[0]) < 1e-5


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("mode", ["reference", "adjoint"])
def test_tma_backward(cuda, name, mode):
    from petl_b200 import ops
    G, Go, f, rng = _setup(name, cuda)
    y = _t(rng.random(G.shape), cuda)
    a, pa = _under(0, lambda: _np(ops.backproject(G, y, mode=mode)))
    b, pb = _under(2, lambda: _np(ops.backproject(G, y, mode=mode)))
    c, pc = _under(1, lambda: _np(ops.backproject(G, y, mode=mode)))
    d, pd = _under(3, lambda: _np(ops.backproject(G, y, mode=mode)))
    assert (pa, pb, pc, pd) == (2 if CASES[name][3] else 1, 1, 0, pa)
    # the split backprojection and the single-pass TMA kernel agree bit for bit
    assert np.array_equal(a, d)
    assert rel_l2(a, b) < 1e-5
    assert rel_l2(a, c) < 1e-5
    if mode == "reference":
        assert rel_l2(a, O.backproject(Go, _np(y))) < 1e-5


@pytest.mark.parametrize("name", ["t1", "panel2mm", "rag4", "odd", "wide", "p90", "p90rag"])
def test_tma_pair_is_exact_adjoint(cuda, name):
    import torch
    from petl_b200 import ops
    G, _, f, rng = _setup(name, cuda)
    x = _t(rng.random(G.vol_shape), cuda)
    y = _t(rng.random(G.shape), cuda)
    (Ax, Aty), path = _under(0, lambda: (ops.project(G, x), ops.backproject(G, y, mode="adjoint")))
    assert path == 2
    lhs = float(torch.sum(Ax.double() * y.double()))
    rhs = float(torch.sum(x.double() * Aty.double()))
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_tma_subsets_slabs_ratio_accumulate(cuda):
    import torch
    from petl_b200 import ops
    G, _, f, rng = _setup("panel2mm", cuda)
    ft = _t(f, cuda)
    y = _t(rng.random(G.shape), cuda)

    def run():
        full = ops.project(G, ft)
        parts = torch.zeros_like(full)
        for s in range(4):
            ops.project(G, ft, parts, subset=(s, 4))
        slabs = torch.zeros_like(full)
        ops.project(G, ft, slabs, v1_range=(0, 5))
        ops.project(G, ft, slabs, v1_range=(5, G.shape[0]))
        meas = torch.poisson(full * 20.0, generator=torch.Generator(device=full.device).manual_seed(3))
        ratio = ops.project_ratio(G, ft, meas)
        b = ops.backproject(G, y)
        b2 = ops.backproject(G, y, subset=(0, 3))
        for s in (1, 2):
            ops.backproject(G, y, f=b2, subset=(s, 3), accumulate=True)
        b3 = ops.backproject(G, y, v1_range=(0, 7))
        ops.backproject(G, y, f=b3, v1_range=(7, G.shape[0]), accumulate=True)
        b4 = ops.backproject(G, y, scale=2.5)
        return full, parts, slabs, meas, ratio, b, b2, b3, b4

    (full, parts, slabs, meas, ratio, b, b2, b3, b4), path = _under(0, run)
    assert path == 2
    (full3, parts3, slabs3, _, ratio3, b_3, b2_3, b3_3, b4_3), path3 = _under(3, run)
    assert path3 == 2
    assert torch.equal(full, full3) and torch.equal(parts, parts3) and torch.equal(slabs, slabs3)
    assert torch.equal(ratio, ratio3)
    assert torch.equal(b, b_3)
    assert torch.equal(b2, b2_3)
    assert torch.equal(b3, b3_3)
    assert torch.equal(b4, b4_3)
    assert torch.equal(full, parts)
    assert torch.equal(full, slabs)
    want = torch.where(full == 0, torch.zeros_like(full), meas / full)
    assert rel_l2(_np(ratio), _np(want)) < 1e-6
    assert rel_l2(_np(b2), _np(b)) < 1e-6
    assert rel_l2(_np(b3), _np(b)) < 1e-6
    assert rel_l2(_np(b4), 2.5 * _np(b)) < 1e-6


def test_tma_full_size_against_first_generation(cuda):
    """The 256x256x128 volume and (65, 129, 128, 256) planogram of the benchmark."""
    import torch
    from petl_b200 import Geometry, ops
    G = Geometry(0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25, volume=(256, 256, 128, 1.0))
    gen = torch.Generator(device=cuda).manual_seed(5)
    f = torch.rand(G.vol_shape, device=cuda, generator=gen)
    a, pa = _under(0, lambda: ops.project(G, f))
    b, pb = _under(2, lambda: ops.project(G, f))
    c, pc = _under(3, lambda: ops.project(G, f))
    assert (pa, pb, pc) == (2, 1, 2)
    assert torch.equal(a, c)
    assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) < 1e-6
    del b, c
    for mode in ("reference", "adjoint"):
        x, px = _under(0, lambda: ops.backproject(G, a, mode=mode))
        z, pz = _under(2, lambda: ops.backproject(G, a, mode=mode))
        w, pw = _under(3, lambda: ops.backproject(G, a, mode=mode))
        assert (px, pz, pw) == (2, 1, 2)
        assert torch.equal(x, w)
        assert float(torch.linalg.vector_norm(x - z) / torch.linalg.vector_norm(z)) < 1e-5


@pytest.mark.parametrize("name", ["t2", "rag4", "odd", "wide", "p90rag"])
@pytest.mark.parametrize("mode", ["reference", "adjoint"])
def test_single_slope_backprojection(cuda, name, mode):
    """The rebinned planogram of FBP (one slope, v1 = 0) backprojects through
    z sums without a plane dimension; bit-equal to the single-pass kernel
    and within 1e-5 of the oracle (reference semantics), with accumulate and
    scale applied as the C ABI passes them."""
    import torch
    from petl_b200 import lib, ops
    G, Go, f, rng = _setup(name, cuda)
    Gr = G.rebinned()
    Gro = O.make_geom(*CASES[name][0], CASES[name][1])
    Gro.N_v1, Gro.v1_0 = 1, 0.0
    y = _t(rng.random(Gr.shape), cuda)
    a, pa = _under(0, lambda: _np(ops.backproject(Gr, y, mode=mode)))
    d, pd = _under(3, lambda: _np(ops.backproject(Gr, y, mode=mode)))
    assert pa == pd
    assert np.array_equal(a, d)
    if mode == "reference":
        assert rel_l2(a, O.backproject(Gro, _np(y))) < 1e-5
    # accumulate with a scale: f + 0.5 A^T y
    L = lib()
    base = _t(rng.random(Gr.vol_shape), cuda)
    out = base.clone()
    m = 0 if mode == "reference" else 1
    assert L.petl_backproject_dev(Gr.ptr, y.data_ptr(), out.data_ptr(), m, 1, 0.5, 0, 1,
                                  torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert L.petl_device_error_flag() == 0
    want = _np(base) + 0.5 * a
    assert np.abs(_np(out) - want).max() <= 1e-6 * np.abs(want).max()

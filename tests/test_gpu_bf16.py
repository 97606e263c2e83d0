"""BF16 storage: bfloat16 volumes and planograms with FP32 footprint
accumulation.  The BF16 kernels are the TMA-staged shear kernels reading and
writing 2-byte elements; on the same (bfloat16-representable) inputs they do
the same FP32 operations as the FP32 kernels, so their outputs equal the FP32
outputs rounded to bfloat16 (forward, data ratio) or equal them exactly
(backprojection, which writes FP32).  OSEM with BF16 storage stays within
bfloat16 rounding of OSEM in FP32."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

CASES = {
    "panel2mm": ((0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0)),
    "t1": ((0.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25), (128, 128, 32, 1.0)),
}


def _setup(name, cuda, seed=0):
    import torch
    from petl_b200 import Geometry
    args, vol = CASES[name]
    G = Geometry(*args, volume=vol)
    rng = np.random.default_rng(seed)
    f = ellipsoids(G.vol_shape, (vol[3], vol[3]), rng, 8) + 0.1 * rng.random(G.vol_shape).astype(np.float32)
    f16 = torch.from_numpy(f.astype(np.float32)).to(cuda).to(torch.bfloat16)
    return G, f16


@pytest.mark.parametrize("name", list(CASES))
def test_bf16_forward_equals_rounded_fp32(cuda, name):
    import torch
    from petl_b200 import lib, ops
    G, f16 = _setup(name, cuda)
    g16 = ops.project_bf16(G, f16)
    assert lib().petl_last_projector_path() == 2
    g32 = ops.project(G, f16.float())
    assert lib().petl_last_projector_path() == 2
    assert torch.equal(g16, g32.to(torch.bfloat16))
    assert lib().petl_device_error_flag() == 0


@pytest.mark.parametrize("mode", ["reference", "adjoint"])
def test_bf16_backward_equals_fp32(cuda, mode):
    import torch
    from petl_b200 import ops
    for name in CASES:
        G, _ = _setup(name, cuda)
        y16 = torch.rand(G.shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(2)).to(torch.bfloat16)
        a = ops.backproject_bf16(G, y16, mode=mode)
        b = ops.backproject(G, y16.float(), mode=mode)
        assert torch.equal(a, b)
        c = ops.backproject_bf16(G, y16, f=a.clone(), mode=mode, accumulate=True, scale=0.5)
        assert rel_l2((c - 1.5 * b).cpu().numpy(), np.zeros(1)) <= 1e-6 * float(b.norm())


def test_bf16_ratio_equals_rounded_fp32(cuda):
    import torch
    from petl_b200 import ops
    G, f16 = _setup("panel2mm", cuda)
    g = ops.project(G, f16.float())
    meas = torch.poisson(g * 50.0, generator=torch.Generator(device=cuda).manual_seed(4)).to(torch.bfloat16)
    r16 = ops.project_ratio_bf16(G, f16, meas)
    r32 = ops.project_ratio(G, f16.float(), meas.float())
    assert torch.equal(r16, r32.to(torch.bfloat16))


def test_bf16_osem_tracks_fp32(cuda):
    import torch
    from petl_b200 import ops, recon
    G, f16 = _setup("panel2mm", cuda)
    g = ops.project(G, f16.float())
    meas = torch.poisson(g * (2e6 / float(g.sum())), generator=torch.Generator(device=cuda).manual_seed(5))
    f32, _ = recon.osem(G, meas, 2, 4)
    # FP32 image, bfloat16 planograms and projector input
    fb = recon.osem_bf16(G, meas.to(torch.bfloat16), 2, 4)
    assert fb.dtype == torch.float32
    assert rel_l2(fb.cpu().numpy(), f32.cpu().numpy()) < 2e-3
    # image stored in bfloat16 as well: within a few bfloat16 ulps
    fbb = recon.osem_bf16(G, meas.to(torch.bfloat16), 2, 4, image="bf16")
    assert fbb.dtype == torch.bfloat16
    assert rel_l2(fbb.float().cpu().numpy(), f32.cpu().numpy()) < 2e-2


def test_bf16_refuses_non_shear_geometry(cuda):
    import torch
    from petl_b200 import Geometry, PetlError, ops
    G = Geometry(30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25, volume=(64, 64, 16, 2.0))
    f16 = torch.ones(G.vol_shape, device=cuda, dtype=torch.bfloat16)
    with pytest.raises(PetlError, match="axis-aligned"):
        ops.project_bf16(G, f16)

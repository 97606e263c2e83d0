"""List-mode binning on the GPU against the oracle and the reference.

The device kernel maps each coincidence to planogram coordinates with the
reference's float operations (rounding-pinned) and deposits it with atomic
adds.  Nearest-bin counts are integers, so they must match the oracle bit
for bit; bilinear deposits add fractional weights in a different order than
the reference's sequential loop, so they are held to 1e-6 relative L2 (and
their total to float accuracy).  The C ABI's bin() parses the reference's
file formats and must reproduce the reference's own bin() (golden vectors)
to the same bound.
"""
import os

import numpy as np
import pytest

import oracle as O
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

BIN_CASES = ["bin_g0", "bin_g0t1", "bin_gpetx"]


def _case(name):
    from petl_b200 import Geometry
    z = load_golden("binning.npz")
    vol = tuple(z[f"{name}_volume"])
    plans = z[f"{name}_planograms"]
    ogeoms = [O.make_geom(*p, vol) for p in plans]
    pgeoms = [Geometry(*p, volume=vol) for p in plans]
    return z, plans, vol, ogeoms, pgeoms


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


@pytest.mark.parametrize("name", BIN_CASES)
@pytest.mark.parametrize("linear", [True, False])
def test_device_binning_matches_oracle(cuda, name, linear):
    import torch
    from petl_b200 import ops, lib
    z, _, _, ogeoms, pgeoms = _case(name)
    blue, pink = z[f"{name}_blue"], z[f"{name}_pink"]
    want = O.bin_events(ogeoms, blue, pink, linear=linear)
    got = ops.bin_events(pgeoms, _t(blue, cuda), _t(pink, cuda), linear=linear)
    torch.cuda.synchronize()
    for w, g in zip(want, got):
        g = g.cpu().numpy()
        if linear:
            assert rel_l2(g, w) < 1e-6
            assert abs(float(g.sum(dtype=np.float64)) - float(w.sum(dtype=np.float64))) < 1e-3
        else:
            assert np.array_equal(g, w)
    assert lib().petl_device_error_flag() == 0


@pytest.mark.parametrize("name", BIN_CASES)
def test_cabi_bin_file_matches_reference(cuda, name, tmp_path):
    """PETLserver.bin on the file the reference binned (rewritten from the
    fixture's events and interaction counts) reproduces the reference's
    planograms, which it overwrites (g is pre-filled with 7)."""
    from petl_b200 import PETLserver, listmode
    z, plans, vol, _, _ = _case(name)
    fmt = str(z[f"{name}_format"])
    path = os.path.join(tmp_path, name + (".lst" if fmt == "lst" else ".dat"))
    if fmt == "lst":
        listmode.write_lst(path, z[f"{name}_blue"], z[f"{name}_pink"])
    else:
        listmode.write_acq(path, z[f"{name}_blue"], z[f"{name}_pink"], (z[f"{name}_nb"], z[f"{name}_np"]))
    s = PETLserver()
    for p in plans:
        s.add_planogram(*p)
    s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(vol)])
    g = [np.full(a.shape, 7.0, np.float32) for a in s.allocate_projections()]
    s.bin(path, g)
    for i, gi in enumerate(g):
        ref = z[f"{name}_g{i}"]
        assert rel_l2(gi, ref) < 1e-6
        assert abs(float(gi.sum(dtype=np.float64)) - float(ref.sum(dtype=np.float64))) < 1e-3


def test_binning_large_random_and_edges(cuda):
    """200k coincidences, a quarter of them outside the acceptance angle;
    empty input; accumulation into a given planogram."""
    import torch
    from petl_b200 import Geometry, ops, listmode
    args = (0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25)
    vol = (128, 128, 64, 2.0)
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(7)
    blue, pink = listmode.coincidences(200000, rng, 128.0, 64.0, 32.0, box=(50.0, 50.0, 25.0))
    # a quarter tilted beyond v_m0 / v_m1: dropped by the acceptance test
    k = len(blue) // 4
    pink[:k, 0] += 400.0
    pink[k:2 * k, 2] += 300.0
    want = O.bin_events(Go, blue, pink)[0]
    got = ops.bin_events(G, _t(blue, cuda), _t(pink, cuda))
    assert rel_l2(got.cpu().numpy(), want) < 1e-6
    # accumulate into a given planogram, and an empty batch is a no-op
    ops.bin_events(G, _t(blue, cuda), _t(pink, cuda), g=got)
    ops.bin_events(G, torch.zeros((0, 3), device=cuda), torch.zeros((0, 3), device=cuda), g=got)
    assert rel_l2(got.cpu().numpy(), 2 * want) < 1e-6
    near = ops.bin_events(G, _t(blue, cuda), _t(pink, cuda), linear=False)
    assert np.array_equal(near.cpu().numpy(), O.bin_events(Go, blue, pink, linear=False)[0])

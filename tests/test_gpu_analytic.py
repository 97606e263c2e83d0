"""Analytic phantoms on the GPU: voxelization, ray tracing and the detector
stopping power against the oracle and the reference.

The voxelizer repeats the reference's host float/double operations with
rounding-pinned intrinsics, so its volumes are bit-identical to the
reference's.  Ray tracing mixes float and double arithmetic whose
contractions (and, in the reference, fast-math divisions) differ in the
last bits, so the planograms are held to a relative L2 bound: 1e-5 against
the oracle (same operations, IEEE divisions) and against the reference's
fast-math kernels.
"""
import os
import sys

import numpy as np
import pytest

import oracle as O
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_golden import PHANTOM, PHANTOM2, _modules  # noqa: E402

RT_CASES = ["g0", "g30", "gpetx"]


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


def _product_solids(spec):
    from petl_b200 import ops
    return [ops.make_solid(t, c, r, v, A, clip) for t, c, r, v, A, clip in spec]


def _oracle_solids(spec):
    return [O.make_solid(t, c, r, v, A, clip) for t, c, r, v, A, clip in spec]


def _origin(nx, ny, nz, vw, vh):
    f32 = np.float32
    return (float(f32((0 - 0.5 * (nx - 1)) * vw)), float(f32((0 - 0.5 * (ny - 1)) * vw)),
            float(f32((0 - 0.5 * (nz - 1)) * vh)))


def test_device_voxelize_matches_reference(cuda):
    from petl_b200 import ops, lib
    from petl_b200._lib import petl_solid
    z = load_golden("voxelize.npz")
    nx, ny, nz = (int(v) for v in z["volume"][:3])
    vw, vh = float(z["volume"][3]), float(z["volume"][4])
    x0, y0, z0 = _origin(nx, ny, nz, vw, vh)
    solids = _product_solids(PHANTOM)
    for os_ in (1, 3):
        f = _t(np.full((nz, ny, nx), 0.25, np.float32), cuda)
        ops.voxelize_(f, solids, vw, vh, x0, y0, z0, oversampling=os_)
        assert np.array_equal(f.cpu().numpy(), z[f"f_os{os_}"])
    arr = (petl_solid * len(solids))(*solids)
    lib().petl_solids_scale(arr, len(solids), 1.25, 0.8, 1.1)
    f = _t(np.full((nz, ny, nx), 0.25, np.float32), cuda)
    ops.voxelize_(f, list(arr), vw, vh, x0, y0, z0)
    assert np.array_equal(f.cpu().numpy(), z["f_scaled"])
    solids2 = _product_solids(PHANTOM2)
    for os_ in (1, 5):
        f = _t(np.zeros((nz, ny, nx), np.float32), cuda)
        ops.voxelize_(f, solids2, vw, vh, x0, y0, z0, oversampling=os_)
        assert np.array_equal(f.cpu().numpy(), z[f"f2_os{os_}"])


def test_cabi_voxelize_matches_reference(cuda):
    from petl_b200 import PETLserver
    z = load_golden("voxelize.npz")
    nx, ny, nz = (int(v) for v in z["volume"][:3])
    s = PETLserver()
    s.set_volume(nx, ny, nz, float(z["volume"][3]), float(z["volume"][4]))
    for t, c, r, v, A, clip in PHANTOM:
        assert s.add_object(t, c, r, v, A, clip)
    f = np.full((nz, ny, nx), 0.25, np.float32)
    s.voxelize(f, 3)
    assert np.array_equal(f, z["f_os3"])
    s.scale_phantom(np.array([1.25, 0.8, 1.1]))
    f = np.full((nz, ny, nx), 0.25, np.float32)
    s.voxelize(f)
    assert np.array_equal(f, z["f_scaled"])
    # names as the reference's add_object takes them
    s.clear_phantom()
    assert s.add_object("sphere", 0.0, 5.0, 1.0) and not s.add_object("torus", 0.0, 5.0, 1.0)


def _case(name):
    from petl_b200 import Geometry
    z = load_golden("raytrace.npz")
    vol = tuple(z[f"{name}_volume"])
    plans = z[f"{name}_planograms"]
    return z, plans, vol, [Geometry(*p, volume=vol) for p in plans], [O.make_geom(*p, vol) for p in plans]


@pytest.mark.parametrize("name", RT_CASES)
def test_device_ray_trace_matches_oracle_and_reference(cuda, name):
    from petl_b200 import ops, lib
    z, plans, vol, pg, og = _case(name)
    solids, osolids = _product_solids(PHANTOM), _oracle_solids(PHANTOM)
    _, D, L_, H, _, _, _ = plans[0]
    mods, omods = _product_solids(_modules(D, L_, H)), _oracle_solids(_modules(D, L_, H))
    for i, (G, Go) in enumerate(zip(pg, og)):
        for os_ in (1, 3):
            got = ops.ray_trace(G, solids, oversampling=os_).cpu().numpy()
            assert rel_l2(got, O.ray_trace(Go, osolids, os_)) < 1e-5
            assert rel_l2(got, z[f"{name}_rt{os_}_{i}"]) < 1e-5
        got2 = ops.ray_trace(G, _product_solids(PHANTOM2)).cpu().numpy()
        assert rel_l2(got2, O.ray_trace(Go, _oracle_solids(PHANTOM2), 1)) < 1e-5
        assert rel_l2(got2, z[f"{name}_rt2_{i}"]) < 1e-5
        sp = ops.ray_trace(G, mods, stopping_power=True).cpu().numpy()
        assert rel_l2(sp, O.ray_trace(Go, omods, 1, stopping_power=True)) < 1e-5
        assert rel_l2(sp, z[f"{name}_sp_{i}"]) < 1e-5
        assert sp.max() > 0.1
    assert lib().petl_device_error_flag() == 0


def test_cabi_ray_trace_and_stopping_power(cuda):
    """PETLserver through the C ABI: ray_trace and the raw stopping power
    against the reference; no modules gives a stopping power of 1; an empty
    phantom traces to 0."""
    from petl_b200 import PETLserver
    from petl_b200.server import _pp
    z, plans, vol, _, _ = _case("gpetx")
    s = PETLserver()
    for p in plans:
        s.add_planogram(*p)
    g = s.allocate_projections()
    for a in g:
        a[:] = 7.0
    assert s.libprojectors.stopping_power(_pp(g), 1)
    assert all(np.all(a == 1.0) for a in g)
    assert all(np.all(a == 0.0) for a in s.ray_trace())
    for t, c, r, v, A, clip in PHANTOM:
        s.add_object(t, c, r, v, A, clip)
    _, D, L_, H, _, _, _ = plans[0]
    for _, c, r, v, _, _ in _modules(D, L_, H):
        assert s.add_module(c, r, v)
    rt = s.ray_trace(oversampling=3)
    g = s.allocate_projections()
    assert s.libprojectors.stopping_power(_pp(g), 1)
    for i in range(len(plans)):
        assert rel_l2(rt[i], z[f"gpetx_rt3_{i}"]) < 1e-5
        assert rel_l2(g[i], z[f"gpetx_sp_{i}"]) < 1e-5
    # the server's stopping power is smoothed as the reference's
    sm = s.stopping_power()
    assert sm[0].shape == g[0].shape and not np.array_equal(sm[0], g[0])


def test_ray_trace_many_solids_on_one_line(cuda):
    """40 nested spheres: central lines hit more solids than a thread keeps,
    and the rescanning path gives the oracle's sums."""
    from petl_b200 import Geometry, ops
    args, vol = (0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), (32, 32, 8, 2.0)
    spec = [(0, (0.0, 0.0, 0.0), (r, r, 0.5 * r), 0.1 * (k % 3 + 1), None, None)
            for k, r in enumerate(np.linspace(16.0, 0.5, 40))]
    G, Go = Geometry(*args, volume=vol), O.make_geom(*args, vol)
    got = ops.ray_trace(G, _product_solids(spec)).cpu().numpy()
    want = O.ray_trace(Go, _oracle_solids(spec))
    assert rel_l2(got, want) < 1e-5
    assert got.max() > 0.0


def test_reference_geometry_demo_end_to_end(cuda):
    """The reference's demo/d01_set_geometry.py through PETLserver: six
    planograms at psi 0..150 degrees, the default volume, two ellipsoids
    ray-traced and reconstructed by FBP.  The volume is held to the
    reference's within 5e-4 relative L2 (its backprojector interpolates with
    8-bit texture weights), and the traced planograms' sums to 1e-5."""
    from petl_b200 import PETLserver
    z = load_golden("demo_d01.npz")
    s = PETLserver()
    for psi, D, L_, H, T, vm0, vm1 in z["planograms"]:
        s.add_planogram(psi, D, L_, H, T, vm0, vm1)
    s.set_default_volume()
    nx, ny, nz, vw, vh = z["volume"]
    assert (s.numX(), s.numY(), s.numZ()) == (int(nx), int(ny), int(nz))
    s.add_object("ellipsoid", [0.0, 0.0, 0.0], [90.0, 80.0, 70.0], 100.0)
    s.add_object("ellipsoid", [0.0, 0.0, 0.0], [5.0, 5.0, 5.0], 1000.0)
    g = s.allocate_projections()
    s.ray_trace(g)
    for gi, want in zip(g, z["g_sums"]):
        assert abs(gi.sum(dtype=np.float64) / want - 1.0) < 1e-5
    f = s.allocate_volume()
    s.FBP(g, f)
    assert rel_l2(f, z["f"]) < 5e-4


def test_calc_response_device_composition_equals_host_calls(cuda):
    """calc_response composes the stopping power, the Gaussian and the
    solid-angle model on the GPU; it must equal the same three steps through
    the C ABI on host arrays bit for bit, with and without modules."""
    from petl_b200 import PETLserver
    from petl_b200.server import _pp
    z, plans, vol, _, _ = _case("gpetx")
    s = PETLserver()
    for p in plans:
        s.add_planogram(*p)
    for with_modules in (False, True):
        if with_modules:
            _, D, L_, H, _, _, _ = plans[0]
            for _, c, r, v, _, _ in _modules(D, L_, H):
                s.add_module(c, r, v)
        R = s.calc_response(oversampling=3)
        g = s.allocate_projections()
        assert s.libprojectors.stopping_power(_pp(g), 3)
        s.gaussian_filter(g, 0.6571)
        s.apply_solid_angle_model(g)
        for a, b in zip(R, g):
            assert np.array_equal(a, b)

"""Planogram corrections on the GPU against the oracle and the reference.

The solid-angle factors come from the reference's own host arithmetic and
the device multiply is one rounding, so the results are bit-exact.
apply_corrections divides, selects medians and copies values, all exact
operations, so the device result must equal the oracle bit for bit too: on
the reference's golden case, on random inputs with clustered bad pixels (the
oracle's windows read the divided values before any in-fill, as the kernel
does), on projections too large for the kernel's shared-memory stage, and on
edge cases (no bad pixels, every pixel bad, zero responses).
"""
import numpy as np
import pytest

import oracle as O
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)


def _geoms(plans, vol):
    from petl_b200 import Geometry
    return [Geometry(*p, volume=vol) for p in plans], [O.make_geom(*p, vol) for p in plans]


@pytest.mark.parametrize("name", ["sa_g0", "sa_g0t1", "sa_gpetx", "sa_bench"])
@pytest.mark.parametrize("inverse", [False, True])
def test_device_solid_angle_matches_reference(cuda, name, inverse):
    from petl_b200 import ops, lib
    z = load_golden("solid_angle.npz")
    vol = tuple(z[f"{name}_volume"])
    pg, _ = _geoms(z[f"{name}_planograms"], vol)
    rng = np.random.default_rng(11)
    for i, G in enumerate(pg):
        tab = z[f"{name}_c{int(inverse)}_{i}"]
        x = rng.random(G.shape, dtype=np.float32)
        got = ops.solid_angle_(G, _t(x, cuda), inverse=inverse).cpu().numpy()
        assert np.array_equal(got, x * tab[:, :, None, None])
    assert lib().petl_device_error_flag() == 0


def test_cabi_solid_angle_matches_reference(cuda):
    """PETLserver.apply_solid_angle_model (host arrays through the C ABI) on
    the bench geometry's ones gives the reference's factors."""
    from petl_b200 import PETLserver
    z = load_golden("solid_angle.npz")
    s = PETLserver()
    for p in z["sa_gpetx_planograms"]:
        s.add_planogram(*p)
    model = s.apply_solid_angle_model()
    corr = s.apply_solid_angle_correction()
    for i in range(2):
        assert np.array_equal(model[i], np.broadcast_to(z[f"sa_gpetx_c1_{i}"][:, :, None, None], model[i].shape))
        assert np.array_equal(corr[i], np.broadcast_to(z[f"sa_gpetx_c0_{i}"][:, :, None, None], corr[i].shape))


def _random_case(shape, rng, bad_frac=0.05, distinct=False, zero_frac=0.01):
    lam = rng.uniform(0.05, 3.0, size=shape[:2])[:, :, None, None]
    g = rng.poisson(lam, size=shape).astype(np.float32)
    if distinct == "few":
        # three response values: the median's bucket outgrows the kernel's list
        r = rng.choice(np.array([1.0, 1.25, 1.5], np.float32), size=shape)
    elif distinct:
        r = rng.uniform(0.5, 1.5, size=shape).astype(np.float32)
    else:
        r = (rng.integers(48, 97, size=shape) / 64.0).astype(np.float32)
    u = rng.random(shape)
    # clustered bad pixels: whole 2x3 blocks around random seeds
    seeds = u < bad_frac / 6
    bad = seeds.copy()
    for dj, dk in ((0, 1), (0, 2), (1, 0), (1, 1), (1, 2)):
        bad |= np.roll(np.roll(seeds, dj, axis=2), dk, axis=3)
    r[bad] *= np.float32(0.25)
    r[u > 1.0 - zero_frac] = 0.0
    return g, r


@pytest.mark.parametrize("args,distinct", [
    ((0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), False),
    ((0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25), True),
    ((90.0, 48.0, 24.0, 16.0, 1.0, 0.5, 0.25), False),
    # 256 x 266 bins per projection: more than the shared-memory stage holds
    ((0.0, 128.0, 64.0, 64.0, 0.25, 0.02, 0.01), True),
    # 30 bins per row: rows are not whole float4s (the scalar staging path)
    ((0.0, 64.0, 30.0, 16.0, 2.0, 0.5, 0.25), True),
    # 128 x 140 bins with three response values
    ((0.0, 256.0, 128.0, 128.0, 1.0, 0.05, 0.02), "few"),
])
def test_device_apply_corrections_matches_oracle(cuda, args, distinct):
    from petl_b200 import Geometry, ops, lib
    vol = (32, 32, 8, 2.0)
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(int(args[1] + 10 * args[4]))
    g, r = _random_case(G.shape, rng, distinct=distinct)
    want = O.apply_corrections([Go], [g], [r], 0.75)[0]
    got = ops.apply_corrections_(G, _t(g, cuda), _t(r, cuda), 0.75).cpu().numpy()
    assert np.array_equal(got, want), int((got != want).sum())
    # the case holds zeroed, in-filled and divided bins
    plain = np.where(r == 0, 0, g / np.where(r == 0, 1, r))
    assert np.any((got != plain) & (got != 0))
    assert lib().petl_device_error_flag() == 0


def test_device_apply_corrections_edges(cuda):
    from petl_b200 import Geometry, ops
    args, vol = (0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), (32, 32, 8, 2.0)
    G = Geometry(*args, volume=vol)
    Go = O.make_geom(*args, vol)
    rng = np.random.default_rng(3)
    g = rng.poisson(2.0, size=G.shape).astype(np.float32)
    cases = {
        "uniform r: nothing below threshold": np.ones(G.shape, np.float32),
        "zero r everywhere": np.zeros(G.shape, np.float32),
        # a negative response: every bin of projection (3, 5) lies below
        # 0.75 * median = -0.75, and its divided values are -g (signed zeros)
        "one projection all bad": None,
        # every bin below the threshold; few windows hold values above it
        "threshold above every value": "thr",
    }
    for label, r in cases.items():
        thr = 0.75
        if r is None:
            r = np.ones(G.shape, np.float32)
            r[3, 5] = -1.0
        elif isinstance(r, str):
            r = rng.uniform(0.5, 1.0, size=G.shape).astype(np.float32)
            thr = 10.0
        want = O.apply_corrections([Go], [g], [r], thr)[0]
        got = ops.apply_corrections_(G, _t(g, cuda), _t(r, cuda), thr).cpu().numpy()
        assert np.array_equal(got, want), label


@pytest.mark.parametrize("name", ["g0", "g0t1", "gpetx"])
def test_cabi_apply_corrections_matches_reference(cuda, name):
    """The C ABI's apply_corrections on the reference's golden case (host
    arrays in and out) reproduces the reference's output bit for bit."""
    from petl_b200 import PETLserver
    z = load_golden("corrections.npz")
    s = PETLserver()
    for p in z[f"{name}_planograms"]:
        s.add_planogram(*p)
    n = len(z[f"{name}_planograms"])
    g = [z[f"{name}_g{i}"].copy() for i in range(n)]
    r = [z[f"{name}_r{i}"] for i in range(n)]
    s.set_response(r)
    s.apply_corrections(g)
    for i in range(n):
        plain = np.where(r[i] == 0, np.float32(0), z[f"{name}_g{i}"] / np.where(r[i] == 0, np.float32(1), r[i]))
        want = plain.astype(np.float32).ravel()
        want[z[f"{name}_idx{i}"]] = z[f"{name}_val{i}"]
        assert np.array_equal(g[i].ravel(), want)

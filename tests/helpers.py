"""Shared test helpers: golden-fixture geometry and seeded phantoms."""
import numpy as np

import oracle as O


def oracle_geoms(z):
    vol = tuple(z["volume"])
    return [O.make_geom(p[0], p[1], p[2], p[3], p[4], p[5], p[6], vol) for p in z["planograms"]]


def product_geoms(z):
    from petl_b200 import Geometry
    vol = tuple(z["volume"])
    out = []
    for p in z["planograms"]:
        psi, D, L, H, T, vm0, vm1 = p
        out.append(Geometry(psi, D, L, H, T, vm0, vm1, volume=vol))
    return out


def ellipsoids(shape, vox, rng, n, vmin=0.1, vmax=1.0, background=0.0, axes=None):
    """Seeded ellipsoid phantom, later objects replace earlier ones."""
    nz, ny, nx = shape
    wx, wz = vox
    x = (np.arange(nx) - 0.5 * (nx - 1)) * wx
    y = (np.arange(ny) - 0.5 * (ny - 1)) * wx
    z = (np.arange(nz) - 0.5 * (nz - 1)) * wz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    f = np.full(shape, background, np.float32)
    ext = np.array([nx * wx, ny * wx, nz * wz]) * 0.5
    for _ in range(n):
        if axes is None:
            r = rng.uniform(0.08, 0.3, 3) * ext
        else:
            r = np.minimum(rng.uniform(axes[0], axes[1], 3), ext * 0.95)
        c = rng.uniform(-1, 1, 3) * np.maximum(ext - r, 0)
        val = rng.uniform(vmin, vmax)
        inside = ((X - c[0]) / r[0]) ** 2 + ((Y - c[1]) / r[1]) ** 2 + ((Z - c[2]) / r[2]) ** 2 <= 1.0
        f[inside] = val
    return f

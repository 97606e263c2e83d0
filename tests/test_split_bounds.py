"""Host-side bounds of the split kernels for any psi, checked on the CPU
against a float64 restatement of the footprint rules (the reference's
plane taps and box overlaps, src/projectors.cu:85-168, and the
backprojector's voxel extents, src/projectors.cu:318-345):

* the exact adjoint's x gather (k_gxT) takes, for voxel a on plane p, the
  u0 columns within (fw + 1/2) |r_p trig| + 1/2 of the ray through the
  voxel centre: every column whose forward taps give the voxel a positive
  weight must lie inside, and no column may have more than four taps;
* the reference-semantics backprojector (k_rbp_xy) stages, per 16 x 16
  tile and view, W columns from one below the smallest first bin of the
  tile's corners, W from the host formula (15 T_x (|wx| + |wy|) + width) /
  T_u0 + 4, rounded up to a power of two: every voxel's bin range must lie
  inside;
* the z passes (k_gz, k_gzT) stage per plane or slope the rows their tile
  needs from a host bound on the spread of the per-column shifts: over a
  sweep of further geometries the actual spread stays within it."""
import math

import numpy as np
import pytest

from test_gpu_gsplit import CASES as GCASES

CASES = dict(GCASES)
CASES.update({
    "p30pitch": ((30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (40, 40, 12, 1.5, 1.25)),
    "p75wide": ((75.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.25), (40, 44, 12, 1.9, 1.0, 1.0, -2.0, 0.5)),
    "p0pitch": ((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (44, 40, 12, 1.0, 1.5, 0.5, -1.0, 0.0)),
})


def _fields(name):
    from petl_b200 import Geometry
    args, vol = CASES[name]
    P = Geometry(*args, volume=vol).g
    return {k: getattr(P, k) for k, _ in P._fields_}


@pytest.mark.parametrize("name", list(GCASES))
def test_adjoint_x_gather_window_holds_every_tap(name):
    F = _fields(name)
    cs, sn, Tx, Tu0, u0_0 = F["cos_psi"], F["sin_psi"], F["T_x"], F["T_u0"], F["u0_0"]
    iu = np.arange(F["N_u0"], dtype=np.float64)
    u0 = u0_0 + iu * Tu0
    worst = 0.0
    for iv0 in range(F["N_v0"]):
        v0 = F["v0_0"] + iv0 * F["T_v0"]
        rx, ry = -(v0 * cs + sn), -(v0 * sn - cs)
        xd = abs(rx) >= abs(ry)
        trig = sn if xd else cs
        inv = 1.0 / (rx if xd else ry)
        width = 0.5 * Tu0 * abs(trig)
        fw = 0.5 * Tx / abs(trig) / Tu0
        h = (fw + 0.5) * abs((rx if xd else ry) * trig) + 0.5
        NP, NA = (F["numX"], F["numY"]) if xd else (F["numY"], F["numX"])
        p0, a0 = (F["x_0"], F["y_0"]) if xd else (F["y_0"], F["x_0"])
        for p in range(NP):
            pc = p0 + p * Tx
            t = (pc - (u0 * cs if xd else u0 * sn)) * inv
            ac = (u0 * sn + t * ry) if xd else (u0 * cs + t * rx)
            amin = np.maximum(0, np.ceil((ac - width - 0.5 * Tx - a0) / Tx)).astype(int)
            amax = np.minimum(NA - 1, np.floor((ac + width + 0.5 * Tx - a0) / Tx)).astype(int)
            assert int(np.max(amax - amin + 1)) <= 4
            for j in range(4):
                a = amin + j
                ok = a <= amax
                q = (a0 + a * Tx) - t * (ry if xd else rx)
                c = (q / trig - u0_0) / Tu0
                w = np.minimum(iu + 0.5, c + fw) - np.maximum(iu - 0.5, c - fw)
                hit = ok & (w > 0)
                if not hit.any():
                    continue
                x, y = (pc, a0 + a * Tx) if xd else (a0 + a * Tx, pc)
                cc = (x * ry - y * rx - u0_0) / Tu0  # the voxel centre's u0 bin
                worst = max(worst, float(np.max(np.abs(iu - cc)[hit])) / h)
    assert worst < 0.9  # margin for the kernel's float evaluation


@pytest.mark.parametrize("name", list(CASES))
def test_reference_backprojector_tile_window_holds_every_extent(name):
    F = _fields(name)
    cs, sn, Tx, Tu0, u0_0 = F["cos_psi"], F["sin_psi"], F["T_x"], F["T_u0"], F["u0_0"]
    nx, ny = F["numX"], F["numY"]
    views = [F["v0_0"] + k * F["T_v0"] for k in range(F["N_v0"])]
    need = 0.0
    for v0 in views:
        wy, wx = abs(v0 * cs + sn), abs(-v0 * sn + cs)
        width = Tx * max(wy, wx) / Tu0
        need = max(need, 15 * Tx * (wx + wy) / Tu0 + width)
    W = 1 << max(4, math.ceil(math.log2(math.ceil(need + 4.0))))
    xs = F["x_0"] + np.arange(nx) * Tx
    ys = F["y_0"] + np.arange(ny) * Tx
    X, Y = np.meshgrid(xs, ys)
    T = Y * cs - X * sn
    XDT = X * cs + Y * sn
    for v0 in views:
        wy, wx = v0 * cs + sn, -v0 * sn + cs
        ydom = abs(wy) > abs(wx)
        hx, ht = (0.5 * Tx * sn, 0.5 * Tx * cs) if ydom else (0.5 * Tx * cs, -0.5 * Tx * sn)
        lo_ = (XDT - hx + v0 * (T - ht) - u0_0) / Tu0
        hi_ = (XDT + hx + v0 * (T + ht) - u0_0) / Tu0
        pos = (wy if ydom else wx) >= 0
        A, B = (lo_, hi_) if pos else (hi_, lo_)
        umin = np.maximum(np.ceil(A - 0.5), 0)
        umax = np.minimum(np.floor(B + 0.5), F["N_u0"] - 1)
        for ty in range(0, ny, 16):
            for tx in range(0, nx, 16):
                sl = (slice(ty, min(ty + 16, ny)), slice(tx, min(tx + 16, nx)))
                corners = A[[ty, ty, min(ty + 15, ny - 1), min(ty + 15, ny - 1)],
                            [tx, min(tx + 15, nx - 1), tx, min(tx + 15, nx - 1)]]
                lo = max(0, math.ceil(float(corners.min()) - 0.5) - 1)
                live = umax[sl] >= umin[sl]
                if not live.any():
                    continue
                assert float(umin[sl][live].min()) >= lo
                assert float(umax[sl][live].max()) - lo < W


# geometries beyond the GPU tests' ones: angles near the x/y-driven tie,
# steep slopes (v_m1 up to 0.45), u0 pitch unequal to the voxel width,
# off-centre volumes
SWEEP = [
    ((15.0, 200.0, 100.0, 50.0, 1.0, 0.5, 0.45), (96, 80, 48, 1.0, 1.0, 3.0, -2.0, 1.0)),
    ((44.0, 160.0, 80.0, 40.0, 2.0, 0.5, 0.3), (64, 64, 40, 2.0)),
    ((46.0, 160.0, 80.0, 40.0, 1.5, 0.45, 0.25), (80, 72, 48, 1.5)),
    ((60.0, 256.0, 128.0, 64.0, 1.0, 0.5, 0.25), (128, 128, 64, 1.0)),
    ((100.0, 128.0, 64.0, 32.0, 1.0, 0.5, 0.35), (48, 64, 32, 1.25, 1.0, -4.0, 2.0, 0.0)),
    ((150.0, 300.0, 120.0, 60.0, 2.0, 0.4, 0.2), (96, 96, 30, 2.0, 2.0, 0.0, 0.0, 5.0)),
]


def _sweep_fields(i):
    from petl_b200 import Geometry
    args, vol = SWEEP[i]
    P = Geometry(*args, volume=vol).g
    return {k: getattr(P, k) for k, _ in P._fields_}


def _views(F):
    """Per view: x-driven, 1/r_p, pscale (the u0 coordinate's factor on the
    driving axis), as the kernels' ray_geom forms them."""
    cs, sn = F["cos_psi"], F["sin_psi"]
    out = []
    for iv0 in range(F["N_v0"]):
        v0 = F["v0_0"] + iv0 * F["T_v0"]
        rx, ry = -(v0 * cs + sn), -(v0 * sn - cs)
        xd = abs(rx) >= abs(ry)
        out.append((xd, 1.0 / (rx if xd else ry), cs if xd else sn))
    return out


@pytest.mark.parametrize("i", range(len(SWEEP)))
def test_z_pass_staged_rows_hold_the_shift_spread(i):
    """The z passes stage, per plane (forward) or slope (adjoint), the rows
    a tile needs: its rows + the spread of floor((u1_0 - z_0 - t v1) / T_u1)
    over the tile + 5, the spread bounded on the host by
    (dt vmax + tmax dv1 + dt dv1) / T_u1 (forward: 32 columns x 16 slopes;
    adjoint: 32 columns x 16 planes).  The actual spread of the floors over
    every tile must stay within the bound + 1."""
    F = _sweep_fields(i)
    T_u1, T_x, T_u0 = F["T_u1"], F["T_x"], F["T_u0"]
    v1 = F["v1_0"] + np.arange(F["N_v1"]) * F["T_v1"]
    K = (F["u1_0"] - F["z_0"]) / T_u1
    vmax = float(np.max(np.abs(v1)))
    ext = max(abs(F["x_0"]), abs(F["x_0"] + (F["numX"] - 1) * T_x), abs(F["y_0"]),
              abs(F["y_0"] + (F["numY"] - 1) * T_x))
    uext = max(abs(F["u0_0"]), abs(F["u0_0"] + (F["N_u0"] - 1) * T_u0))
    views = _views(F)
    tmax = max((ext + uext * abs(ps)) * abs(inv) for _, inv, ps in views)
    dtmax = max(32 * T_u0 * abs(ps) * abs(inv) for _, inv, ps in views)
    bound_fwd = (dtmax * vmax + tmax * 15 * abs(F["T_v1"]) + dtmax * 15 * abs(F["T_v1"])) / T_u1
    u0 = F["u0_0"] + np.arange(F["N_u0"]) * T_u0
    for xd, inv, ps in views:
        NP = F["numX"] if xd else F["numY"]
        pc = (F["x_0"] if xd else F["y_0"]) + np.arange(NP) * T_x
        t = (pc[:, None] - u0[None, :] * ps) * inv  # [plane][u0]
        dt_view = (15 * T_x + 31 * T_u0 * abs(ps)) * abs(inv)
        bound_adj = dt_view * vmax / T_u1
        for c0 in range(0, F["N_u0"], 32):
            tc = t[:, c0:c0 + 32]
            # forward: per plane, over the tile's columns and 16 slopes
            for s0 in range(0, F["N_v1"], 16):
                nc = K - tc[:, :, None] * (v1[s0:s0 + 16] / T_u1)[None, None, :]
                fl = np.floor(nc)
                spread = fl.max(axis=(1, 2)) - fl.min(axis=(1, 2))
                assert float(spread.max()) <= math.ceil(bound_fwd) + 1
            # adjoint: per slope, over the tile's columns and 16 planes
            for p0 in range(0, NP, 16):
                nc = K - tc[p0:p0 + 16, :, None] * (v1 / T_u1)[None, None, :]
                fl = np.floor(nc)
                spread = fl.max(axis=(0, 1)) - fl.min(axis=(0, 1))
                assert float(spread.max()) <= math.ceil(bound_adj) + 1

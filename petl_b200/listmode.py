"""List-mode coincidence data: the reference's two file formats and a seeded
synthetic source.

The reference bins list-mode files through ``bin(float** g, char* file)``
(src/petl_c_interface.h:55, src/binning.cpp:558-660):

* files ending in ``.lst``: records of two events, each ``float pos[4]``
  (x, y, z in mm, energy) then ``uint64 time`` (48 bytes per coincidence,
  src/binning.cpp:10-19, 67-151);
* any other name: ``int64 N`` then per coincidence, for blue then pink,
  ``int16 n_interactions``, ``float pos[3]``, ``float energy`` and
  ``n_interactions - 1`` further interaction records of 18 bytes that are
  skipped (src/binning.cpp:575-612).

z is measured from the chest wall (the bottom edge of the panels): the
binning shifts u1 by the panel half-height.  Positions are in mm.

``coincidences`` draws seeded events for a dual-panel geometry: emission
points inside a box, isotropic directions, kept when both ends hit the
panels (half-lengths L x H at distance R from the centre, rotated by psi).
"""
import numpy as np


def coincidences(n, rng, R, L, H, psi_deg=0.0, box=(20.0, 20.0, 10.0), chest_wall=True):
    """n coincidences (blue, pink), each (n, 3) float32 in mm, on the panels
    of one planogram (half-lengths R, L, H); blue and pink are assigned to
    the two panels at random."""
    psi = np.deg2rad(psi_deg)
    c, s = np.cos(psi), np.sin(psi)
    blue = np.empty((0, 3), np.float32)
    pink = np.empty((0, 3), np.float32)
    while len(blue) < n:
        m = 2 * (n - len(blue)) + 64
        e = rng.uniform(-1.0, 1.0, (m, 3)) * np.asarray(box)
        d = rng.standard_normal((m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        # panel frame: y' along the panel normal, x' along the panel
        ey = -s * e[:, 0] + c * e[:, 1]
        dy = -s * d[:, 0] + c * d[:, 1]
        ok = np.abs(dy) > 1e-3
        tp = (R - ey) / np.where(ok, dy, 1.0)
        tm = (-R - ey) / np.where(ok, dy, 1.0)
        Pp = e + tp[:, None] * d
        Pm = e + tm[:, None] * d
        for P in (Pp, Pm):
            xp = c * P[:, 0] + s * P[:, 1]
            ok &= (np.abs(xp) <= L) & (np.abs(P[:, 2]) <= H)
        Pp, Pm = Pp[ok], Pm[ok]
        swap = rng.random(len(Pp)) < 0.5
        b = np.where(swap[:, None], Pm, Pp)
        p = np.where(swap[:, None], Pp, Pm)
        if chest_wall:
            b[:, 2] += H
            p[:, 2] += H
        blue = np.concatenate([blue, b.astype(np.float32)])
        pink = np.concatenate([pink, p.astype(np.float32)])
    return blue[:n], pink[:n]


def interaction_counts(n, rng, extra):
    """Interactions per side (int16, >= 1): a fraction `extra` of the events
    carries 1-2 further interactions, which the binning skips."""
    nb = 1 + (rng.random(n) < extra) * rng.integers(1, 3, n)
    npk = 1 + (rng.random(n) < extra) * rng.integers(1, 3, n)
    return nb.astype(np.int16), npk.astype(np.int16)


def write_acq(path, blue, pink, counts=None):
    """Binary coincidence file (the non-``.lst`` format); `counts` = (blue,
    pink) interactions per event (default one each)."""
    blue = np.asarray(blue, np.float32)
    pink = np.asarray(pink, np.float32)
    n = len(blue)
    nb = np.ones(n, np.int16) if counts is None else np.asarray(counts[0], np.int16)
    npk = np.ones(n, np.int16) if counts is None else np.asarray(counts[1], np.int16)
    if (nb == 1).all() and (npk == 1).all():  # fixed 36-byte records
        rec = np.zeros(n, dtype=[("nb", "<i2"), ("b", "<f4", 4), ("np", "<i2"), ("p", "<f4", 4)])
        rec["nb"] = 1
        rec["np"] = 1
        rec["b"][:, :3] = blue
        rec["b"][:, 3] = 511.0
        rec["p"][:, :3] = pink
        rec["p"][:, 3] = 511.0
        with open(path, "wb") as fh:
            fh.write(np.int64(n).tobytes())
            fh.write(rec.tobytes())
        return
    parts = [np.int64(n).tobytes()]
    junk = np.zeros(1, dtype=[("n", "<i2"), ("v", "<f4", 4)])
    for i in range(n):
        for cnt, pos in ((nb[i], blue[i]), (npk[i], pink[i])):
            parts.append(np.int16(cnt).tobytes())
            parts.append(np.asarray([pos[0], pos[1], pos[2], 511.0], np.float32).tobytes())
            for _ in range(int(cnt) - 1):
                junk["n"] = 1
                junk["v"] = (1.0, 2.0, 3.0, 100.0)
                parts.append(junk.tobytes())
    with open(path, "wb") as fh:
        fh.write(b"".join(parts))


def write_lst(path, blue, pink, energy=511.0):
    """``.lst`` coincidence file: 48-byte records (pos[4] + uint64 time per
    event)."""
    blue = np.asarray(blue, np.float32)
    pink = np.asarray(pink, np.float32)
    rec = np.zeros(len(blue), dtype=[("b", "<f4", 4), ("bt", "<u8"), ("p", "<f4", 4), ("pt", "<u8")])
    rec["b"][:, :3] = blue
    rec["b"][:, 3] = energy
    rec["p"][:, :3] = pink
    rec["p"][:, 3] = energy
    rec["bt"] = np.arange(len(blue), dtype=np.uint64)
    rec["pt"] = rec["bt"]
    with open(path, "wb") as fh:
        fh.write(rec.tobytes())

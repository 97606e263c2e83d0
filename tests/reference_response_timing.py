"""Times the detector stopping power of the PET/X scanner preset (two
planograms, psi 0 and 90 degrees, and its 120 crystal blocks,
src/petx_server.py:9-42) through the reference C ABI of the reference library
(oracle/_ref/libpetl_ref.so, built from the reference sources by
``make -C oracle ref``; its stoppingPowerKernel runs on the GPU) and of this
library, on host arrays, and compares the two planogram sets.

    python tests/reference_response_timing.py > response_timing.json

Times are host wall-clock per call (the reference: one call; this
library: best of 2 after a warm-up).  The device-only time of this
library's kernel is taken with CUDA events.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import Ref, ptr  # noqa: E402

PITCH = 1.6
PLANOGRAMS = [(0.0, 101.0, 251.52, 156.72, PITCH), (90.0, 266.6, 125.12, 156.72, PITCH)]


def v_m1(D, H, T):
    return min(1.0, (H - 1.5 * T) / D)  # src/petl_server.py:498-501


def main():
    import torch
    from petl_b200 import PETLserver, ops
    from petl_b200.server import _pp, petx_modules
    mods = petx_modules()
    res = {"workload": "PET/X preset: planograms psi 0 (D 101, L 251.52, H 156.72) and psi 90 (D 266.6, "
                       "L 125.12, H 156.72), T 1.6 mm, v_m0 1; 120 crystal blocks (0.0815 / mm)",
           "modules": len(mods)}
    s = PETLserver()
    for psi, D, L_, H, T in PLANOGRAMS:
        s.add_planogram(psi, D, L_, H, T)
    for c, r in mods:
        s.add_module(c, r)
    shapes = [tuple(int(v) for v in s.get_planogramSize(i)) for i in range(2)]
    res["shapes"] = shapes
    res["bins"] = int(sum(np.prod(sh) for sh in shapes))
    g = [torch.empty(sh, dtype=torch.float32).pin_memory().numpy() for sh in shapes]
    s.libprojectors.stopping_power(_pp(g), 1)
    ts = []
    for _ in range(2):
        t0 = time.perf_counter()
        s.libprojectors.stopping_power(_pp(g), 1)
        ts.append(time.perf_counter() - t0)
    res["ours_cabi_s"] = min(ts)
    # device-only
    geoms = s.geometries_from_model()
    solids = [ops.make_solid(1, c, r, 0.0815) for c, r in mods]
    out = [torch.empty(G.shape, device="cuda") for G in geoms]
    ops.ray_trace(geoms, solids, g=out, stopping_power=True)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ops.ray_trace(geoms, solids, g=out, stopping_power=True)
    b.record()
    torch.cuda.synchronize()
    res["ours_device_s"] = a.elapsed_time(b) * 1e-3
    res["ours_device_lines_per_s"] = res["bins"] / res["ours_device_s"]
    # the reference
    ref = Ref()
    m = ref.L.create_new_model()
    ref.L.set_model(m)
    for psi, D, L_, H, T in PLANOGRAMS:
        ref.L.add_planogram(psi, D, L_, H, 1.0, v_m1(D, H, T), T)
    eye, zero = np.eye(3, dtype=np.float32), np.zeros(3, np.float32)
    for c, r in mods:
        ref.L.add_module(1, ptr(np.array(c, np.float32)), ptr(np.array(r, np.float32)), 0.0815, ptr(eye), ptr(zero))
    assert [tuple(x) for x in ref.shapes()] == shapes
    gr = [np.zeros(sh, np.float32) for sh in ref.shapes()]
    t0 = time.perf_counter()
    ref.L.stopping_power(ref.pp(gr), 1)
    res["reference_cabi_s"] = time.perf_counter() - t0
    res["speedup_cabi"] = res["reference_cabi_s"] / res["ours_cabi_s"]
    res["rel_l2_ours_vs_reference"] = [float(np.linalg.norm(x.astype(np.float64) - y) / np.linalg.norm(y))
                                       for x, y in zip(g, gr)]
    print(json.dumps(res))


if __name__ == "__main__":
    main()

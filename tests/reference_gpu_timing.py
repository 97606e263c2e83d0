"""Times the reference library's own GPU projector and backprojector (test
infrastructure; compiled from the reference sources by ``make -C oracle
ref`` into oracle/_ref/libpetl_ref.so) next to this library's, both through
the reference C ABI on host arrays, on the 256x256x128 / (65,129,128,256)
workload and on the 128x128x64 / (33,65,64,128) one.

    python tests/reference_gpu_timing.py > ref_timing.json

Each call of the reference C ABI copies the volume and the planogram
between host and device and launches one kernel per v1 slice; the same
calls of libpetl.so stage the host arrays through pinned, pipelined slabs.
Times are host wall-clock per call (best of ``reps`` after one warm-up).
Kernel-only reference times come from an ncu launch list of this script.
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import Ref, ellipsoids, ptr  # noqa: E402

CASES = {
    "256x256x128": ((0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25), (256, 256, 128, 1.0, 1.0, 0.0, 0.0, 0.0)),
    "128x128x64": ((0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0, 2.0, 0.0, 0.0, 0.0)),
}


def best(fn, reps):
    fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ok = fn()
        ts.append(time.perf_counter() - t0)
        if ok is False:
            raise RuntimeError("call failed")
    return min(ts)


def time_lib(L, plan, vol, reps, pp):
    m = L.create_new_model()
    L.set_model(m)
    psi, D, Lp, H, T, vm0, vm1 = plan
    assert L.add_planogram(psi, D, Lp, H, vm0, vm1, T)
    assert L.set_volume(*vol)
    s = (ctypes.c_int * 4)()
    L.get_planogramSize(0, s)
    shape = tuple(s)
    nz, ny, nx = vol[2], vol[1], vol[0]
    f = ellipsoids((nz, ny, nx), (vol[3], vol[4]), np.random.default_rng(0), 12)
    g = np.zeros(shape, np.float32)
    b = np.zeros((nz, ny, nx), np.float32)
    tf = best(lambda: L.project(pp([g]), ptr(f)), reps)
    tb = best(lambda: L.backproject(pp([g]), ptr(b)), reps)
    return {"shape": list(shape), "project_s": tf, "backproject_s": tb, "pairs_per_s": 1.0 / (tf + tb)}


def main():
    reps = int(sys.argv[1]) if len(sys.argv) > 1 else 3
    ref = Ref()
    out = {"what": "reference C ABI on host arrays, wall-clock per call (best of %d)" % reps}
    # this library through the same C ABI, same argument types
    mine = Ref(os.path.join(ROOT, "petl_b200", "libpetl.so"))
    for name, (plan, vol) in CASES.items():
        out["reference_" + name] = time_lib(ref.L, plan, vol, reps, Ref.pp)
        out["petl_b200_" + name] = time_lib(mine.L, plan, vol, reps, Ref.pp)
    print(json.dumps(out))


if __name__ == "__main__":
    main()

"""Times the reference's list-mode workflow demo (demo/d02_bin_and_reconstruct.py)
stage by stage through the reference C ABI of the reference library
(oracle/_ref/libpetl_ref.so, built from the reference sources by
``make -C oracle ref``) and of this library: the PET/X preset with its 120
crystal blocks, the response (stopping power, the 0.6571-bin Gaussian, the
solid-angle model; one line per bin), list-mode binning of a .lst file,
set_volume(120, 120, 120, 0.5), apply_corrections, FBP.  The demo's own
list-mode files are not available; a seeded file of coincidences on the
PET/X panels stands in (petl_b200.listmode, the reference's 48-byte .lst
records).

    python tests/reference_demo_timing.py [--events N] > demo_timing.json

Host wall-clock per stage, one run each after a warm-up of this library's
pipeline.  The reference's stopping power and Gaussian run on the GPU, its
binning and corrections partly on the host (16 cores here).
"""
import argparse
import ctypes
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import Ref, ptr  # noqa: E402

fpp = ctypes.POINTER(ctypes.POINTER(ctypes.c_float))


def ours(path):
    from petl_b200 import PETXserver
    t = {}
    s = PETXserver()
    s.print_warnings = False
    t0 = time.perf_counter()
    s.calc_response(1)
    t["calc_response"] = time.perf_counter() - t0
    g = s.allocate_projections()
    t0 = time.perf_counter()
    s.bin(path, g)
    t["bin"] = time.perf_counter() - t0
    s.set_volume(120, 120, 120, 0.5)
    f = s.allocate_volume()
    t0 = time.perf_counter()
    s.apply_corrections(g)
    t["apply_corrections"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    s.FBP(g, f)
    t["FBP"] = time.perf_counter() - t0
    return t, f, [x.copy() for x in s.response]


def reference(path):
    from petl_b200.server import petx_modules
    ref = Ref()
    L = ref.L
    L.gaussian_filter.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_float, ctypes.c_int]
    L.gaussian_filter.restype = ctypes.c_bool
    L.set_default_volume.argtypes = [ctypes.c_float]
    m = L.create_new_model()
    L.set_model(m)
    for psi, D, L_, H in ((0.0, 101.0, 251.52, 156.72), (90.0, 266.6, 125.12, 156.72)):
        L.add_planogram(psi, D, L_, H, 1.0, min(1.0, (H - 2.4) / D), 1.6)  # PETLserver defaults
    L.set_default_volume(1.0)
    eye, zero = np.eye(3, dtype=np.float32), np.zeros(3, np.float32)
    for c, r in petx_modules():
        L.add_module(1, ptr(np.array(c, np.float32)), ptr(np.array(r, np.float32)), 0.0815, ptr(eye), ptr(zero))
    shapes = ref.shapes()
    t = {}
    # PETLserver.calc_response(1): stopping_power (+ Gaussian), then the
    # solid-angle model applied to it (src/petl_server.py:578-605, 995-1055)
    t0 = time.perf_counter()
    R = [np.zeros(sh, np.float32) for sh in shapes]
    L.stopping_power(ref.pp(R), 1)
    for r in R:
        L.gaussian_filter(ptr(r), r.shape[0] * r.shape[1], r.shape[2], r.shape[3], 0.6571, 2)
    L.set_solid_angle_correction(ref.pp(R), True)
    t["calc_response"] = time.perf_counter() - t0
    g = [np.zeros(sh, np.float32) for sh in shapes]
    t0 = time.perf_counter()
    L.bin(ref.pp(g), path.encode())
    t["bin"] = time.perf_counter() - t0
    L.set_volume(120, 120, 120, 0.5, 0.5, 0.0, 0.0, 0.0)
    f = np.zeros((120, 120, 120), np.float32)
    t0 = time.perf_counter()
    L.apply_corrections(ref.pp(g), ref.pp(R), 0.75)
    t["apply_corrections"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    L.FBP(ref.pp(g), ptr(f))
    t["FBP"] = time.perf_counter() - t0
    return t, f, R


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--events", type=int, default=4_000_000)
    a = ap.parse_args()
    from petl_b200 import listmode
    rng = np.random.default_rng(2)
    n0 = a.events // 2
    b0, p0 = listmode.coincidences(n0, rng, 50.5, 125.76, 78.36, box=(30.0, 30.0, 30.0))
    b1, p1 = listmode.coincidences(a.events - n0, rng, 133.3, 62.56, 78.36, psi_deg=90.0, box=(30.0, 30.0, 30.0))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "petx.lst")
        listmode.write_lst(path, np.concatenate([b0, b1]), np.concatenate([p0, p1]))
        ours(path)  # warm-up
        t_ours, f_ours, R_ours = ours(path)
        t_ref, f_ref, R_ref = reference(path)
    res = {"workload": "demo/d02_bin_and_reconstruct.py with the PET/X preset, calc_response(1), "
                       f"{a.events} seeded coincidences in a .lst file, set_volume(120, 120, 120, 0.5), "
                       "apply_corrections, FBP",
           "ours_s": t_ours, "reference_s": t_ref,
           "ours_total_s": sum(t_ours.values()), "reference_total_s": sum(t_ref.values()),
           "rel_l2_response": [float(np.linalg.norm(x.astype(np.float64) - y) / np.linalg.norm(y))
                               for x, y in zip(R_ours, R_ref)],
           "rel_l2_fbp": float(np.linalg.norm(f_ours.astype(np.float64) - f_ref) / np.linalg.norm(f_ref))}
    res["speedup_total"] = res["reference_total_s"] / res["ours_total_s"]
    print(json.dumps(res))


if __name__ == "__main__":
    main()

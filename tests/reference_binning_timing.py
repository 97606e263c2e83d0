"""Times the reference library's own list-mode binning (CPU code, compiled
from the reference sources by ``make -C oracle ref`` into
oracle/_ref/libpetl_ref.so; test infrastructure) next to this library's bin()
on the same .lst file, both through the reference C ABI on host arrays, on
the (65,129,128,256) planogram of add_planogram(0, 256, 128, 128, T=1, 0.5,
0.25).

    python tests/reference_binning_timing.py [--events N] > ref_binning.json

The reference queues events per planogram and flushes every 1000 events
with OpenMP over all v1 slices (src/binning.cpp:662-790), on all host
cores; this library parses the file on the host in batches and bins them on
the GPU.  Times are host wall-clock per call (best of 2 after a warm-up).
"""
import argparse
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

from make_golden import Ref  # noqa: E402

ARGS = (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)
VOL = (256, 256, 128, 1.0, 1.0, 0.0, 0.0, 0.0)


def best(fn, reps=2):
    fn()
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return min(ts)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--events", type=int, default=1_000_000)
    a = ap.parse_args()
    from petl_b200 import PETLserver, listmode
    rng = np.random.default_rng(3)
    blue, pink = listmode.coincidences(a.events, rng, 128.0, 64.0, 64.0, box=(60.0, 60.0, 50.0))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "events.lst")
        listmode.write_lst(path, blue, pink)
        ref = Ref()
        ref.model([ARGS], VOL)
        gr = [np.zeros(s, np.float32) for s in ref.shapes()]
        t_ref = best(lambda: ref.L.bin(ref.pp(gr), path.encode()))
        s = PETLserver()
        s.add_planogram(*ARGS)
        s.set_volume(*[int(v) if i < 3 else float(v) for i, v in enumerate(VOL[:5])])
        go = [np.zeros(gr[0].shape, np.float32)]
        t_ours = best(lambda: s.bin(path, go))
        d = go[0].astype(np.float64) - gr[0]
        rel = float(np.linalg.norm(d) / np.linalg.norm(gr[0]))
    print(json.dumps({"events": a.events, "cores": os.cpu_count(), "reference_s": t_ref,
                      "reference_events_per_s": a.events / t_ref, "ours_s": t_ours,
                      "ours_events_per_s": a.events / t_ours, "speedup": t_ref / t_ours,
                      "rel_l2_ours_vs_reference": rel}))


if __name__ == "__main__":
    main()

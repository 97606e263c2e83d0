"""Benchmark: forward + back projections per second at 256x256x128.

Workload (one "step"): one separable-footprint forward projection of a
256x256x128 float32 volume (1 mm voxels) into the planogram (65, 129, 128,
256) of a dual-panel geometry with 1 mm bins, 256 mm separation and 128 mm
panels (add_planogram(0, 256, 128, 128, 1, 0.5, 0.25)), followed by one
backprojection of that planogram (reference backprojector semantics).  The
phantom is 30 seeded ellipsoids plus a 1 % background.  Data are synthetic;
the reference publishes no benchmark data set.

* ``value``: steps/s with volume and planogram resident in HBM, timed with
  CUDA events per step on the launching stream; the L2 is flushed (a 256 MB
  write) between steps, outside the timed events.
* ``e2e``: the same steps through the reference-compatible C ABI
  (project / backproject on pinned host arrays), host<->device copies inside.
* ``roofline``: the dominant projection call (forward: x-shift pass +
  z-tap kernel; backward: z-gather kernel + x-gather pass, one launch each
  per chunk of views, one chunk at this size): its algorithmic bytes
  (volume + planogram, read once and written once) per call against
  measured HBM bandwidth, and the call's DRAM traffic from the committed ncu
  capture; ``fp32`` adds the binding figure, 2*nnz(A) flops per call against
  the nominal FP32 rate at the measured clock.
* ``cpu_baseline``: the FP32 CPU restatement (oracle) on all host cores, on
  a bounded sample (two v1 slices), extrapolated to a full step.
* ``reference_gpu``: the reference's own GPU build (its sources compiled
  for sm_100a) through its C ABI on numpy host arrays, with this library on
  the same calls beside it (single-GPU runs).
* ``serving``: the served-reconstruction workload (200 OSEM requests of
  four volume sizes; petl_b200.studies.study_serving): p50 / p99 latency and
  recons/s of the continuous-batching server and of the one-at-a-time device
  path, at 20 arrivals/s and at saturation (single-GPU runs).

``--impl reference`` times the reference path's CPU implementation (the
oracle restatement: the reference has no CPU projector) instead.
Multi-GPU runs are independent replicas (the path needs no collective).
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+back projections/s & % HBM roofline at 256²×128; served recon p50/p99"
UNIT = "fwd+back pairs/s"
GEOM_ARGS = (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)   # psi, D, L, H, T, v_m0, v_m1
VOLUME = (256, 256, 128, 1.0)
WORKLOAD = "SF fwd+back projection, vol 256x256x128 @1mm, planogram (65,129,128,256)"


def phantom(rng, shape=(128, 256, 256), vox=(1.0, 1.0), n=30):
    """30 seeded ellipsoids (axes 5-40 mm) plus 1 % uniform background."""
    nz, ny, nx = shape
    wx, wz = vox
    x = ((np.arange(nx) - 0.5 * (nx - 1)) * wx).astype(np.float32)
    y = ((np.arange(ny) - 0.5 * (ny - 1)) * wx).astype(np.float32)
    z = ((np.arange(nz) - 0.5 * (nz - 1)) * wz).astype(np.float32)
    f = np.zeros(shape, np.float32)
    ext = np.array([nx * wx, ny * wx, nz * wz]) * 0.5
    for _ in range(n):
        r = np.minimum(rng.uniform(5.0, 40.0, 3), ext * 0.9)
        c = rng.uniform(-1, 1, 3) * (ext - r)
        val = np.float32(rng.uniform(0.1, 1.0))
        zs = slice(max(0, int((c[2] - r[2]) / wz + nz / 2) - 1), min(nz, int((c[2] + r[2]) / wz + nz / 2) + 2))
        ys = slice(max(0, int((c[1] - r[1]) / wx + ny / 2) - 1), min(ny, int((c[1] + r[1]) / wx + ny / 2) + 2))
        xs = slice(max(0, int((c[0] - r[0]) / wx + nx / 2) - 1), min(nx, int((c[0] + r[0]) / wx + nx / 2) + 2))
        Z, Y, X = np.meshgrid(z[zs], y[ys], x[xs], indexing="ij")
        inside = ((X - c[0]) / r[0]) ** 2 + ((Y - c[1]) / r[1]) ** 2 + ((Z - c[2]) / r[2]) ** 2 <= 1.0
        f[zs, ys, xs][inside] = val
    f += np.float32(0.01 * f.max())
    return f


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured", d
    except Exception:
        return 6650.0, "fallback", {}


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index=0):
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="petl_clocks_", suffix=".csv")
        os.close(fd)
        self.index = index

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                try:
                    rows.append((float(p[1]), float(p[2]), p[5:9]))
                except ValueError:
                    pass
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = sorted(r[0] for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[2]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows)}


SAMPLE_SLICES = (16, 48)   # v1 slices timed by the CPU sample (a quarter and three quarters of the range)
_SAMPLE_PHANTOM = {}


def cpu_sample(slices=SAMPLE_SLICES, nthreads=0):
    """FP32 CPU restatement (oracle) of fwd+back on the given v1 slices of the
    workload: each slice projected, then backprojected.  Returns the seconds
    taken and the fraction of one fwd+back pair that the slices are."""
    import oracle as O
    G = O.make_geom(*GEOM_ARGS[:5], GEOM_ARGS[5], GEOM_ARGS[6], VOLUME)
    if "f" not in _SAMPLE_PHANTOM:
        _SAMPLE_PHANTOM["f"] = phantom(np.random.default_rng(0))
    f = _SAMPLE_PHANTOM["f"]
    t_f = t_b = 0.0
    for a in slices:
        t0 = time.perf_counter()
        g = O.project_band(G, f, a, a + 1, nthreads=nthreads, dtype=np.float32)
        t1 = time.perf_counter()
        O.backproject_band(G, g, a, a + 1, nthreads=nthreads, dtype=np.float32)
        t2 = time.perf_counter()
        t_f += t1 - t0
        t_b += t2 - t1
    frac = len(slices) / G.N_v1
    cores = nthreads if nthreads > 0 else (os.cpu_count() or 1)
    return {"seconds": t_f + t_b, "pairs": frac, "cores": cores,
            "sample": f"v1 slices {list(slices)} of {G.N_v1} (fwd {t_f:.2f} s + back {t_b:.2f} s) = "
                      f"{len(slices)}/{G.N_v1} of a fwd+back pair, throughput extrapolated by "
                      f"x{1 / frac:.1f}; FP32 C++/OpenMP restatement of the reference kernels"}


def cpu_baseline(nthreads=0):
    r = cpu_sample(nthreads=nthreads)
    return {"value": r["pairs"] / r["seconds"], "unit": UNIT, "cores": r["cores"], "kind": "port",
            "sample": r["sample"]}


def reference_gpu_baseline(f_host, steps=2):
    """The reference library's own GPU projector and backprojector (its
    unmodified sources compiled for sm_100a into oracle/_ref/libpetl_ref.so),
    timed like a reference user calls them: its C ABI on numpy (pageable)
    host arrays, host<->device copies inside, wall clock per pair after one
    warm-up pair.  This library's libpetl.so is timed on the same calls and
    arrays for comparison.  A reported baseline; None without the build."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libpetl_ref.so")
    if not os.path.exists(path):
        return None
    fp = ctypes.POINTER(ctypes.c_float)

    def bind(libpath):
        L = ctypes.CDLL(libpath)
        L.create_new_model.restype = ctypes.c_int
        L.set_model.argtypes = [ctypes.c_int]
        L.add_planogram.argtypes = [ctypes.c_float] * 7
        L.add_planogram.restype = ctypes.c_bool
        L.set_volume.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 5
        L.set_volume.restype = ctypes.c_bool
        for n in ("project", "backproject"):
            getattr(L, n).argtypes = [ctypes.POINTER(fp), fp]
            getattr(L, n).restype = ctypes.c_bool
        return L

    psi, D, Lp, H, T, vm0, vm1 = GEOM_ARGS
    g = np.zeros((65, 129, 128, 256), np.float32)
    b = np.zeros_like(f_host)
    gp = (fp * 1)(g.ctypes.data_as(fp))
    out = {}
    for name, libpath in (("reference", path), ("petl_b200", os.path.join(ROOT, "petl_b200", "libpetl.so"))):
        L = bind(libpath)
        L.set_model(L.create_new_model())
        if not (L.add_planogram(psi, D, Lp, H, vm0, vm1, T) and L.set_volume(*VOLUME, 1.0, 0.0, 0.0, 0.0)):
            return None
        ts = []
        for k in range(steps + 1):
            t0 = time.perf_counter()
            ok = L.project(gp, f_host.ctypes.data_as(fp)) and L.backproject(gp, b.ctypes.data_as(fp))
            if not ok:
                return None
            if k:
                ts.append(time.perf_counter() - t0)
        out[name] = {"value": 1.0 / float(np.mean(ts)), "unit": UNIT, "steps": steps}
    return {"value": out["reference"]["value"], "unit": UNIT, "steps": steps,
            "host_arrays": "numpy (pageable), as the reference binding passes them",
            "build": "reference sources unmodified, nvcc -arch=sm_100a --use_fast_math (oracle/Makefile)",
            "this_library_same_calls": out["petl_b200"]["value"]}


def max_over_ranks(x, world, device=None):
    """The maximum of a per-rank number over all ranks (device timings are
    reported as the slowest rank's); the number itself for one rank."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, steps, total_ms):
    """Whole-job throughput of `world` independent replicas that each ran
    `steps` steps, timed by the slowest rank's total_ms (weak scaling: the
    per-GPU work is fixed)."""
    return world * steps / (total_ms / 1e3)


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    # one step = the sampled v1 slices of one fwd+back pair (a bounded sample
    # of the workload); throughput = pairs sampled / seconds
    t_all = []
    base = None
    for i in range(args.warmup + args.steps):
        r = cpu_sample()
        if i >= args.warmup:
            t_all.append(r["seconds"])
            base = r
    step = float(np.mean(t_all))
    val = base["pairs"] / step
    line = {"metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "path": "reference CPU restatement (oracle), all host cores",
                       "step": f"{base['pairs']:.4f} of a fwd+back pair (the sampled v1 slices)"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": base["cores"], "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-serving", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    from petl_b200 import Geometry, PETLserver, lib, ops
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    G = Geometry(*GEOM_ARGS[:5], GEOM_ARGS[5], GEOM_ARGS[6], volume=VOLUME)
    rng = np.random.default_rng(1234 + rank)
    f_host = phantom(rng)
    f = torch.from_numpy(f_host).to(dev)
    g = torch.empty(G.shape, device=dev, dtype=torch.float32)
    fb = torch.empty_like(f)
    flush = torch.empty(64 * 1024 * 1024, device=dev, dtype=torch.float32)  # 256 MB > L2
    nnz = ops.nnz(G)

    def step():
        ops.project(G, f, g)
        ops.backproject(G, g, fb)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    launches0 = lib().petl_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.zero_()
        e0, e1, e2 = ev[k]
        e0.record()
        ops.project(G, f, g)
        e1.record()
        ops.backproject(G, g, fb)
        e2.record()
    torch.cuda.synchronize()
    launches = lib().petl_launch_count() - launches0
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    t_fwd = [a.elapsed_time(b) for a, b, _ in ev]
    t_bwd = [b.elapsed_time(c) for _, b, c in ev]
    total_ms = max_over_ranks(float(np.sum(t_fwd) + np.sum(t_bwd)), world, dev)
    ms_per_step = total_ms / args.steps
    value = replica_value(world, args.steps, total_ms)

    # roofline of the dominant kernel
    hbm, peak_kind, peaks = read_peaks()
    avg_f, avg_b = float(np.mean(t_fwd)), float(np.mean(t_bwd))
    dom = "forward" if avg_f >= avg_b else "backward"
    t_dom = max(avg_f, avg_b) / 1e3
    alg_bytes = 4.0 * (G.n_voxels + G.n_rays)
    achieved = alg_bytes / t_dom / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(dom)
        except Exception:
            traffic = None
    sm_clock = (clk or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * sm_clock * 1e6 / 1e12
    fp32_ach = 2.0 * nnz / t_dom / 1e12
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "kernel": dom, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_launch": alg_bytes,
                "fp32": {"achieved": fp32_ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": fp32_ach / fp32_peak,
                         "nnz": nnz, "peak_kind": "nominal 148 SM x 128 FMA/clk x 2 at the median SM clock",
                         "note": "binding roofline: the path is FP32-issue bound"},
                "ms_forward": avg_f, "ms_backward": avg_b}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "geometry": "add_planogram(0, 256, 128, 128, T=1, 0.5, 0.25)",
                       "volume": "256x256x128 @ 1 mm", "planogram": list(G.shape),
                       "backprojector": "reference semantics, exact weights",
                       "l2": "256 MB flush between steps, outside the per-step CUDA events",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline, "gpu_launches": int(launches), "clocks": clk}

    if not args.no_e2e:
        s = PETLserver()
        s.add_planogram(*GEOM_ARGS)
        s.set_volume(*VOLUME)
        fh = torch.from_numpy(f_host).pin_memory()
        gh = torch.empty(G.shape, dtype=torch.float32).pin_memory()
        bh = torch.empty(G.vol_shape, dtype=torch.float32).pin_memory()
        fnp, gnp, bnp = fh.numpy(), gh.numpy(), bh.numpy()
        s.project([gnp], fnp)
        s.backproject([gnp], bnp)
        ts = []
        for _ in range(max(1, args.e2e_steps)):
            t0 = time.perf_counter()
            s.project([gnp], fnp)
            s.backproject([gnp], bnp)
            ts.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(float(np.mean(ts)), world, dev)
        nb_f, nb_g = 4 * G.n_voxels, 4 * G.n_rays
        line["e2e"] = {"value": world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": nb_f + nb_g,
                       "d2h_bytes_per_step": nb_g + nb_f, "steps": len(ts),
                       "path": "PETLserver.project + backproject (reference C ABI, pinned host arrays)"}
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline()
        if world == 1:
            line["reference_gpu"] = reference_gpu_baseline(f_host)
    if world == 1 and not args.no_serving:
        # the metric's second half: served reconstructions, p50 / p99
        del g, fb, flush
        torch.cuda.empty_cache()
        from petl_b200.studies import study_serving
        line["serving"] = study_serving()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Reconstruction workloads beyond the fwd+back headline, one JSON line each.

    python -m petl_b200.studies pipeline    # 256x256x128: PFDR, FBP, 8-subset OSEM x 4
    python -m petl_b200.studies penalized   # 4 x 128x128x64, NLL + RD + TV, 50 steps, FD check
    python -m petl_b200.studies storage     # 256x256x128 OSEM 10 x 8 subsets, FP32 vs BF16 storage
    python -m petl_b200.studies serving     # 200 Poisson-arrival OSEM requests, p50/p99
    python -m petl_b200.studies binning     # list-mode binning, device and C-ABI file rates
    python -m petl_b200.studies corrections # solid angle and apply_corrections, device and C ABI
    python -m petl_b200.studies response    # PET/X stopping power (120 blocks) and calc_response
    python -m petl_b200.studies kernels     # PFDR, ramp, FBP, RD/TV stencils: device time, HBM fraction

All inputs are synthetic and seeded: ellipsoid phantoms (replace semantics,
later ellipsoids overwrite earlier ones), forward projected with the
library's projector and Poisson sampled on the GPU.  Times are CUDA-event
times on the device except the serving latencies, which are host
wall-clock from submission to the result on the host.  Accuracy against
the FP64 oracle is established by the test suite (tests/), not here.
"""
import argparse
import json
import math
import time

import numpy as np
import torch

from . import ops, recon
from .geometry import Geometry


def phantom(shape, pitch, rng, n, axes=(5.0, 40.0), vmin=0.1, vmax=1.0, background=0.0, device="cuda"):
    """Seeded ellipsoids in a [z, y, x] volume of voxel pitch (wx, wz) mm."""
    nz, ny, nx = shape
    wx, wz = pitch
    x = (torch.arange(nx, device=device) - 0.5 * (nx - 1)) * wx
    y = (torch.arange(ny, device=device) - 0.5 * (ny - 1)) * wx
    z = (torch.arange(nz, device=device) - 0.5 * (nz - 1)) * wz
    f = torch.full(shape, float(background), device=device)
    ext = np.array([nx * wx, ny * wx, nz * wz]) * 0.5
    for _ in range(n):
        r = np.minimum(rng.uniform(axes[0], axes[1], 3), ext * 0.95)
        c = rng.uniform(-1, 1, 3) * np.maximum(ext - r, 0)
        val = float(rng.uniform(vmin, vmax))
        inside = (((x - c[0]) / r[0]) ** 2)[None, None, :] + (((y - c[1]) / r[1]) ** 2)[None, :, None] + \
            (((z - c[2]) / r[2]) ** 2)[:, None, None] <= 1.0
        f[inside] = val
    return f


def poisson_data(G, f, counts, seed, return_scale=False):
    y = ops.project(G, f)
    scale = counts / float(y.sum())
    y.mul_(scale)
    y = torch.poisson(y, generator=torch.Generator(device=y.device).manual_seed(seed))
    return (y, scale) if return_scale else y


def _rel(img, ref, scale=1.0):
    """relative L2 of img / scale against ref (images live on the counts scale)"""
    return float((img / scale - ref).norm() / ref.norm())


class Timer:
    def __init__(self):
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)

    def __enter__(self):
        torch.cuda.synchronize()
        self.a.record()
        return self

    def __exit__(self, *exc):
        self.b.record()
        torch.cuda.synchronize()
        self.ms = self.a.elapsed_time(self.b)


CFG1 = dict(args=(0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25), volume=(256, 256, 128, 1.0))
CFG0 = dict(args=(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25), volume=(128, 128, 64, 2.0))


def study_pipeline(seed=0):
    G = Geometry(*CFG1["args"], volume=CFG1["volume"])
    rng = np.random.default_rng(seed)
    f = phantom(G.vol_shape, (1.0, 1.0), rng, 30)
    f += 0.01 * float(f.max())
    y, scale = poisson_data(G, f, 5e7, seed, return_scale=True)
    out = {"study": "pipeline", "workload": "vol 256x256x128 @1mm, planogram (65,129,128,256), 5e7 counts",
           "geometry": "add_planogram(0, 256, 128, 128, T=1, 0.5, 0.25)"}
    for _ in range(2):  # warm-up of every stage
        ops.pfdr(G, y)
        ops.fbp(G, y)
    with Timer() as t:
        reb = ops.pfdr(G, y)
    out["pfdr_ms"] = t.ms
    with Timer() as t:
        img = ops.fbp(G, y)
    out["fbp_ms"] = t.ms
    sens = [recon.sensitivity(G, [y], subset=(s, 8)) for s in range(8)]
    with Timer() as t:
        fo, _ = recon.osem(G, y, 4, 8, sens=sens)
    out["osem_4x8_ms"] = t.ms
    out["osem_ms_per_iteration"] = t.ms / 4
    # sanity only: images live on the counts scale and only the field of
    # view (voxels with sensitivity) can be reconstructed
    fov = ops.backproject(G, torch.ones_like(y)) > 0
    out["osem_image_rel_l2_vs_phantom_fov"] = _rel(fo[fov], f[fov], scale)
    a = float((img[fov] * f[fov]).sum() / (img[fov] * img[fov]).sum())  # least-squares scale of the FBP image
    out["fbp_image_rel_l2_vs_phantom_fov_fitted_scale"] = _rel(img[fov] * a, f[fov])
    out["fbp_fitted_scale_over_data_scale"] = 1.0 / (a * scale)
    out["rebinned_shape"] = list(reb.shape)
    return out


def _peak_hbm_gbs():
    import os
    try:
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                               "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def study_kernels(seed=0, reps=10, proj_size=256):
    """Device time of the rebinning and regularizer kernels (CUDA events,
    median of `reps`, the L2 flushed before each) with their algorithmic
    bytes and the fraction of the measured HBM bandwidth: PFDR (reads the
    planogram once, writes the rebinned one), the ramp filter (reads and
    writes the rebinned planogram), FBP (PFDR + ramp + the N_v1 = 1
    backprojection), and the RD / TV gradients (read the volume, write the
    gradient) at 128x128x64 and 256x256x128; then the projectors by
    orientation on a proj_size^2 x proj_size/2 volume at 1 mm (256 by
    default; 128 gives a small case for kernel captures)."""
    peak, kind = _peak_hbm_gbs()
    flush = torch.empty(64 * 1024 * 1024, device="cuda")

    def timed(fn):
        fn()
        ts = []
        for _ in range(reps):
            flush.zero_()
            with Timer() as t:
                fn()
            ts.append(t.ms)
        return float(np.median(ts))

    out = {"study": "kernels", "hbm_peak_gbs": peak, "hbm_peak_kind": kind}
    for name, cfg in (("256x256x128", CFG1), ("128x128x64", CFG0)):
        G = Geometry(*cfg["args"], volume=cfg["volume"])
        rng = np.random.default_rng(seed)
        f = phantom(G.vol_shape, (cfg["volume"][3],) * 2, rng, 12) + 0.01
        y = ops.project(G, f)
        Gr = G.rebinned()
        reb = ops.pfdr(G, y)
        nb_g, nb_r, nb_f = 4 * y.numel(), 4 * reb.numel(), 4 * f.numel()
        r = {}
        t = timed(lambda: ops.pfdr(G, y, reb))
        r["pfdr_ms"], r["pfdr_hbm_frac"] = t, (nb_g + nb_r) / (t * 1e6) / peak
        work = reb.clone()
        t = timed(lambda: ops.ramp_(Gr, work))
        r["ramp_ms"], r["ramp_hbm_frac"] = t, 2 * nb_r / (t * 1e6) / peak
        t = timed(lambda: ops.fbp(G, y))
        r["fbp_ms"] = t
        Df = torch.empty_like(f)
        t = timed(lambda: ops.rd_gradient(f, 2.0, 0.01, out=Df))
        r["rd_gradient_ms"], r["rd_gradient_hbm_frac"] = t, 2 * nb_f / (t * 1e6) / peak
        t = timed(lambda: ops.tv_gradient(f, 1e-4, 0.01, 1.0, out=Df))
        r["tv_gradient_ms"], r["tv_gradient_hbm_frac"] = t, 2 * nb_f / (t * 1e6) / peak
        t = timed(lambda: ops.tv_cost(f, 1e-4, 0.01, 1.0))
        r["tv_cost_ms"], r["tv_cost_hbm_frac"] = t, nb_f / (t * 1e6) / peak
        t = timed(lambda: ops.rd_cost(f, 2.0, 0.01))
        r["rd_cost_ms"], r["rd_cost_hbm_frac"] = t, nb_f / (t * 1e6) / peak
        r["planogram"], r["rebinned"], r["volume"] = list(G.shape), list(reb.shape), list(f.shape)
        out[name] = r
    # projectors by planogram orientation at 256x256x128 (1 mm): psi = 0 and
    # 90 run the shear-warp kernels (90 on the volume with x and y
    # exchanged), psi = 30 the split kernels for any psi; backward in the
    # reference's semantics and as the exact adjoint; FP32 fraction of
    # 2 nnz(A) flops per call at the nominal rate (148 SM x 128 FMA/clk at
    # 1965 MHz)
    fp32_peak = 148 * 128 * 2 * 1965e6 / 1e12
    from . import lib
    n = int(proj_size)
    for psi in (0.0, 90.0, 30.0):
        G = Geometry(psi, float(n), n / 2.0, n / 2.0, 1.0, 0.5, 0.25, volume=(n, n, n // 2, 1.0))
        f = phantom(G.vol_shape, (1.0, 1.0), np.random.default_rng(seed), 12) + 0.01
        g = torch.empty(G.shape, device="cuda")
        b = torch.empty_like(f)
        nnz = ops.nnz(G)
        ops.project(G, f, g)
        path = lib().petl_last_projector_path()
        ops.backproject(G, g, b)
        path_b = lib().petl_last_projector_path()
        ops.backproject(G, g, b, mode="adjoint")
        path_a = lib().petl_last_projector_path()
        ts_f, ts_b, ts_a = [], [], []
        for _ in range(reps):
            flush.zero_()
            with Timer() as t:
                ops.project(G, f, g)
            ts_f.append(t.ms)
            flush.zero_()
            with Timer() as t:
                ops.backproject(G, g, b)
            ts_b.append(t.ms)
            flush.zero_()
            with Timer() as t:
                ops.backproject(G, g, b, mode="adjoint")
            ts_a.append(t.ms)
        tf, tb, ta = float(np.median(ts_f)), float(np.median(ts_b)), float(np.median(ts_a))
        out[f"project_psi{int(psi)}"] = {"planogram": list(G.shape), "path": path, "path_backward": path_b,
                                         "path_adjoint": path_a, "forward_ms": tf, "backward_ms": tb,
                                         "adjoint_ms": ta, "nnz": nnz,
                                         "forward_fp32_frac": 2 * nnz / (tf * 1e-3) / 1e12 / fp32_peak,
                                         "backward_fp32_frac": 2 * nnz / (tb * 1e-3) / 1e12 / fp32_peak,
                                         "adjoint_fp32_frac": 2 * nnz / (ta * 1e-3) / 1e12 / fp32_peak}
    return out


def study_penalized(seed=0, steps=50, fd_voxels=64):
    from . import penalized
    G = Geometry(*CFG0["args"], volume=CFG0["volume"])
    rng = np.random.default_rng(seed)
    vols, data = [], []
    for b in range(4):
        f = phantom(G.vol_shape, (2.0, 2.0), np.random.default_rng(seed + b), 12)
        vols.append(f)
        data.append(poisson_data(G, f, 1e6, seed + b))
    yb = torch.stack(data)
    rd = (2.0, 0.01)                 # gamma, beta (26 neighbours)
    tv = (1e-4, 0.01, 1.0, 26)       # delta = 1e-4 (eps), beta_tv = 0.01 (chosen), p = 1
    penalized.reconstruct(G, yb, iters=2, rd=rd, tv=tv)  # warm-up
    with Timer() as t:
        fr, hist = penalized.reconstruct(G, yb, iters=steps, rd=rd, tv=tv)
    f0 = fr[0].contiguous()
    cand = torch.nonzero(f0.reshape(-1) > 0.05 * float(f0.max())).reshape(-1).cpu().numpy()
    vox = rng.choice(cand, fd_voxels, replace=False)
    got, fd = penalized.fd_check(f0, G, yb[0], vox, h=1e-3, rd=rd, tv=tv)
    got = got.cpu().numpy()
    fd = fd.numpy()
    rel = np.abs(got - fd) / np.maximum(np.abs(fd), 1e-12)
    h = hist.numpy()
    return {"study": "penalized", "workload": "4 x vol 128x128x64 @2mm, planogram (33,65,64,128), 1e6 counts each",
            "objective": "Poisson NLL + RD(gamma=2, beta=0.01, 26-nbr) + TV(delta=1e-4, p=1, beta=0.01, 26-nbr)",
            "steps": steps, "total_ms": t.ms, "ms_per_step_batch4": t.ms / steps,
            "objective_first": h[0].tolist(), "objective_last": h[-1].tolist(),
            "monotone_fraction": float((np.diff(h, axis=0) <= 0).mean()),
            "fd_voxels": fd_voxels, "fd_h": 1e-3, "fd_rel_err_median": float(np.median(rel)),
            "fd_rel_err_max": float(rel.max())}


def study_storage(seed=0, iters=10, subsets=8):
    G = Geometry(*CFG1["args"], volume=CFG1["volume"])
    rng = np.random.default_rng(seed)
    f = phantom(G.vol_shape, (1.0, 1.0), rng, 30)
    f += 0.01 * float(f.max())
    y = poisson_data(G, f, 5e7, seed)
    y16 = y.to(torch.bfloat16)
    sens = [recon.sensitivity(G, [y], subset=(s, subsets)) for s in range(subsets)]
    recon.osem(G, y, 1, subsets, sens=sens)
    with Timer() as t32:
        f32, _ = recon.osem(G, y, iters, subsets, sens=sens)
    recon.osem_bf16(G, y16, 1, subsets, sens=sens)
    with Timer() as t16:
        f16 = recon.osem_bf16(G, y16, iters, subsets, sens=sens)
    with Timer() as t16b:
        f16b = recon.osem_bf16(G, y16, iters, subsets, sens=sens, image="bf16")
    ng, nv = y.numel(), f.numel()
    # per subset step: read meas + write ratio (forward), read ratio (backward),
    # volume traffic: read f (forward), write d, read f, d, sens, write f (update)
    sub = ng / subsets
    def traffic(eb):
        return iters * subsets * (3 * sub * eb + nv * 4 * 4 + nv * eb * 2)
    p32 = ops.project(G, f32)
    p16 = ops.project(G, f16.float())
    return {"study": "storage", "workload": "vol 256x256x128 @1mm, planogram (65,129,128,256), 5e7 counts, "
            f"OSEM {iters} it x {subsets} subsets",
            "fp32_ms": t32.ms, "bf16_ms": t16.ms, "bf16_image_ms": t16b.ms,
            "image_rel_l2_bf16img_vs_fp32": float((f16b.float() - f32).norm() / f32.norm()),
            "fp32_bytes": traffic(4), "bf16_bytes": traffic(2),
            "fp32_GBps": traffic(4) / (t32.ms * 1e6), "bf16_GBps": traffic(2) / (t16.ms * 1e6),
            "image_rel_l2_bf16_vs_fp32": float((f16.float() - f32).norm() / f32.norm()),
            "image_max_abs_bf16_vs_fp32": float((f16.float() - f32).abs().max()),
            "proj_rel_l2_bf16_vs_fp32": float((p16 - p32).norm() / p32.norm())}


def _serving_requests(n, rate, seed, device, sizes=(64, 128, 192, 256)):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    reqs = []
    for i in range(n):
        N = int(rng.choice(list(sizes)))
        T = float(rng.choice([1.0, 1.5, 2.0]))
        D = float(rng.choice([200.0, 250.0, 300.0]))
        counts = float(math.exp(rng.uniform(math.log(1e5), math.log(5e7))))
        S = int(rng.choice([4, 8]))
        it = int(rng.integers(2, 7))
        reqs.append(dict(t=float(t[i]), N=N, T=T, D=D, counts=counts, S=S, it=it))
    return reqs


def study_serving(n=200, rate=20.0, seed=0, max_active=16, budget_gb=150.0, modes=("arrivals", "saturation"),
                  sizes=(64, 128, 192, 256)):
    """The serving workload: n OSEM requests with seeded Poisson arrivals at
    `rate`/s (mode "arrivals") or all submitted at t = 0 ("saturation"),
    served (a) by the continuous-batching server (as configured by default,
    and with batched launches of like-geometry requests) and (b) one request at a
    time by the plain device path (host data to the device, recon.osem, the
    image back to the host, in arrival order).  Latency is host wall clock
    from a request's arrival to its image on the host; recons/s is n over
    the time from the first arrival to the last result.  `sizes` restricts
    the volume sizes N drawn (the workload draws all four)."""
    from .serving import ReconServer
    reqs = _serving_requests(n, rate, seed, "cuda", sizes)
    # geometry classes: N in {64,128,192,256}, T in {1,1.5,2} mm, D in
    # {200,250,300} mm (the workload draws T and D from [1,2] and [200,300];
    # a request's work depends on them only through its planogram shape and
    # slopes, which the grid spans, and one pinned planogram per distinct
    # geometry would need up to 1.1 GB of page-locked host memory each).
    # Requests of a class share one Poisson realisation at the class's first
    # drawn counts: the work does not depend on the counts.
    classes = {}
    for r in reqs:
        key = (r["N"], r["T"], r["D"])
        if key not in classes:
            N, T, D = key
            G = Geometry(0.0, D, N * T / 2, N * T / 2, T, 0.5, 0.25, volume=(N, N, N // 2, T))
            f = phantom(G.vol_shape, (T, T), np.random.default_rng(hash(key) % 2**31), 8)
            y = poisson_data(G, f, r["counts"], 1)
            host = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
            host.copy_(y.cpu())
            classes[key] = (G, host)
            del y, f
    torch.cuda.synchronize()

    def arrivals(mode):
        return [r["t"] if mode == "arrivals" else 0.0 for r in reqs]

    def summary(lat, wall, extra=None):
        lat = np.array(lat)
        out = {"recons_per_s": n / wall, "wall_s": wall, "p50_s": float(np.percentile(lat, 50)),
               "p99_s": float(np.percentile(lat, 99)), "max_s": float(lat.max())}
        out.update(extra or {})
        return out

    def serve_server(mode, batch=1):
        at = arrivals(mode)
        with ReconServer(hbm_budget_gb=budget_gb, max_active=max_active, depth=2, batch=batch) as srv:
            for key, (G, host) in classes.items():  # warm-up: one request per class
                srv.wait(srv.submit(G, host, 4, 1))
            t0 = time.perf_counter()
            ids = []
            for r, a in zip(reqs, at):
                now = time.perf_counter() - t0
                if a > now:
                    time.sleep(a - now)
                G, host = classes[(r["N"], r["T"], r["D"])]
                ids.append(srv.submit(G, host, r["S"], r["it"]))
            lat = []
            for i in ids:  # the server's own clock: submission (= arrival) to the result on the host
                lat.append(srv.wait(i)[1])
            wall = time.perf_counter() - t0
            st = srv.stats()
            bs = srv.batch_stats()
        return summary(lat, wall, {"hbm_peak_gb": st["hbm_peak_bytes"] / 1e9, "failed": st["failed"],
                                   "max_active": max_active, "batch_max": batch, **bs})

    def serve_sequential(mode):
        at = arrivals(mode)
        for key, (G, host) in classes.items():  # warm-up
            recon.osem(G, host.to("cuda", non_blocking=True), 1, 4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat = []
        for r, a in zip(reqs, at):
            now = time.perf_counter() - t0
            if a > now:
                time.sleep(a - now)
            G, host = classes[(r["N"], r["T"], r["D"])]
            f, _ = recon.osem(G, host.to("cuda", non_blocking=True), r["it"], r["S"])
            f.cpu()
            lat.append(time.perf_counter() - t0 - a)
        wall = time.perf_counter() - t0
        return summary(lat, wall)

    # GPU-seconds of the mix: every request alone on the device, back to back
    gpu_s = 0.0
    for r in reqs:
        G, host = classes[(r["N"], r["T"], r["D"])]
        g = host.to("cuda")
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        recon.osem(G, g, r["it"], r["S"])
        b.record()
        torch.cuda.synchronize()
        gpu_s += a.elapsed_time(b) / 1e3
    out = {"study": "serving", "workload": f"{n} OSEM requests, Poisson arrivals {rate}/s (seed {seed}), "
           f"N in {{{','.join(str(v) for v in sizes)}}} (vol NxNxN/2 at pitch T in {{1,1.5,2}} mm), L=H=N*T/2, "
           "D in {200,250,300} mm, "
           "4 or 8 subsets, 2-6 iterations", "geometry_classes": len(classes), "budget_gb": budget_gb,
           "gpu_seconds_per_request": gpu_s / n,
           "bound_recons_per_s": n / gpu_s,
           "bound_note": "device time of the requests run alone back to back: no schedule of them on one GPU "
                         "serves more than n / that many per second unless requests share launches"}
    # an unmeasured pass first: the library's memory pool grows to the
    # workload's peak in whichever pass runs first (about 10 % of that
    # pass's throughput when measured)
    serve_server("saturation")
    for mode in modes:
        srv = serve_server(mode)
        bat = serve_server(mode, batch=8)
        seq = serve_sequential(mode)
        out[mode] = {"server": srv, "server_batched": bat, "one_at_a_time": seq,
                     "throughput_ratio": srv["recons_per_s"] / seq["recons_per_s"],
                     "p99_ratio": srv["p99_s"] / seq["p99_s"],
                     "batched_throughput_ratio": bat["recons_per_s"] / srv["recons_per_s"],
                     "batched_p99_ratio": bat["p99_s"] / srv["p99_s"]}
    return out


def study_binning(seed=0, n_events=16_000_000, n_file=8_000_000, tmpdir="/tmp"):
    """List-mode binning at the 256x256x128 geometry (planogram (65,129,128,
    256)): device-resident events binned by the kernel (events/s), and a
    .lst file binned through the reference C ABI (parse + copies + kernel +
    the planogram back to the host)."""
    import os
    from . import listmode
    from .server import PETLserver
    args = (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)
    G = Geometry(*args, volume=(256, 256, 128, 1.0))
    rng = np.random.default_rng(seed)
    parts_b, parts_p = [], []
    for k in range(0, n_events, 2_000_000):
        b, p = listmode.coincidences(min(2_000_000, n_events - k), rng, 128.0, 64.0, 64.0, box=(60.0, 60.0, 50.0))
        parts_b.append(b)
        parts_p.append(p)
    blue_h, pink_h = np.concatenate(parts_b), np.concatenate(parts_p)
    blue = torch.from_numpy(blue_h).cuda()
    pink = torch.from_numpy(pink_h).cuda()
    g = torch.zeros(G.shape, device="cuda")
    res = {"study": "binning", "workload": f"{n_events} coincidences on the panels of "
           "add_planogram(0, 256, 128, 128, T=1, 0.5, 0.25), planogram (65,129,128,256), bilinear deposits"}
    for linear in (True, False):
        ops.bin_events(G, blue, pink, g=g, linear=linear)
        ts = []
        for _ in range(3):
            g.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ops.bin_events(G, blue, pink, g=g, linear=linear)
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        key = "linear" if linear else "nearest"
        res[f"device_{key}_ms"] = float(np.median(ts))
        res[f"device_{key}_events_per_s"] = n_events / (np.median(ts) * 1e-3)
    res["binned_fraction"] = float(g.sum()) / n_events  # nearest: events landing in a bin
    path = os.path.join(tmpdir, f"petl_binning_{os.getpid()}.lst")
    listmode.write_lst(path, blue_h[:n_file], pink_h[:n_file])
    s = PETLserver()
    s.add_planogram(*args)
    s.set_volume(256, 256, 128, 1.0)
    gh = [np.empty(G.shape, np.float32)]
    s.bin(path, gh)
    t0 = time.perf_counter()
    s.bin(path, gh)
    t = time.perf_counter() - t0
    os.remove(path)
    res.update({"file_events": n_file, "file_bytes": n_file * 48, "cabi_file_s": t,
                "cabi_file_events_per_s": n_file / t})
    return res


def study_corrections(seed=0, reps=5):
    """Planogram corrections on the 256x256x128 geometry's planogram
    (65,129,128,256), device-resident: the solid-angle scaling (8 bytes of
    HBM traffic per bin) and apply_corrections (12 bytes per bin) with two
    responses: detector gaps (responses in [0.9, 1.1], 2 % of the bins at a
    tenth of that: 2 % of the bins in-filled) and a stress case (responses
    in [0.5, 1.5]: a quarter of the bins in-filled).  Then both through the
    reference C ABI on pinned host arrays."""
    from .server import PETLserver
    args = (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)
    G = Geometry(*args, volume=(256, 256, 128, 1.0))
    rng = np.random.default_rng(seed)
    sh = G.shape
    nbins = int(np.prod(sh))
    g_h = rng.poisson(1.0, size=sh).astype(np.float32)
    g = torch.from_numpy(g_h).cuda()
    work = torch.empty_like(g)
    flush = torch.empty(64 << 20, device="cuda", dtype=torch.float32)  # 256 MB > L2
    res = {"study": "corrections", "workload": "planogram (65,129,128,256) of add_planogram(0, 256, 128, 128, "
           "T=1, 0.5, 0.25), Poisson(1) data; L2 flushed before each timed call", "bins": nbins}

    def timed(fn):
        fn()
        ts = []
        for _ in range(reps):
            work.copy_(g)
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return float(np.median(ts))

    t = timed(lambda: ops.solid_angle_(G, work))
    res.update({"solid_angle_ms": t, "solid_angle_gbs": 8.0 * nbins / (t * 1e6)})
    responses = {}
    r = rng.uniform(0.9, 1.1, size=sh).astype(np.float32)
    r[rng.random(sh) < 0.02] *= np.float32(0.1)
    responses["gaps"] = r
    responses["stress"] = rng.uniform(0.5, 1.5, size=sh).astype(np.float32)
    for key, r_h in responses.items():
        r = torch.from_numpy(r_h).cuda()
        t = timed(lambda: ops.apply_corrections_(G, work, r, 0.75))
        res.update({f"corrections_{key}_ms": t, f"corrections_{key}_gbs": 12.0 * nbins / (t * 1e6)})
    del r
    s = PETLserver()
    s.add_planogram(*args)
    gp = [torch.from_numpy(g_h).pin_memory().numpy()]
    rp = [torch.from_numpy(responses["gaps"]).pin_memory().numpy()]
    s.set_response(rp)
    ts = []
    for _ in range(3):
        gp[0][:] = g_h
        t0 = time.perf_counter()
        s.apply_corrections(gp)
        ts.append(time.perf_counter() - t0)
    res["cabi_corrections_gaps_ms"] = 1e3 * min(ts)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        s.apply_solid_angle_correction(gp)
        ts.append(time.perf_counter() - t0)
    res["cabi_solid_angle_ms"] = 1e3 * min(ts)
    return res


def study_response(seed=0, reps=3):
    """The PET/X detector response: the stopping power of its 120 crystal
    blocks over both planograms (463 M coincidence lines), device-resident
    (CUDA events), then PETLserver.calc_response (stopping power through the
    C ABI, the 0.6571-bin Gaussian, the solid-angle model) on host arrays."""
    from .server import PETXserver, petx_modules
    s = PETXserver()
    geoms = s.geometries_from_model()
    solids = [ops.make_solid(1, c, r, 0.0815) for c, r in petx_modules()]
    out = [torch.empty(G.shape, device="cuda") for G in geoms]
    lines = sum(int(np.prod(G.shape)) for G in geoms)
    ops.ray_trace(geoms, solids, g=out, stopping_power=True)
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ops.ray_trace(geoms, solids, g=out, stopping_power=True)
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    res = {"study": "response", "workload": "PET/X preset, planograms (63,63,96,220) and (97,167,96,244), "
           "120 crystal blocks", "lines": lines, "stopping_power_device_ms": float(np.median(ts)),
           "lines_per_s": lines / (np.median(ts) * 1e-3)}
    del out
    t0 = time.perf_counter()
    R = s.calc_response(oversampling=1)
    res["calc_response_s"] = time.perf_counter() - t0
    res["response_mean"] = [float(r.mean()) for r in R]
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("study", choices=["pipeline", "penalized", "storage", "serving", "binning", "corrections",
                                      "response", "kernels"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--sizes", default="64,128,192,256", help="serving: volume sizes N drawn")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: arrivals per second")
    ap.add_argument("--reps", type=int, default=0, help="kernels: timed calls per figure (0: the study's default)")
    ap.add_argument("--proj-size", type=int, default=256, help="kernels: volume N x N x N/2 of the projector timings")
    a = ap.parse_args(argv)
    fn = {"pipeline": study_pipeline, "penalized": study_penalized, "storage": study_storage,
          "binning": study_binning, "corrections": study_corrections, "response": study_response,
          "kernels": study_kernels}
    if a.study == "serving":
        res = study_serving(n=a.requests, seed=a.seed, rate=a.rate,
                            sizes=tuple(int(v) for v in a.sizes.split(",")))
    elif a.study == "kernels":
        res = study_kernels(seed=a.seed, reps=a.reps if a.reps > 0 else 10, proj_size=a.proj_size)
    else:
        res = fn[a.study](seed=a.seed)
    print(json.dumps(res))


if __name__ == "__main__":
    main()

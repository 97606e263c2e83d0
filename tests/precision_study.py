"""Storage-precision study against the FP64 oracle (test infrastructure).

    python tests/precision_study.py > precision.json

1. Projections at 256x256x128 (planogram (65,129,128,256)): the projection of
   a seeded phantom with FP32 storage and with BF16 storage (volume rounded
   to bfloat16, planogram written in bfloat16, FP32 accumulation in both)
   against the FP64 oracle projection of the same (FP32) phantom.
2. Images at 128x128x64 (planogram (33,65,64,128)): OSEM, 10 iterations x 8
   subsets, with FP32 storage, with BF16 planograms and projector input (FP32
   image), and with the image stored in BF16 too, on the GPU against the
   same OSEM run by the FP64 oracle, all from one Poisson data set.  The full
   256x256x128 FP64 OSEM would take tens of CPU minutes; the smaller geometry
   has the same slopes and pitch ratio.

Prints one JSON line with relative L2 and max-abs errors per variant.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import oracle as O  # noqa: E402
from helpers import ellipsoids  # noqa: E402


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.abs(a - b).max())


def main():
    import torch
    from petl_b200 import Geometry, ops, recon
    dev = torch.device("cuda:0")
    out = {"study": "precision", "reference": "FP64 oracle (oracle/oracle.cpp), all host threads"}

    # 1. projections at full size
    args, vol = (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25), (256, 256, 128, 1.0)
    G, Go = Geometry(*args, volume=vol), O.make_geom(*args, vol)
    rng = np.random.default_rng(0)
    f = ellipsoids(G.vol_shape, (1.0, 1.0), rng, 30, axes=(5.0, 40.0))
    f += 0.01 * f.max()
    ft = torch.from_numpy(f).to(dev)
    p32 = ops.project(G, ft).cpu().numpy()
    p16 = ops.project_bf16(G, ft.to(torch.bfloat16)).float().cpu().numpy()
    t0 = time.time()
    p64 = O.project(Go, f)[0]
    out["oracle_projection_s"] = time.time() - t0
    out["proj_fp32_rel_l2"], out["proj_fp32_max_abs"] = rel(p32, p64)
    out["proj_bf16_rel_l2"], out["proj_bf16_max_abs"] = rel(p16, p64)
    out["proj_bytes_fp32"] = int(4 * (p32.size + f.size))
    out["proj_bytes_bf16"] = int(2 * (p32.size + f.size))
    del p32, p16, p64

    # 2. OSEM images at 128x128x64
    args, vol = (0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0)
    G, Go = Geometry(*args, volume=vol), O.make_geom(*args, vol)
    f = ellipsoids(G.vol_shape, (2.0, 2.0), np.random.default_rng(1), 12, axes=(5.0, 40.0))
    y = O.project(Go, f)[0]
    y *= 5e6 / y.sum()
    y = np.random.default_rng(2).poisson(y).astype(np.float32)
    t0 = time.time()
    f64 = O.osem(Go, y, 10, 8)
    out["oracle_osem_s"] = time.time() - t0
    yt = torch.from_numpy(y).to(dev)
    f32, _ = recon.osem(G, yt, 10, 8)
    f16 = recon.osem_bf16(G, yt.to(torch.bfloat16), 10, 8)                  # FP32 image, BF16 planograms/projector input
    f16b = recon.osem_bf16(G, yt.to(torch.bfloat16), 10, 8, image="bf16")   # image stored in BF16 too
    out["image_fp32_rel_l2"], out["image_fp32_max_abs"] = rel(f32.cpu().numpy(), f64)
    out["image_bf16_rel_l2"], out["image_bf16_max_abs"] = rel(f16.float().cpu().numpy(), f64)
    out["image_bf16img_rel_l2"], out["image_bf16img_max_abs"] = rel(f16b.float().cpu().numpy(), f64)
    out["image_scale_max"] = float(np.abs(f64).max())
    print(json.dumps(out))


if __name__ == "__main__":
    main()

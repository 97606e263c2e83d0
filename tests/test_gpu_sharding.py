"""Sharded OSEM on the GPU with one NCCL rank (the pool gives one GPU): the
driver, its device backend and the all-reduce must give recon.osem's image
bit for bit.  The rank runs in a child process so that its process group
does not outlive the test."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _child(port):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from conftest import load_golden
    from petl_b200 import Geometry, recon
    from petl_b200.sharding import sharded_osem
    z = load_golden("mlem_g0.npz")
    vol = tuple(z["volume"])
    G = Geometry(*z["planograms"][0], volume=vol)
    G90 = Geometry(90.0, *z["planograms"][0][1:], volume=vol)
    g = torch.from_numpy(z["g"].astype(np.float32)).cuda()
    g90 = g.clone()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    try:
        for geoms, data in (([G], [g]), ([G, G90], [g, g90])):
            want, _ = recon.osem(geoms, data, 2, 4)
            got = sharded_osem(geoms, data, 2, 4)
            torch.cuda.synchronize()
            assert torch.equal(got, want), float((got - want).abs().max())
    finally:
        dist.destroy_process_group()
    print("ok")


def test_sharded_osem_one_rank_equals_osem(cuda):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, __file__, str(port)], capture_output=True, text=True, env=env,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]


if __name__ == "__main__":
    _child(int(sys.argv[1]))

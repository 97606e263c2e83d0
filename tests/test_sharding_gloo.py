"""The sharded OSEM driver (petl_b200.sharding) with two and three gloo
ranks on the CPU: every rank owns a slab of v1 slices of each planogram,
the partial updates are summed by one all-reduce per subset, and the image
every rank ends with must equal single-process OSEM.  The per-rank
arithmetic is the FP64 oracle here (a test backend; the library's kernels
need a GPU), so the comparison checks the sharding, the exchange and the
update logic to FP64 round-off."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


class OracleBackend:
    """Per-rank arithmetic of sharded OSEM on the CPU oracle."""

    @staticmethod
    def ratio(G, f, g, out, subset, v1_range):
        import torch
        import oracle as O
        p = O.project_sub(G, f.numpy(), *subset)
        b, e = v1_range
        r = np.zeros_like(p)
        gv = g.numpy()
        nz = p[b:e] != 0.0
        rr = np.zeros_like(p[b:e])
        rr[nz] = gv[b:e][nz] / p[b:e][nz]
        r[b:e] = rr
        out.copy_(torch.from_numpy(r))

    @staticmethod
    def back(G, y, d, subset, v1_range):
        import torch
        import oracle as O
        b, e = v1_range
        ym = np.zeros(tuple(y.shape))
        ym[b:e] = y.numpy()[b:e]
        d += torch.from_numpy(O.backproject_sub(G, ym, *subset))

    @staticmethod
    def update(f, d, sens):
        import torch
        f *= torch.where(sens != 0, d / sens, torch.zeros_like(d))


def _case():
    import oracle as O
    vol = (32, 32, 8, 2.0)
    plans = [(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), (90.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)]
    geoms = [O.make_geom(*p, vol) for p in plans]
    rng = np.random.default_rng(12)
    f = np.zeros(geoms[0].vol_shape)
    f[2:6, 8:24, 8:24] = rng.uniform(0.5, 1.5, size=(4, 16, 16))
    g = [rng.poisson(np.maximum(p, 0.0)).astype(np.float64) for p in O.project(geoms, f)]
    return geoms, g


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from petl_b200.sharding import sharded_osem
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        geoms, g = _case()
        f = torch.ones(geoms[0].vol_shape, dtype=torch.float64)
        out = sharded_osem(geoms, [torch.from_numpy(x) for x in g], 2, 4, f=f, backend=OracleBackend)
        q.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_osem_equals_single_process(world):
    import multiprocessing as mp
    import socket
    import oracle as O
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    geoms, g = _case()
    want = O.osem(geoms, g, 2, 4)
    for rank, f in res:
        assert np.max(np.abs(f - want)) <= 1e-10 * np.max(np.abs(want)), rank
    # every rank holds the same image
    assert all(np.array_equal(res[0][1], f) for _, f in res)


def test_v1_shards_cover_every_slice_once():
    sys.path.insert(0, ROOT)
    from petl_b200.sharding import v1_shards
    for n, w in [(65, 8), (9, 2), (3, 4), (1, 1)]:
        sh = v1_shards(n, w)
        assert sh[0][0] == 0 and sh[-1][1] == n and len(sh) == w
        assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
        sizes = [e - b for b, e in sh]
        assert max(sizes) - min(sizes) <= 1

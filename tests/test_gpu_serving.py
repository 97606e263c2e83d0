"""The reconstruction server: continuous batching must not change results.

Each request's image is bit-identical whether it runs alone or in a mix of
requests of other geometries and sizes, equals the device-resident OSEM
driver on the same data, and admission keeps the reserved HBM within the
budget."""
import numpy as np
import pytest

from helpers import ellipsoids

pytestmark = pytest.mark.gpu

GEOMS = [
    ((0.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0), 4, 2),
    ((0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0), 8, 1),
    # rows not a multiple of 4 floats: first-generation shear kernels
    ((0.0, 100.0, 50.0, 26.0, 1.5, 0.45, 0.2), (50, 58, 15, 1.5, 1.5, 3.0, -4.5, 1.5), 3, 2),
    # psi = 30 degrees: general kernels
    ((30.0, 128.0, 64.0, 32.0, 2.0, 0.5, 0.25), (64, 64, 16, 2.0), 2, 1),
]


def _requests(cuda, seed=0):
    import torch
    from petl_b200 import Geometry, ops
    rng = np.random.default_rng(seed)
    out = []
    for args, vol, S, it in GEOMS:
        G = Geometry(*args, volume=vol)
        f = ellipsoids(G.vol_shape, (vol[3], vol[4] if len(vol) > 4 else vol[3]), rng, 6) + 0.05
        y = ops.project(G, torch.from_numpy(f.astype(np.float32)).to(cuda))
        y = torch.poisson(y * (1e5 / float(y.sum())), generator=torch.Generator(device=cuda).manual_seed(seed))
        host = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(y.cpu())
        out.append((G, host, S, it))
    return out


def test_alone_equals_mix_equals_driver(cuda):
    import torch
    from petl_b200 import recon
    from petl_b200.serving import ReconServer
    reqs = _requests(cuda)
    alone = []
    with ReconServer(hbm_budget_gb=40, max_active=1) as srv:
        for G, g, S, it in reqs:
            alone.append(srv.wait(srv.submit(G, g, S, it))[0])
    with ReconServer(hbm_budget_gb=40, max_active=8, depth=2) as srv:
        ids = [srv.submit(G, g, S, it) for G, g, S, it in reqs] + [srv.submit(G, g, S, it) for G, g, S, it in reqs]
        mix = [srv.wait(i)[0] for i in ids]
        st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    for a, b, c in zip(alone, mix[:len(reqs)], mix[len(reqs):]):
        assert np.array_equal(a, b) and np.array_equal(a, c)
    for (G, g, S, it), a in zip(reqs, alone):
        f, _ = recon.osem(G, g.to(cuda), it, S)
        assert np.abs(f.cpu().numpy() - a).max() <= 1e-6 * np.abs(a).max()


def test_admission_respects_budget(cuda):
    from petl_b200.serving import ReconServer
    reqs = _requests(cuda, seed=1)[:2]
    G, g, S, it = reqs[1]
    vol = np.prod(G.vol_shape) * 4
    need = 4 * 2 * np.prod(G.shape) + (2 + S) * vol
    budget = 1.5 * need / 1e9  # room for one such request at a time
    with ReconServer(hbm_budget_gb=budget, max_active=8) as srv:
        ids = [srv.submit(G, g, S, it) for _ in range(3)]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["hbm_peak_bytes"] <= budget * 1e9
    assert all(np.array_equal(res[0][0], r[0]) for r in res)
    # the later requests queued behind the budget
    assert res[2][2] > 0.0


def test_batched_launches_equal_alone(cuda):
    """Requests of one geometry and subset count share kernel launches, each
    at its own subset (subsets of unequal view counts included); every image
    equals the request run alone, bit for bit, and the batched server issued
    batched steps."""
    import time

    import torch
    from petl_b200 import Geometry, ops
    from petl_b200.serving import ReconServer
    args, vol = (0.0, 256.0, 128.0, 64.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0)
    G = Geometry(*args, volume=vol)
    S = 4
    assert G.shape[1] % S != 0  # subsets of unequal view counts
    rng = np.random.default_rng(11)
    data = []
    for k in range(6):
        f = ellipsoids(G.vol_shape, (2.0, 2.0), rng, 6) + 0.05
        y = ops.project(G, torch.from_numpy(f.astype(np.float32)).to(cuda))
        y = torch.poisson(y * (1e5 / float(y.sum())), generator=torch.Generator(device=cuda).manual_seed(k))
        host = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
        host.copy_(y.cpu())
        data.append((host, 1 + k % 3))
    with ReconServer(hbm_budget_gb=60, max_active=1) as srv:
        alone = [srv.wait(srv.submit(G, g, S, it))[0] for g, it in data]
        assert srv.batch_stats()["batched_steps"] == 0
    # all at once: like-geometry steps batched from the first step on
    with ReconServer(hbm_budget_gb=60, max_active=8, depth=2, batch=8) as srv:
        ids = [srv.submit(G, g, S, it) for g, it in data]
        together = [srv.wait(i)[0] for i in ids]
        bs = srv.batch_stats()
    assert bs["batched_steps"] > 0 and bs["member_steps"] >= 2 * bs["batched_steps"]
    # staggered: later requests join while the first ones are at other subsets
    with ReconServer(hbm_budget_gb=60, max_active=8, depth=1, batch=8) as srv:
        ids = []
        for g, it in data:
            ids.append(srv.submit(G, g, S, it))
            time.sleep(0.002)
        staggered = [srv.wait(i)[0] for i in ids]
    # batching off (the default): the same
    with ReconServer(hbm_budget_gb=60, max_active=8) as srv:
        ids = [srv.submit(G, g, S, it) for g, it in data]
        unbatched = [srv.wait(i)[0] for i in ids]
        assert srv.batch_stats()["batched_steps"] == 0
    for a, b, c, d in zip(alone, together, staggered, unbatched):
        assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)

"""Failure detection without a GPU fault.

* Bounded waits.  The projector kernels wait on their staged copies with a
  bounded number of polls; petl_force_wait_timeout(1) makes every such wait
  give up at once.  The kernels must then set the device error word, drain the
  copies they started (with the full bound) and return without hanging,
  the context must stay usable, the reference-compatible calls must report
  the failure (false -> TypeError in the binding), and with the default
  bound restored the same call must reproduce its earlier output bit for
  bit.  Covered for the split kernels (default dispatch) and the
  single-pass TMA kernels (dispatch 3), forward and both backward modes.
* Allocation failures.  petl_inject_alloc_failure(n) fails the n-th scratch
  allocation of a reference-compatible call; for every n the call either
  reports failure or, where the library falls back to a kernel family that
  needs no scratch, returns the right result, and the memory pool holds no
  allocation afterwards.
* Server deadlines and cancellation: a pending request past its deadline
  is dropped, a cancelled one fails, an active one stops between steps, and
  the server keeps serving with unchanged results.
"""
import time

import numpy as np
import pytest

from conftest import rel_l2
from helpers import ellipsoids

pytestmark = pytest.mark.gpu

ARGS = (0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25)
VOL = (128, 128, 64, 2.0)


def _setup(cuda):
    import torch
    from petl_b200 import Geometry
    G = Geometry(*ARGS, volume=VOL)
    f = ellipsoids(G.vol_shape, (2.0, 2.0), np.random.default_rng(5), 8) + 0.05
    return G, torch.from_numpy(f.astype(np.float32)).to(cuda)


def _timing_out(fn):
    import torch
    from petl_b200 import lib
    L = lib()
    assert L.petl_device_error_flag() == 0
    L.petl_force_wait_timeout(1)
    try:
        out = fn()
        torch.cuda.synchronize()
    finally:
        L.petl_force_wait_timeout(0)
    return out, L.petl_device_error_flag()


@pytest.mark.parametrize("dispatch", [0, 3])
def test_bounded_waits_give_up_and_the_device_stays_usable(cuda, dispatch):
    import torch
    from petl_b200 import lib, ops
    L = lib()
    G, f = _setup(cuda)
    assert L.petl_set_dispatch(dispatch) == 0
    try:
        want = ops.project(G, f)
        want_b = {m: ops.backproject(G, want, mode=m) for m in ("reference", "adjoint")}
        torch.cuda.synchronize()
        assert L.petl_last_projector_path() == 2 and L.petl_device_error_flag() == 0
        # every wait on staged data gives up at once: the kernels return
        _, flag = _timing_out(lambda: ops.project(G, f))
        assert flag == 1
        for m in ("reference", "adjoint"):
            _, flag = _timing_out(lambda: ops.backproject(G, want, mode=m))
            assert flag == 1
        # the same calls with the default bound reproduce the earlier outputs
        again = ops.project(G, f)
        assert torch.equal(again, want)
        for m in ("reference", "adjoint"):
            assert torch.equal(ops.backproject(G, want, mode=m), want_b[m])
        torch.cuda.synchronize()
        assert L.petl_device_error_flag() == 0
    finally:
        L.petl_set_dispatch(0)


def test_pfdr_wait_gives_up_and_recovers(cuda):
    import torch
    from petl_b200 import Geometry, lib, ops
    G = Geometry(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25, volume=(128, 128, 64, 2.0))
    y = torch.rand(G.shape, device=cuda, generator=torch.Generator(device=cuda).manual_seed(3))
    want = ops.pfdr(G, y)
    torch.cuda.synchronize()
    assert lib().petl_device_error_flag() == 0
    _, flag = _timing_out(lambda: ops.pfdr(G, y))
    assert flag == 1
    assert torch.equal(ops.pfdr(G, y), want)


def test_reference_calls_report_a_wait_that_gave_up(cuda):
    from petl_b200 import PETLserver, lib
    L = lib()
    G, f = _setup(cuda)
    s = PETLserver()
    s.add_planogram(*ARGS)
    s.set_volume(*VOL)
    fh = f.cpu().numpy()
    g = s.allocate_projections()
    s.project(g, fh)
    want = g[0].copy()
    L.petl_force_wait_timeout(1)
    try:
        with pytest.raises(TypeError):
            s.project(g, fh)
        with pytest.raises(TypeError):
            s.backproject(g, np.zeros_like(fh))
    finally:
        L.petl_force_wait_timeout(0)
    assert L.petl_device_error_flag() == 0  # the calls read and cleared it
    s.project(g, fh)
    assert np.array_equal(g[0], want)


def test_injected_allocation_failures_leak_nothing(cuda):
    import torch
    from petl_b200 import PETLserver, lib
    L = lib()
    G, f = _setup(cuda)
    s = PETLserver()
    s.add_planogram(*ARGS)
    s.set_volume(*VOL)
    fh = f.cpu().numpy()
    g = s.allocate_projections()
    b = np.zeros_like(fh)
    torch.cuda.synchronize()
    base = L.petl_scratch_in_use()
    assert base >= 0
    c0 = L.petl_scratch_alloc_count()
    s.project(g, fh)
    want_g = g[0].copy()
    c1 = L.petl_scratch_alloc_count()
    s.backproject(g, b)
    want_b = b.copy()
    c2 = L.petl_scratch_alloc_count()
    n_proj, n_back = c1 - c0, c2 - c1
    assert n_proj >= 2 and n_back >= 2
    for call, n, check in (("project", n_proj, lambda: rel_l2(g[0], want_g) == 0.0),
                           ("backproject", n_back, lambda: rel_l2(b, want_b) == 0.0)):
        for k in range(1, n + 1):
            g[0][:] = want_g
            b[:] = -1.0
            L.petl_inject_alloc_failure(k)
            try:
                if call == "project":
                    s.project(g, fh)
                else:
                    s.backproject(g, b)
                ok = True
            except TypeError:
                ok = False
            finally:
                L.petl_inject_alloc_failure(0)
            torch.cuda.synchronize()
            if ok:  # a fallback without the failed scratch: the result must still hold
                assert check(), (call, k)
            assert L.petl_scratch_in_use() == base, (call, k)
            assert L.petl_device_error_flag() == 0
    # and a clean call afterwards
    s.project(g, fh)
    assert np.array_equal(g[0], want_g)


def test_server_deadlines_and_cancellation(cuda):
    import torch
    from petl_b200 import PetlError, ops, recon
    from petl_b200.serving import ReconServer
    G, f = _setup(cuda)
    y = ops.project(G, f)
    y = torch.poisson(y * (1e6 / float(y.sum())), generator=torch.Generator(device=cuda).manual_seed(1))
    host = torch.empty(y.shape, dtype=torch.float32, pin_memory=True)
    host.copy_(y.cpu())
    with ReconServer(hbm_budget_gb=40, max_active=1) as srv:
        a = srv.submit(G, host, 8, 40)             # holds the only slot for a while
        b = srv.submit(G, host, 8, 2, deadline_s=0.0)
        c = srv.submit(G, host, 8, 2)
        srv.cancel(c)
        d = srv.submit(G, host, 4, 2)
        with pytest.raises(PetlError, match="deadline exceeded before admission"):
            srv.wait(b)
        with pytest.raises(PetlError, match="cancelled"):
            srv.wait(c)
        fa = srv.wait(a)[0]
        fd = srv.wait(d)[0]
        # an active request stops between steps at its deadline
        t0 = time.perf_counter()
        e = srv.submit(G, host, 8, 100000, deadline_s=0.2)
        with pytest.raises(PetlError, match="deadline exceeded"):
            srv.wait(e)
        assert time.perf_counter() - t0 < 30.0
        # and an active one that is cancelled
        h = srv.submit(G, host, 8, 100000)
        while srv.stats()["active"] < 1:
            time.sleep(0.01)
        srv.cancel(h)
        with pytest.raises(PetlError, match="cancelled"):
            srv.wait(h)
        fd2 = srv.wait(srv.submit(G, host, 4, 2))[0]
        st = srv.stats()
    assert st["failed"] == 4 and st["completed"] == 3
    assert np.array_equal(fd, fd2)
    for got, S, it in ((fa, 8, 40), (fd, 4, 2)):
        want, _ = recon.osem(G, host.to(cuda), it, S)
        assert np.abs(want.cpu().numpy() - got).max() <= 1e-6 * np.abs(got).max()

"""Host <-> device copies of caller arrays: pageable host arrays move
through the library's pinned ring (several 32 MB buffers), pinned ones
directly.  Round trips must reproduce the data exactly for sizes from empty
to several ring buffers, with byte counts that fill no buffer evenly."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pinned", [False, True])
def test_copy_round_trips(cuda, pinned):
    import torch
    from petl_b200 import lib
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(1)
    for nbytes in (0, 1, 4097, (32 << 20) + 12345, (100 << 20) + 3):
        src = rng.integers(0, 256, size=nbytes, dtype=np.uint8)
        if pinned:
            t = torch.from_numpy(src.copy()).pin_memory()
            src_h = t.numpy()
            back = torch.empty(nbytes, dtype=torch.uint8).pin_memory().numpy()
        else:
            src_h = src
            back = np.empty(nbytes, np.uint8)
        dev = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=cuda)
        assert lib().petl_copy_to_device(ctypes.c_void_p(dev.data_ptr()), ctypes.c_void_p(src_h.ctypes.data),
                                         nbytes, st) == 0
        assert lib().petl_copy_to_host(ctypes.c_void_p(back.ctypes.data), ctypes.c_void_p(dev.data_ptr()),
                                       nbytes, st) == 0
        assert np.array_equal(back, src)
        if nbytes:
            assert np.array_equal(dev[:nbytes].cpu().numpy(), src)


def test_concurrent_copies_share_the_ring(cuda):
    """An upload on one stream and a download on another, from two host
    threads at once, each through more than four ring buffers of pageable
    memory: the shared pinned ring must hand a slot to the download only
    after the upload's copy out of it finished (both round trips exact)."""
    import threading

    import torch
    from petl_b200 import lib
    L = lib()
    nbytes = (200 << 20) + 77  # seven 32 MB ring buffers and a ragged tail
    rng = np.random.default_rng(7)
    up_src = rng.integers(0, 256, size=nbytes, dtype=np.uint8)
    down_src = rng.integers(0, 256, size=nbytes, dtype=np.uint8)
    dev_up = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    dev_down = torch.from_numpy(down_src).to(cuda)
    down_back = np.empty(nbytes, np.uint8)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    rcs = {}

    def up():
        for _ in range(3):
            rcs.setdefault("up", []).append(L.petl_copy_to_device(
                ctypes.c_void_p(dev_up.data_ptr()), ctypes.c_void_p(up_src.ctypes.data), nbytes,
                ctypes.c_void_p(s1.cuda_stream)))

    def down():
        for _ in range(3):
            rcs.setdefault("down", []).append(L.petl_copy_to_host(
                ctypes.c_void_p(down_back.ctypes.data), ctypes.c_void_p(dev_down.data_ptr()), nbytes,
                ctypes.c_void_p(s2.cuda_stream)))

    th = [threading.Thread(target=up), threading.Thread(target=down)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    assert rcs["up"] == [0, 0, 0] and rcs["down"] == [0, 0, 0]
    assert np.array_equal(dev_up.cpu().numpy(), up_src)
    assert np.array_equal(down_back, down_src)

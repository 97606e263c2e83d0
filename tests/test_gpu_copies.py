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

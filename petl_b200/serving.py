"""Reconstruction server (continuous batching on one GPU), Python front end.

``ReconServer`` wraps the C++ server of libpetl.so (include/petl_device.h,
petl_server_*): requests are OSEM reconstructions of one planogram each,
admitted by HBM budget and run concurrently on their own CUDA streams;
like-geometry requests may share kernel launches (batched steps, off by
default).  The
planogram of a request must stay alive until its result is collected; the
front end keeps a reference for that.  Use pinned host tensors
(``torch.empty(..., pin_memory=True)``) for the data so that the copy in is
asynchronous.
"""
import ctypes

import numpy as np

from ._lib import check, lib


class ReconServer:
    def __init__(self, hbm_budget_gb=150.0, max_active=16, depth=2, device=0, batch=1):
        """batch: members of a batched step at most (1, the default: every
        request launches its own kernels on its own stream; up to 8: small
        steps of like-geometry requests share launches, which measured the
        same throughput and a higher p99 on the serving workload)."""
        L = lib()
        self._s = L.petl_server_create(float(hbm_budget_gb) * 1e9, int(max_active), int(depth), int(device))
        if not self._s:
            raise RuntimeError(L.petl_last_error().decode())
        self._keep = {}
        self._shapes = {}
        check(L.petl_server_set_batching(self._s, int(batch)), "server_set_batching")

    def submit(self, geom, g, num_subsets, num_iter, deadline_s=None):
        """Queue OSEM of planogram ``g`` (float32, host numpy array or CPU
        tensor, contiguous, shape geom.shape); returns the request id.  With
        ``deadline_s`` the request fails ("deadline exceeded") if it has not
        finished that many seconds after submission: dropped before
        admission, or stopped between subset steps."""
        if hasattr(g, "data_ptr"):
            ptr = g.data_ptr()
            assert g.dtype.__str__() == "torch.float32" and g.is_contiguous() and not g.is_cuda
        else:
            g = np.ascontiguousarray(g, dtype=np.float32)
            ptr = g.ctypes.data
        assert tuple(g.shape) == tuple(geom.shape), (g.shape, geom.shape)
        rid = ctypes.c_longlong(0)
        dl = -1.0 if deadline_s is None else float(deadline_s)
        check(lib().petl_server_submit_deadline(self._s, geom.ptr, ctypes.c_void_p(ptr), int(num_subsets),
                                                int(num_iter), dl, ctypes.byref(rid)), "server_submit")
        self._keep[rid.value] = (g, geom)
        self._shapes[rid.value] = tuple(geom.vol_shape)
        return rid.value

    def wait(self, rid):
        """(image as a float32 numpy array, latency s, queueing s)."""
        out = np.empty(self._shapes[rid], np.float32)
        lat, q = ctypes.c_double(0.0), ctypes.c_double(0.0)
        rc = lib().petl_server_wait(self._s, ctypes.c_longlong(rid), ctypes.c_void_p(out.ctypes.data),
                                    ctypes.byref(lat), ctypes.byref(q))
        self._keep.pop(rid, None)
        self._shapes.pop(rid, None)
        check(rc, "server_wait")
        return out, lat.value, q.value

    def cancel(self, rid):
        """Cancel a request (its wait() then raises with "cancelled")."""
        check(lib().petl_server_cancel(self._s, ctypes.c_longlong(rid)), "server_cancel")

    def stats(self):
        buf = (ctypes.c_double * 6)()
        lib().petl_server_stats(self._s, buf)
        keys = ("completed", "failed", "active", "pending", "hbm_bytes", "hbm_peak_bytes")
        return dict(zip(keys, list(buf)))

    def batch_stats(self):
        """Batched steps issued so far and the member steps they served."""
        buf = (ctypes.c_double * 2)()
        lib().petl_server_batch_stats(self._s, buf)
        return {"batched_steps": int(buf[0]), "member_steps": int(buf[1])}

    def close(self):
        if self._s:
            lib().petl_server_destroy(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

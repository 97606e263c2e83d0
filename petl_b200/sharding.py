"""One-exchange sharding of OSEM / MLEM over GPUs, one process per GPU.

Each rank owns a contiguous slab of v1 slices of every planogram (the
oblique segments of the reference's planogram layout, src/planogram.cpp:
143-186) and keeps the full image.  Per subset a rank computes the data
ratio g / P f for its own slices (the forward projection needs no exchange:
the image is replicated) and backprojects them into a partial update; the
partial updates are summed over ranks by one all-reduce of the image, and
every rank then applies the same multiplicative update, so the images stay
identical.  The sensitivity of each subset is built the same way once.  This
is the reference's own planogram-level split (src/petl.cpp:235-273 sums the
per-planogram backprojections on the host) moved to slices within planograms
and to a collective over NVLink.

The arithmetic runs through a backend with four operations (ratio, back,
update, and fill helpers); ``DeviceBackend`` is the library's kernels.  With
one rank the result equals ``recon.osem`` bit for bit.
"""
import torch
import torch.distributed as dist

from . import ops
from .geometry import as_list


def v1_shards(n_v1, world):
    """Contiguous [begin, end) ranges of v1 slices per rank, sizes differing
    by at most one (a rank may own none when n_v1 < world)."""
    base, extra = divmod(int(n_v1), int(world))
    out, b = [], 0
    for r in range(world):
        e = b + base + (1 if r < extra else 0)
        out.append((b, e))
        b = e
    return out


class DeviceBackend:
    """The library's kernels on CUDA tensors."""

    @staticmethod
    def ratio(G, f, g, out, subset, v1_range):
        return ops.project_ratio(G, f, g, out=out, subset=subset, v1_range=v1_range)

    @staticmethod
    def back(G, y, d, subset, v1_range):
        ops.backproject(G, y, f=d, accumulate=True, subset=subset, v1_range=v1_range)

    @staticmethod
    def update(f, d, sens):
        ops.mlem_update_(f, d, sens)


def sharded_osem(geoms, g, num_iter, num_subsets, f=None, group=None, backend=None):
    """OSEM with interleaved view subsets (iv0 mod S), the planograms' v1
    slices split over the ranks of ``group``; one all-reduce (sum) of the
    image per subset step.  Every rank passes the full planograms g (only
    its own slices are read) and gets the same image back."""
    backend = backend or DeviceBackend
    geoms = as_list(geoms)
    gl = as_list(g)
    rank = dist.get_rank(group) if group is not None or dist.is_initialized() else 0
    world = dist.get_world_size(group) if group is not None or dist.is_initialized() else 1
    shards = [v1_shards(G.shape[0], world)[rank] for G in geoms]
    S = int(num_subsets)
    if f is None:
        f = torch.ones(geoms[0].vol_shape, device=gl[0].device, dtype=torch.float32)
    elif not torch.any(f):
        f.fill_(1.0)
    else:
        f.clamp_(min=0.0)

    def reduce_(x):
        if world > 1:
            dist.all_reduce(x, op=dist.ReduceOp.SUM, group=group)
        return x

    sens = []
    for s in range(S):
        d = torch.zeros_like(f)
        for G, gi, sh in zip(geoms, gl, shards):
            if sh[1] > sh[0]:
                backend.back(G, torch.ones_like(gi), d, (s, S), sh)
        reduce_(d)
        d[d == 0.0] = 1.0
        sens.append(d)
    ratio = [torch.zeros_like(x) for x in gl]
    d = torch.empty_like(f)
    for _ in range(num_iter):
        for s in range(S):
            d.zero_()
            for G, gi, ri, sh in zip(geoms, gl, ratio, shards):
                if sh[1] > sh[0]:
                    backend.ratio(G, f, gi, ri, (s, S), sh)
                    backend.back(G, ri, d, (s, S), sh)
            reduce_(d)
            backend.update(f, d, sens[s])
    return f

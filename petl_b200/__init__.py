"""petl_b200: B200-native planogram PET reconstruction core.

* ``petl_b200.PETLserver`` -- the reference Python operator surface
  (src/petl_server.py) over the reference-compatible C ABI of libpetl.so;
  numpy arrays in, numpy arrays out.
  ``petl_b200.PETXserver`` -- the PET/X scanner preset on top of it.
* ``petl_b200.ops`` -- device-resident operators on torch CUDA tensors.
* ``petl_b200.recon`` -- MLEM / OSEM / RWLS drivers that stay on the GPU.
* ``petl_b200.autograd`` -- torch.autograd.Function wrappers (projector with
  its exact adjoint as backward, RD and TV penalties).
* ``petl_b200.Geometry`` -- one planogram plus its volume.
"""
from ._lib import LIB_PATH, PetlError, lib  # noqa: F401
from .geometry import Geometry  # noqa: F401


def __getattr__(name):
    # heavy submodules (torch) load lazily
    if name in ("ops", "recon", "autograd", "server", "serving"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    if name in ("PETLserver", "PETXserver"):
        from . import server
        return getattr(server, name)
    raise AttributeError(name)

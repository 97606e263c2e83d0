"""Device-resident operators on torch CUDA tensors.

Each function calls one entry point of ``libpetl.so`` (include/petl_device.h)
on the current torch stream; tensors must be contiguous float32 CUDA tensors.
PyTorch provides only device memory and streams here.  Scalars that the
library reduces in FP64 come back as float64 0-d CUDA tensors (no host sync).
"""
import ctypes

import numpy as np
import torch

from ._lib import PetlError, check, lib
from .geometry import Geometry, as_list

REFERENCE = 0
ADJOINT = 1
_MODES = {"reference": REFERENCE, "adjoint": ADJOINT, REFERENCE: REFERENCE, ADJOINT: ADJOINT}


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(t, name="tensor"):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise PetlError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float32:
        raise PetlError(f"{name} must be float32")
    if not t.is_contiguous():
        raise PetlError(f"{name} must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def _n(t):
    return ctypes.c_longlong(t.numel())


def _dev16(t, name="tensor"):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise PetlError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.bfloat16:
        raise PetlError(f"{name} must be bfloat16")
    if not t.is_contiguous():
        raise PetlError(f"{name} must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


# ----------------------------------------------------------------------------
# projectors
# ----------------------------------------------------------------------------
def project(geom, f, g=None, subset=None, v1_range=None):
    """g = P f (reference src/projectors.cu:11-238).

    ``subset=(first, step)`` computes only the views iv0 = first + k*step and
    leaves the others of ``g`` untouched; ``v1_range=(b, e)`` restricts the
    v1 slices.  ``geom`` may be a list of geometries (one planogram each), in
    which case ``g`` is a list."""
    geoms = as_list(geom)
    if g is None:
        g = [torch.zeros(G.shape, device=f.device, dtype=torch.float32) for G in geoms]
    gl = as_list(g)
    first, step = subset if subset is not None else (0, 1)
    for G, gi in zip(geoms, gl):
        b, e = v1_range if v1_range is not None else (0, G.shape[0])
        check(lib().petl_project_range_dev(G.ptr, _dev(f, "f"), _dev(gi, "g"), b, e, first, step, _stream()),
              "project")
    return g if isinstance(geom, (list, tuple)) else gl[0]


def bin_events(geom, blue, pink, g=None, linear=True, chest_wall=True):
    """Coincidences blue[i], pink[i] ((n, 3) float32 device tensors, mm)
    binned into the planogram(s) of ``geom`` (src/binning.cpp:614-790):
    bilinear in (u1, u0) (the reference's binning) or the nearest bin, z from
    the chest wall (the reference's origin) or from the centre.  A new,
    zeroed ``g`` is allocated unless given; a given ``g`` is added to."""
    geoms = as_list(geom)
    if g is None:
        g = [torch.zeros(G.shape, device=blue.device, dtype=torch.float32) for G in geoms]
    gl = as_list(g)
    n = int(blue.shape[0]) if blue.dim() > 1 else int(blue.numel()) // 3
    if int(pink.numel()) != 3 * n or int(blue.numel()) != 3 * n:
        raise ValueError("bin_events: blue and pink must both hold n xyz triples")
    for G, gi in zip(geoms, gl):
        check(lib().petl_bin_events_dev(G.ptr, _dev(blue, "blue"), _dev(pink, "pink"), n, _dev(gi, "g"),
                                        1 if linear else 0, 1 if chest_wall else 0, _stream()), "bin_events")
    return g if isinstance(geom, (list, tuple)) else gl[0]


# ----------------------------------------------------------------------------
# analytic phantoms
# ----------------------------------------------------------------------------
SOLID_TYPES = {"ellipsoid": 0, "ball": 0, "sphere": 0, "parallelepiped": 1, "box": 1, "can_x": 2, "can_y": 3,
               "can_z": 4, "can": 4, "cone_x": 5, "cone_y": 6, "cone_z": 7, "cone": 7}


def make_solid(kind, c, r, val, A=None, clip=None):
    """One analytic solid (geometricObject::init, src/phantom.cpp:535-640):
    kind is a type number 0..7 or a name (ellipsoid, box, can_x/y/z, cone_x/y/z);
    A a 3x3 rotation (default identity), clip per-axis clipping (default none)."""
    from ._lib import petl_solid
    t = SOLID_TYPES[kind.lower()] if isinstance(kind, str) else int(kind)
    c = np.ascontiguousarray(np.broadcast_to(np.asarray(c, np.float32), (3,)))
    r = np.ascontiguousarray(np.broadcast_to(np.asarray(r, np.float32), (3,)))
    A = np.eye(3, dtype=np.float32) if A is None else np.ascontiguousarray(A, np.float32)
    clip = np.zeros(3, np.float32) if clip is None else np.ascontiguousarray(clip, np.float32)
    s = petl_solid()
    fptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))  # noqa: E731
    if lib().petl_solid_init(ctypes.byref(s), t, fptr(c), fptr(r), float(val), fptr(A), fptr(clip)) != 0:
        raise ValueError("invalid solid")
    return s


def _solid_array(solids):
    from ._lib import petl_solid
    arr = (petl_solid * max(1, len(solids)))(*solids)
    return arr, len(solids)


def voxelize_(f, solids, voxel_width, voxel_height=None, x_0=None, y_0=None, z_0=None, oversampling=1):
    """Writes the solids, in order, into the device volume f [z][y][x]
    (phantom::voxelize, src/phantom.cpp:105-335); x_0/y_0/z_0 default to a
    volume centred on the origin."""
    nz, ny, nx = f.shape
    vh = voxel_width if voxel_height is None else voxel_height
    x_0 = float(np.float32(-0.5 * (nx - 1) * voxel_width)) if x_0 is None else x_0
    y_0 = float(np.float32(-0.5 * (ny - 1) * voxel_width)) if y_0 is None else y_0
    z_0 = float(np.float32(-0.5 * (nz - 1) * vh)) if z_0 is None else z_0
    arr, n = _solid_array(solids)
    check(lib().petl_voxelize_dev(arr, n, _dev(f, "f"), nx, ny, nz, float(voxel_width), float(vh), float(x_0),
                                  float(y_0), float(z_0), int(oversampling), _stream()), "voxelize")
    return f


def ray_trace(geom, solids, g=None, oversampling=1, stopping_power=False):
    """Analytic ray tracing of the planogram(s) through the solids
    (src/analytic_ray_tracing_gpu.cu:693-994): line integrals, or with
    stopping_power the product of the two half-lines' absorption
    probabilities."""
    geoms = as_list(geom)
    if g is None:
        g = [torch.empty(G.shape, device="cuda", dtype=torch.float32) for G in geoms]
    gl = as_list(g)
    arr, n = _solid_array(solids)
    for G, gi in zip(geoms, gl):
        check(lib().petl_ray_trace_dev(G.ptr, arr, n, _dev(gi, "g"), int(oversampling), 1 if stopping_power else 0,
                                       _stream()), "ray_trace")
    return g if isinstance(geom, (list, tuple)) else gl[0]


def solid_angle_(geom, g, inverse=False):
    """Scales each projection (iv1, iv0) of the planogram(s) g in place by the
    solid-angle correction 2 pi (1 + v0^2 + v1^2)^1.5 / (T_v1 T_v0), or by
    its inverse, the solid-angle model (src/planogram.cpp:262-302)."""
    for G, gi in zip(as_list(geom), as_list(g)):
        check(lib().petl_solid_angle_dev(G.ptr, _dev(gi, "g"), 1 if inverse else 0, _stream()), "solid_angle")
    return g


def apply_corrections_(geom, g, r, threshold=0.75):
    """PETL::apply_corrections in place on device planograms: g = g / r, then
    per projection the bins outside the field of view are zeroed and the bins
    whose response is below threshold * median(r) get the median of their
    5x5 window's divided values above that level (src/petl.cpp:163-192,
    src/median_filter.cu)."""
    for G, gi, ri in zip(as_list(geom), as_list(g), as_list(r)):
        if tuple(gi.shape) != tuple(G.shape) or tuple(ri.shape) != tuple(G.shape):
            raise ValueError("apply_corrections: g and r must have the planogram's shape")
        check(lib().petl_apply_corrections_dev(G.ptr, _dev(gi, "g"), _dev(ri, "r"), float(threshold), _stream()),
              "apply_corrections")
    return g


def project_ratio(geom, f, meas, out=None, subset=None, v1_range=None):
    """out = meas / (P f) with 0 where P f == 0 (the MLEM data ratio of the
    reference, src/petl_server.py:1593-1594), computed inside the projector."""
    geoms = as_list(geom)
    ml = as_list(meas)
    if out is None:
        out = [torch.empty_like(m) for m in ml]
    ol = as_list(out)
    first, step = subset if subset is not None else (0, 1)
    for G, mi, oi in zip(geoms, ml, ol):
        b, e = v1_range if v1_range is not None else (0, G.shape[0])
        check(lib().petl_project_ratio_dev(G.ptr, _dev(f, "f"), _dev(mi, "meas"), _dev(oi, "out"), b, e, first, step,
                                           _stream()), "project_ratio")
    return out if isinstance(geom, (list, tuple)) else ol[0]


def backproject(geom, g, f=None, mode="reference", accumulate=False, scale=1.0, subset=None, v1_range=None):
    """f = P^T g summed over planograms.

    mode 'reference' follows the reference backprojector's visibility rules
    (src/projectors.cu:240-377) with exact bilinear weights; mode 'adjoint'
    is the exact transpose of ``project``."""
    geoms = as_list(geom)
    gl = as_list(g)
    if f is None:
        f = torch.empty(geoms[0].vol_shape, device=gl[0].device, dtype=torch.float32)
        accumulate = False
    first, step = subset if subset is not None else (0, 1)
    m = _MODES[mode]
    for i, (G, gi) in enumerate(zip(geoms, gl)):
        b, e = v1_range if v1_range is not None else (0, G.shape[0])
        acc = 1 if (accumulate or i > 0) else 0
        check(lib().petl_backproject_range_dev(G.ptr, _dev(gi, "g"), _dev(f, "f"), m, acc, float(scale), b, e,
                                               first, step, _stream()), "backproject")
    return f


# ----------------------------------------------------------------------------
# BF16 storage: bfloat16 volumes / planograms, FP32 footprint accumulation
# ----------------------------------------------------------------------------
def project_bf16(geom, f, g=None, subset=None, v1_range=None):
    """g = P f with f and g in bfloat16 (one geometry)."""
    if g is None:
        g = torch.zeros(geom.shape, device=f.device, dtype=torch.bfloat16)
    first, step = subset if subset is not None else (0, 1)
    b, e = v1_range if v1_range is not None else (0, geom.shape[0])
    check(lib().petl_project_bf16_dev(geom.ptr, _dev16(f, "f"), _dev16(g, "g"), b, e, first, step, _stream()),
          "project_bf16")
    return g


def project_ratio_bf16(geom, f, meas, out=None, subset=None, v1_range=None):
    """out = meas / (P f) (0 where P f == 0), all bfloat16."""
    if out is None:
        out = torch.empty_like(meas)
    first, step = subset if subset is not None else (0, 1)
    b, e = v1_range if v1_range is not None else (0, geom.shape[0])
    check(lib().petl_project_ratio_bf16_dev(geom.ptr, _dev16(f, "f"), _dev16(meas, "meas"), _dev16(out, "out"), b, e,
                                            first, step, _stream()), "project_ratio_bf16")
    return out


def backproject_bf16(geom, g, f=None, mode="reference", accumulate=False, scale=1.0, subset=None, v1_range=None):
    """f (float32) = P^T g with g in bfloat16."""
    if f is None:
        f = torch.empty(geom.vol_shape, device=g.device, dtype=torch.float32)
        accumulate = False
    first, step = subset if subset is not None else (0, 1)
    b, e = v1_range if v1_range is not None else (0, geom.shape[0])
    check(lib().petl_backproject_bf16_dev(geom.ptr, _dev16(g, "g"), _dev(f, "f"), _MODES[mode], 1 if accumulate else 0,
                                          float(scale), b, e, first, step, _stream()), "backproject_bf16")
    return f


def to_bf16(x, out=None):
    """bfloat16 copy of a float32 tensor (round to nearest even)."""
    if out is None:
        out = torch.empty(x.shape, device=x.device, dtype=torch.bfloat16)
    check(lib().petl_to_bf16_dev(_dev(x, "x"), _dev16(out, "out"), _n(x), _stream()), "to_bf16")
    return out


def mlem_update_bf16_(f, d, sens):
    """f (bfloat16) *= d / sens with d/0 -> 0."""
    check(lib().petl_mlem_update_bf16_dev(_dev16(f, "f"), _dev(d, "d"), _dev(sens, "sens"), _n(f), _stream()),
          "mlem_update_bf16")
    return f


def nnz(geom):
    """Exact count of nonzero (ray, voxel) footprint weights of P."""
    out = ctypes.c_double(0.0)
    check(lib().petl_project_nnz_dev(geom.ptr, ctypes.byref(out), _stream()), "project_nnz")
    return out.value


# ----------------------------------------------------------------------------
# PFDR / ramp / FBP
# ----------------------------------------------------------------------------
def pfdr(geom, g, g_reb=None):
    """PFDR rebinning (src/pfdr.cu:159-315) -> [N_v0][N_u1][N_u0]."""
    if g_reb is None:
        g_reb = torch.empty(geom.rebinned_shape, device=g.device, dtype=torch.float32)
    check(lib().petl_pfdr_dev(geom.ptr, _dev(g, "g"), _dev(g_reb, "g_reb"), _stream()), "PFDR")
    return g_reb


def ramp_(geom_reb, g_reb, apply_weight=True):
    """In-place ramp filter of a rebinned planogram (src/ramp_filter.cu:156-348),
    followed by the inverse planogram weight when ``apply_weight``."""
    check(lib().petl_ramp_dev(geom_reb.ptr, _dev(g_reb, "g_reb"), 1 if apply_weight else 0, _stream()), "ramp")
    return g_reb


def fbp(geom, g, f=None, accumulate=False):
    """FBP of one or more planograms (PETL::doFBP, src/petl.cpp:310-355)."""
    geoms = as_list(geom)
    gl = as_list(g)
    if f is None:
        f = torch.empty(geoms[0].vol_shape, device=gl[0].device, dtype=torch.float32)
        accumulate = False
    for i, (G, gi) in enumerate(zip(geoms, gl)):
        check(lib().petl_fbp_dev(G.ptr, _dev(gi, "g"), _dev(f, "f"), 1 if (accumulate or i > 0) else 0, _stream()),
              "FBP")
    return f


# ----------------------------------------------------------------------------
# regularizers: volumes [N1][N2][N3] (2-D inputs are treated as N1 = 1)
# ----------------------------------------------------------------------------
def _dims(f):
    s = tuple(f.shape)
    if len(s) == 2:
        return (1,) + s
    if len(s) != 3:
        raise PetlError("regularizers take 2-D or 3-D arrays")
    return s


def _scalar(f):
    return torch.zeros((), device=f.device, dtype=torch.float64)


def rd_gradient(f, delta, beta, out=None):
    out = torch.empty_like(f) if out is None else out
    check(lib().petl_rd_gradient_dev(_dev(f, "f"), _dev(out, "Df"), *_dims(f), float(delta), float(beta), _stream()),
          "rd_gradient")
    return out


def rd_cost(f, delta, beta):
    out = _scalar(f)
    check(lib().petl_rd_cost_dev(_dev(f, "f"), *_dims(f), float(delta), float(beta), ctypes.c_void_p(out.data_ptr()),
                                 _stream()), "rd_cost")
    return out


def tv_gradient(f, delta, beta=0.0, p=1.0, num_neighbors=26, out=None):
    out = torch.empty_like(f) if out is None else out
    check(lib().petl_tv_gradient_dev(_dev(f, "f"), _dev(out, "Df"), *_dims(f), float(delta), float(beta), float(p),
                                     int(num_neighbors), _stream()), "tv_gradient")
    return out


def tv_cost(f, delta, beta=0.0, p=1.0, num_neighbors=26):
    out = _scalar(f)
    check(lib().petl_tv_cost_dev(_dev(f, "f"), *_dims(f), float(delta), float(beta), float(p), int(num_neighbors),
                                 ctypes.c_void_p(out.data_ptr()), _stream()), "tv_cost")
    return out


def tv_quadform(f, d, delta, beta=0.0, p=1.0, num_neighbors=26):
    out = _scalar(f)
    check(lib().petl_tv_quadform_dev(_dev(f, "f"), _dev(d, "d"), *_dims(f), float(delta), float(beta), float(p),
                                     int(num_neighbors), ctypes.c_void_p(out.data_ptr()), _stream()), "tv_quadform")
    return out


def gaussian_filter_(f, fwhm=2.0, num_dims=3):
    check(lib().petl_gaussian_filter_dev(_dev(f, "f"), *_dims(f), float(fwhm), int(num_dims), _stream()),
          "gaussian_filter")
    return f


# ----------------------------------------------------------------------------
# elementwise / reductions
# ----------------------------------------------------------------------------
def rdivide_(denom, num):
    """denom = num / denom, 0 where denom == 0 (reference RDIV)."""
    check(lib().petl_rdivide_dev(_dev(num, "num"), _dev(denom, "denom"), _n(denom), _stream()), "rdivide")
    return denom


def divide_(x, y):
    """x = x / y, 0 where y == 0 (reference DIV)."""
    check(lib().petl_divide_dev(_dev(x, "x"), _dev(y, "y"), _n(x), _stream()), "divide")
    return x


def multiply_(x, y):
    check(lib().petl_multiply_dev(_dev(x, "x"), _dev(y, "y"), _n(x), _stream()), "multiply")
    return x


def reciprocal_(x, divide_by_zero_value=0.0):
    check(lib().petl_reciprocal_dev(_dev(x, "x"), _n(x), float(divide_by_zero_value), _stream()), "reciprocal")
    return x


def axpby_(x, y, a, b):
    check(lib().petl_axpby_dev(_dev(x, "x"), _dev(y, "y"), float(a), float(b), _n(x), _stream()), "axpby")
    return x


def dot(x, y, w=None):
    """sum(x*y*w) accumulated in FP64 on the device (0-d float64 tensor)."""
    out = _scalar(x)
    wp = _dev(w, "w") if w is not None else ctypes.c_void_p(0)
    check(lib().petl_dot_dev(_dev(x, "x"), _dev(y, "y"), wp, _n(x), ctypes.c_void_p(out.data_ptr()), _stream()),
          "dot")
    return out


def loglik(g, Pf):
    """Poisson log-likelihood sum(g log Pf - Pf) over Pf > 0, FP64."""
    out = _scalar(g)
    check(lib().petl_loglik_dev(_dev(g, "g"), _dev(Pf, "Pf"), _n(g), ctypes.c_void_p(out.data_ptr()), _stream()),
          "loglik")
    return out


def poisson_grad_(Pf, g):
    """Pf = 1 - g/Pf where Pf > 0, else 0, in place: d/d(Pf) of the Poisson
    negative log-likelihood sum(Pf - g log Pf)."""
    check(lib().petl_poisson_grad_dev(_dev(Pf, "Pf"), _dev(g, "g"), _n(Pf), _stream()), "poisson_grad")
    return Pf


def mlem_update_(f, d, sens):
    check(lib().petl_mlem_update_dev(_dev(f, "f"), _dev(d, "d"), _dev(sens, "sens"), _n(f), _stream()), "mlem_update")
    return f


def osl_update_(f, d, sens, Df):
    check(lib().petl_osl_update_dev(_dev(f, "f"), _dev(d, "d"), _dev(sens, "sens"), _dev(Df, "Df"), _n(f),
                                    _stream()), "osl_update")
    return f


__all__ = ["Geometry", "project", "project_ratio", "backproject", "nnz", "pfdr", "ramp_", "fbp", "rd_gradient", "rd_cost",
           "tv_gradient", "tv_cost", "tv_quadform", "gaussian_filter_", "rdivide_", "divide_", "multiply_",
           "reciprocal_", "axpby_", "dot", "loglik", "poisson_grad_", "mlem_update_", "osl_update_", "project_bf16",
           "project_ratio_bf16", "backproject_bf16", "mlem_update_bf16_", "to_bf16", "REFERENCE", "ADJOINT"]

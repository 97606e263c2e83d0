"""ctypes face of the CPU oracle (``liboracle.so``) -- test infrastructure only.

The C++ restatement lives in ``oracle.cpp``; this module adds the pieces the
reference writes in Python or composes on the host:

* the C-ABI conventions of ``add_planogram`` (full lengths halved, psi in
  degrees; reference ``src/petl_c_interface.cpp:216-219``),
* multi-planogram projection / backprojection (``src/petl.cpp:205-277``),
* FBP as ``PETL::doFBP`` composes it (``src/petl.cpp:310-355``),
* the MLEM loop of ``PETLserver.MLEM`` (``src/petl_server.py:1534-1606``)
  with the dataCube elementwise rules (``src/data_cube.cpp:141-155``).

Everything here runs in float64 unless a ``_f32`` variant is requested.
"""
import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class Geom(ctypes.Structure):
    """Mirror of ``oracle_geom`` (one planogram + the volume)."""
    _fields_ = [(n, ctypes.c_float) for n in ("psi", "R", "L", "H", "v_m0", "v_m1")] + \
               [(n, ctypes.c_int) for n in ("N_v1", "N_v0", "N_u1", "N_u0")] + \
               [(n, ctypes.c_float) for n in ("T_v1", "T_v0", "T_u1", "T_u0",
                                                "v1_0", "v0_0", "u1_0", "u0_0",
                                                "cos_psi", "sin_psi")] + \
               [(n, ctypes.c_int) for n in ("numX", "numY", "numZ")] + \
               [(n, ctypes.c_float) for n in ("voxelWidth", "voxelHeight", "x_0", "y_0", "z_0")]

    @property
    def shape(self):
        return (self.N_v1, self.N_v0, self.N_u1, self.N_u0)

    @property
    def vol_shape(self):
        return (self.numZ, self.numY, self.numX)

    def copy(self):
        g = Geom()
        ctypes.pointer(g)[0] = self
        return g


class Solid(ctypes.Structure):
    """oracle_solid (oracle.h)."""
    _fields_ = [("type", ctypes.c_int), ("centers", ctypes.c_float * 3), ("radii", ctypes.c_float * 3),
                ("val", ctypes.c_float), ("A", ctypes.c_float * 9), ("clip", (ctypes.c_float * 4) * 6),
                ("rotated", ctypes.c_int), ("num_clip", ctypes.c_int), ("clip_cone", ctypes.c_float * 2),
                ("given_c", ctypes.c_float * 3), ("given_r", ctypes.c_float * 3)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: run `make -C oracle` (or __graft_entry__.build())")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        dp, fp = P(ctypes.c_double), P(ctypes.c_float)
        gp = P(Geom)
        L.oracle_planogram_init.argtypes = [gp] + [ctypes.c_float] * 7
        L.oracle_planogram_init.restype = ctypes.c_int
        L.oracle_bin_events.argtypes = [gp, fp, fp, ctypes.c_longlong, fp, ctypes.c_int, ctypes.c_int]
        sp = ctypes.POINTER(Solid)
        L.oracle_solid_init.argtypes = [sp, ctypes.c_int, fp, fp, ctypes.c_float, fp, fp]
        L.oracle_voxelize.argtypes = [sp, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_float] * 5 + [ctypes.c_int]
        L.oracle_ray_trace.argtypes = [gp, sp, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_solid_angle_factor.argtypes = [gp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_solid_angle_factor.restype = ctypes.c_float
        L.oracle_solid_angle.argtypes = [gp, fp, ctypes.c_int]
        L.oracle_median.argtypes = [fp, ctypes.c_longlong]
        L.oracle_median.restype = ctypes.c_float
        L.oracle_apply_corrections.argtypes = [gp, fp, fp, ctypes.c_float, ctypes.c_int]
        L.oracle_set_volume.argtypes = [gp, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_float] * 5
        L.oracle_optimal_fft_size.argtypes = [ctypes.c_int]
        L.oracle_optimal_fft_size.restype = ctypes.c_int
        L.oracle_project_f64.argtypes = [gp, dp, dp, ctypes.c_int]
        L.oracle_project_f32.argtypes = [gp, fp, fp, ctypes.c_int]
        L.oracle_backproject_f64.argtypes = [gp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.oracle_project_sub_f64.argtypes = [gp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_backproject_sub_f64.argtypes = [gp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_project_band_f64.argtypes = [gp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_backproject_band_f64.argtypes = [gp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_project_band_f32.argtypes = [gp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_backproject_band_f32.argtypes = [gp, fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_backproject_f32.argtypes = [gp, fp, fp, ctypes.c_int, ctypes.c_int]
        L.oracle_project_nnz.argtypes = [gp, ctypes.c_int]
        L.oracle_project_nnz.restype = ctypes.c_double
        L.oracle_project_nnz_t.argtypes = [gp, ctypes.c_int, ctypes.c_int]
        L.oracle_project_nnz_t.restype = ctypes.c_double
        L.oracle_pfdr_f64.argtypes = [gp, dp, dp, ctypes.c_int]
        L.oracle_ramp_f64.argtypes = [gp, dp, ctypes.c_long, ctypes.c_int]
        L.oracle_fft_c2c.argtypes = [dp, ctypes.c_int, ctypes.c_int]
        L.oracle_rd_gradient_f64.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.oracle_rd_cost_f64.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double]
        L.oracle_rd_cost_f64.restype = ctypes.c_double
        L.oracle_tv_cost_f64.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.oracle_tv_cost_f64.restype = ctypes.c_double
        L.oracle_tv_gradient_f64.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_int, ctypes.c_int]
        L.oracle_tv_quadform_f64.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.oracle_tv_quadform_f64.restype = ctypes.c_double
        _LIB = L
    return _LIB


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ----------------------------------------------------------------------------
# geometry
# ----------------------------------------------------------------------------
def make_geom(psi_deg, D, L, H, T, v_m0, v_m1, vol):
    """One planogram as the C-ABI ``add_planogram(psi, D, L, H, v_m0, v_m1, T)``
    defines it, plus the volume ``vol = (numX, numY, numZ, voxelWidth,
    voxelHeight, offsetX, offsetY, offsetZ)``."""
    g = Geom()
    # src/petl_c_interface.cpp:216-219 (float arguments, double arithmetic)
    psi = np.float32(psi_deg * math.pi / 180.0)
    ok = lib().oracle_planogram_init(ctypes.byref(g), float(psi), float(np.float32(0.5 * np.float32(D))),
                                     float(np.float32(0.5 * np.float32(L))),
                                     float(np.float32(0.5 * np.float32(H))),
                                     float(np.float32(v_m0)), float(np.float32(v_m1)), float(np.float32(T)))
    if not ok:
        raise ValueError("invalid planogram")
    set_volume(g, *vol)
    return g


def set_volume(g, numX, numY, numZ, voxelWidth, voxelHeight=0.0, offsetX=0.0, offsetY=0.0, offsetZ=0.0):
    if voxelHeight == 0.0:
        voxelHeight = voxelWidth
    lib().oracle_set_volume(ctypes.byref(g), int(numX), int(numY), int(numZ), float(voxelWidth),
                            float(voxelHeight), float(offsetX), float(offsetY), float(offsetZ))
    return g


def optimal_fft_size(n):
    return lib().oracle_optimal_fft_size(int(n))


# ----------------------------------------------------------------------------
# projectors
# ----------------------------------------------------------------------------
def project(geoms, f, dtype=np.float64, nthreads=0):
    """P f for each planogram (``PETL::project``, src/petl.cpp:205-224)."""
    if isinstance(geoms, Geom):
        geoms = [geoms]
    out = []
    for G in geoms:
        if dtype == np.float32:
            fc = _f(f)
            g = np.zeros(G.shape, np.float32)
            lib().oracle_project_f32(ctypes.byref(G), _ptr(fc, ctypes.c_float), _ptr(g, ctypes.c_float), nthreads)
        else:
            fc = _d(f)
            g = np.zeros(G.shape, np.float64)
            lib().oracle_project_f64(ctypes.byref(G), _ptr(fc, ctypes.c_double), _ptr(g, ctypes.c_double), nthreads)
        out.append(g)
    return out


def backproject(geoms, g, dtype=np.float64, texmode=0, nthreads=0):
    """P^T g summed over planograms (``PETL::backproject``, src/petl.cpp:226-277)."""
    if isinstance(geoms, Geom):
        geoms, g = [geoms], [g]
    f = None
    for G, gi in zip(geoms, g):
        if dtype == np.float32:
            gc = _f(gi)
            fi = np.zeros(G.vol_shape, np.float32)
            lib().oracle_backproject_f32(ctypes.byref(G), _ptr(gc, ctypes.c_float), _ptr(fi, ctypes.c_float),
                                         int(texmode), nthreads)
        else:
            gc = _d(gi)
            fi = np.zeros(G.vol_shape, np.float64)
            lib().oracle_backproject_f64(ctypes.byref(G), _ptr(gc, ctypes.c_double), _ptr(fi, ctypes.c_double),
                                         int(texmode), nthreads)
        f = fi if f is None else f + fi
    return f


def project_band(G, f, v1_begin, v1_end, nthreads=0, dtype=np.float64):
    """The v1 slices [v1_begin, v1_end) of P f (FP64, or FP32 for timing): the
    same rays as ``project`` computes for those slices
    (src/projectors.cu:11-238)."""
    shape = (v1_end - v1_begin,) + tuple(G.shape[1:])
    if dtype == np.float32:
        fc = _f(f)
        g = np.zeros(shape, np.float32)
        lib().oracle_project_band_f32(ctypes.byref(G), _ptr(fc, ctypes.c_float), _ptr(g, ctypes.c_float),
                                      int(v1_begin), int(v1_end), nthreads)
        return g
    fc = _d(f)
    g = np.zeros(shape, np.float64)
    lib().oracle_project_band_f64(ctypes.byref(G), _ptr(fc, ctypes.c_double), _ptr(g, ctypes.c_double),
                                  int(v1_begin), int(v1_end), nthreads)
    return g


def backproject_band(G, g_band, v1_begin, v1_end, nthreads=0, dtype=np.float64):
    """Backprojection of the v1 slices [v1_begin, v1_end) only; g_band holds
    just those slices (FP64, or FP32 for timing; src/projectors.cu:240-377
    summed over the band)."""
    assert np.shape(g_band)[0] == v1_end - v1_begin
    if dtype == np.float32:
        gc = _f(g_band)
        f = np.zeros(G.vol_shape, np.float32)
        lib().oracle_backproject_band_f32(ctypes.byref(G), _ptr(gc, ctypes.c_float), _ptr(f, ctypes.c_float),
                                          int(v1_begin), int(v1_end), nthreads)
        return f
    gc = _d(g_band)
    f = np.zeros(G.vol_shape, np.float64)
    lib().oracle_backproject_band_f64(ctypes.byref(G), _ptr(gc, ctypes.c_double), _ptr(f, ctypes.c_double),
                                      int(v1_begin), int(v1_end), nthreads)
    return f


def project_nnz(G, nthreads=0, single=False):
    return lib().oracle_project_nnz_t(ctypes.byref(G), nthreads, 1 if single else 0)


# ----------------------------------------------------------------------------
# list-mode binning
# ----------------------------------------------------------------------------
def bin_events(geoms, blue, pink, linear=True, chest_wall=True):
    """Coincidences (blue[i], pink[i], xyz in mm) binned into zeroed float32
    planograms, one per geometry, in event order (src/binning.cpp:614-790)."""
    blue, pink = _f(blue).reshape(-1, 3), _f(pink).reshape(-1, 3)
    out = []
    for G in (geoms if isinstance(geoms, (list, tuple)) else [geoms]):
        g = np.zeros(G.shape, np.float32)
        lib().oracle_bin_events(ctypes.byref(G), _ptr(blue, ctypes.c_float), _ptr(pink, ctypes.c_float),
                                len(blue), _ptr(g, ctypes.c_float), 1 if linear else 0, 1 if chest_wall else 0)
        out.append(g)
    return out


# ----------------------------------------------------------------------------
# analytic phantoms
# ----------------------------------------------------------------------------
def make_solid(kind, c, r, val, A=None, clip=None):
    """geometricObject::init (src/phantom.cpp:535-640) with the Python
    defaults of PETLserver.add_object (identity A, no clipping)."""
    c = _f(np.broadcast_to(np.asarray(c, np.float32), (3,)))
    r = _f(np.broadcast_to(np.asarray(r, np.float32), (3,)))
    A = np.eye(3, dtype=np.float32) if A is None else _f(A)
    clip = np.zeros(3, np.float32) if clip is None else _f(clip)
    s = Solid()
    if not lib().oracle_solid_init(ctypes.byref(s), int(kind), _ptr(c, ctypes.c_float), _ptr(r, ctypes.c_float),
                                   float(val), _ptr(A, ctypes.c_float), _ptr(clip, ctypes.c_float)):
        raise ValueError("invalid solid")
    return s


def scale_solids(solids, sx, sy, sz):
    """phantom::scale_phantom (src/phantom.cpp:1120-1141): centres and radii
    per axis; clipping planes' y, z normals by sy, sz and offsets by sx."""
    for s in solids:
        for k, f in enumerate((sx, sy, sz)):
            s.centers[k] = np.float32(np.float32(s.centers[k]) * np.float32(f))
            s.radii[k] = np.float32(np.float32(s.radii[k]) * np.float32(f))
        for i in range(s.num_clip):
            s.clip[i][1] = np.float32(np.float32(s.clip[i][1]) * np.float32(sy))
            s.clip[i][2] = np.float32(np.float32(s.clip[i][2]) * np.float32(sz))
            s.clip[i][3] = np.float32(np.float32(s.clip[i][3]) * np.float32(sx))
    return solids


def _solids(solids):
    return (Solid * max(1, len(solids)))(*solids), len(solids)


def voxelize(solids, f, voxel_width, voxel_height, x_0, y_0, z_0, oversampling=1):
    """phantom::voxelize into a copy of f [z][y][x] (src/phantom.cpp:105-335)."""
    out = np.array(f, np.float32, copy=True, order="C")
    nz, ny, nx = out.shape
    arr, n = _solids(solids)
    lib().oracle_voxelize(arr, n, _ptr(out, ctypes.c_float), nx, ny, nz, voxel_width, voxel_height, x_0, y_0, z_0,
                          int(oversampling))
    return out


def ray_trace(G, solids, oversampling=1, stopping_power=False, nthreads=0):
    """rayTracingKernel / stoppingPowerKernel on one planogram
    (src/analytic_ray_tracing_gpu.cu:693-846)."""
    g = np.zeros(G.shape, np.float32)
    arr, n = _solids(solids)
    lib().oracle_ray_trace(ctypes.byref(G), arr, n, _ptr(g, ctypes.c_float), int(oversampling),
                           1 if stopping_power else 0, nthreads)
    return g


# ----------------------------------------------------------------------------
# corrections
# ----------------------------------------------------------------------------
def solid_angle(geoms, g, inverse=False):
    """Planograms scaled by the solid-angle correction (inverse: the model),
    src/planogram.cpp:262-302; returns new float32 arrays."""
    out = []
    for G, gi in zip(geoms if isinstance(geoms, (list, tuple)) else [geoms], g):
        a = np.array(gi, np.float32, copy=True, order="C")
        lib().oracle_solid_angle(ctypes.byref(G), _ptr(a, ctypes.c_float), 1 if inverse else 0)
        out.append(a)
    return out


def median(x):
    """src/vector_ops.cpp:358-374 on a float32 array."""
    a = _f(x).ravel()
    return float(lib().oracle_median(_ptr(a, ctypes.c_float), a.size))


def apply_corrections(geoms, g, r, threshold=0.75, nthreads=0):
    """PETL::apply_corrections: g / r then the bad-pixel median in-fill
    (src/petl.cpp:163-192, src/median_filter.cu:11-190); new float32 arrays."""
    out = []
    geoms = geoms if isinstance(geoms, (list, tuple)) else [geoms]
    for G, gi, ri in zip(geoms, g, r):
        a = np.array(gi, np.float32, copy=True, order="C")
        b = _f(ri)
        lib().oracle_apply_corrections(ctypes.byref(G), _ptr(a, ctypes.c_float), _ptr(b, ctypes.c_float),
                                       threshold, nthreads)
        out.append(a)
    return out


# ----------------------------------------------------------------------------
# PFDR / ramp / FBP
# ----------------------------------------------------------------------------
def pfdr(G, g, nthreads=0):
    gc = _d(g)
    out = np.zeros((G.N_v0, G.N_u1, G.N_u0), np.float64)
    lib().oracle_pfdr_f64(ctypes.byref(G), _ptr(gc, ctypes.c_double), _ptr(out, ctypes.c_double), nthreads)
    return out


def rebinned_geom(G):
    """Geometry after ``PETL::doPFDR`` (src/petl.cpp:379-380): N_v1 = 1, v1_0 = 0."""
    R = G.copy()
    R.N_v1 = 1
    R.v1_0 = 0.0
    return R


def ramp(G, rows, nthreads=0):
    r = np.array(rows, dtype=np.float64, copy=True, order="C")
    lib().oracle_ramp_f64(ctypes.byref(G), _ptr(r, ctypes.c_double), int(r.size // G.N_u0), nthreads)
    return r


def fbp(geoms, g, nthreads=0):
    """``PETL::doFBP`` (src/petl.cpp:310-355) for a list of planograms."""
    if isinstance(geoms, Geom):
        geoms, g = [geoms], [g]
    rebinned, rgeoms = [], []
    for G, gi in zip(geoms, g):
        if G.N_v1 > 1:
            gr = pfdr(G, gi, nthreads)
            Gr = rebinned_geom(G)
        else:
            gr = np.asarray(gi, np.float64).reshape(G.N_v0, G.N_u1, G.N_u0)
            Gr = G
        gr = ramp(Gr, gr, nthreads)
        # apply_planogram_weight(inverse) (src/planogram.cpp:304-333)
        for iv0 in range(Gr.N_v0):
            v1 = np.float32(np.float32(0) * np.float32(Gr.T_v1) + np.float32(Gr.v1_0))
            v0 = np.float32(np.float32(iv0) * np.float32(Gr.T_v0) + np.float32(Gr.v0_0))
            c = np.float32(1.0 / math.sqrt(1.0 + float(v1) * float(v1) + float(v0) * float(v0)))
            gr[iv0] *= float(np.float32(1.0) / c)
        rebinned.append(gr.reshape(1, Gr.N_v0, Gr.N_u1, Gr.N_u0))
        rgeoms.append(Gr)
    f = None
    for Gr, gr in zip(rgeoms, rebinned):
        fi = backproject(Gr, gr, nthreads=nthreads)
        # FBPweight scale (src/petl.cpp:254-259)
        fi *= float(np.float32(np.float32(Gr.T_v0) * np.float32(Gr.T_u0) / np.float32(Gr.voxelWidth)))
        f = fi if f is None else f + fi
    return f


def fft_c2c(x, sign=-1):
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().oracle_fft_c2c(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size, int(sign))
    return a


# ----------------------------------------------------------------------------
# regularizers
# ----------------------------------------------------------------------------
def _shape3(f):
    f = np.asarray(f)
    if f.ndim == 2:
        return (1,) + f.shape
    return f.shape


def gaussian_filter(f, fwhm, num_dims=3):
    """gaussian_filter (src/relative_differences.cu:314-411): for every voxel,
    the weighted mean over the (2r+1)^d window with indices clamped at the
    borders and weights exp(-(squared distance to the clamped index)/(2 sigma))
    (the reference divides by 2 sigma, not 2 sigma^2); sigma = FWHM / (2
    sqrt(2 ln 2)), r = ceil(sqrt(2 ln 10) sigma) in float.  num_dims 1 filters
    along the first axis, 2 along the last two, 3 along all three.  FP64."""
    f = np.asarray(f, np.float64)
    sigma = np.float32(fwhm) / (np.float32(2.0) * np.sqrt(np.float32(2.0) * np.log(np.float32(2.0))))
    r = int(np.ceil(np.sqrt(np.float32(2.0) * np.log(np.float32(10.0))) * sigma))
    denom = 1.0 / (2.0 * float(sigma))
    axes = {1: (0,), 2: (1, 2)}.get(num_dims, (0, 1, 2))
    n = f.shape
    grids = np.meshgrid(*[np.arange(m) for m in n], indexing="ij")
    val = np.zeros_like(f)
    wsum = np.zeros_like(f)
    import itertools
    for offs in itertools.product(range(-r, r + 1), repeat=len(axes)):
        idx = list(grids)
        dist = np.zeros_like(f)
        for a, d in zip(axes, offs):
            sh = np.clip(grids[a] + d, 0, n[a] - 1)
            idx[a] = sh
            dist += (grids[a] - sh).astype(np.float64) ** 2
        w = np.exp(-denom * dist)
        val += w * f[tuple(idx)]
        wsum += w
    return val / wsum


def rd_gradient(f, delta, beta, nthreads=0):
    N = _shape3(f)
    fc = _d(f).reshape(N)
    out = np.zeros(N, np.float64)
    lib().oracle_rd_gradient_f64(_ptr(fc, ctypes.c_double), _ptr(out, ctypes.c_double), *N,
                                 float(delta), float(beta), nthreads)
    return out.reshape(np.shape(f))


def rd_cost(f, delta, beta):
    N = _shape3(f)
    fc = _d(f).reshape(N)
    return lib().oracle_rd_cost_f64(_ptr(fc, ctypes.c_double), *N, float(delta), float(beta))


def tv_cost(f, delta, beta=0.0, p=1.0, num_neighbors=26):
    N = _shape3(f)
    fc = _d(f).reshape(N)
    return lib().oracle_tv_cost_f64(_ptr(fc, ctypes.c_double), *N, float(delta), float(beta), float(p),
                                    int(num_neighbors))


def tv_gradient(f, delta, beta=0.0, p=1.0, num_neighbors=26, nthreads=0):
    N = _shape3(f)
    fc = _d(f).reshape(N)
    out = np.zeros(N, np.float64)
    lib().oracle_tv_gradient_f64(_ptr(fc, ctypes.c_double), _ptr(out, ctypes.c_double), *N, float(delta),
                                 float(beta), float(p), int(num_neighbors), nthreads)
    return out.reshape(np.shape(f))


def tv_quadform(f, d, delta, beta=0.0, p=1.0, num_neighbors=26):
    N = _shape3(f)
    fc, dc = _d(f).reshape(N), _d(d).reshape(N)
    return lib().oracle_tv_quadform_f64(_ptr(fc, ctypes.c_double), _ptr(dc, ctypes.c_double), *N,
                                        float(delta), float(beta), float(p), int(num_neighbors))


def diffuse(f, delta, num_iter, p=1.0, num_neighbors=26):
    """``Diffuse`` (src/total_variation.cu:813-868) in float64."""
    f = _d(f).copy()
    for _ in range(num_iter):
        d = tv_gradient(f, delta, 1.0, p, num_neighbors)
        num = float(np.sum(d * d))
        den = tv_quadform(f, d, delta, 1.0, p, num_neighbors)
        if den <= 1.0e-16:
            break
        f -= (num / den) * d
    return f


def tv_denoise(f, delta, beta, num_iter, p=1.0, num_neighbors=26):
    """``TVdenoise`` (src/total_variation.cu:870-935) in float64."""
    f = _d(f).copy()
    f0 = f.copy()
    for _ in range(num_iter):
        d = tv_gradient(f, delta, beta, p, num_neighbors)
        num = float(np.sum(d * d))
        den = tv_quadform(f, d, delta, beta, p, num_neighbors)
        if den <= 1.0e-16:
            break
        s = num / den
        f = (1.0 - s) * f - s * (d - f0)
    return f


# ----------------------------------------------------------------------------
# MLEM (src/petl_server.py:1534-1606) with dataCube rules (src/data_cube.cpp)
# ----------------------------------------------------------------------------
def _rdivide(denom, num):
    out = np.zeros_like(denom)
    nz = denom != 0.0
    out[nz] = num[nz] / denom[nz]
    return out


def _divide(x, y):
    out = np.zeros_like(x)
    nz = y != 0.0
    out[nz] = x[nz] / y[nz]
    return out


def mlem(geoms, g, num_iter, f=None, delta=2.0, beta=0.0, nthreads=0, response=None):
    """PETLserver.MLEM (src/petl_server.py:1534-1606).  With a response R the
    projector includes it (src/petl_server.py:723-747, on during MLEM):
    P f -> R P f, backprojection of y -> P^T (R y), sensitivity P^T R."""
    if isinstance(geoms, Geom):
        geoms, g = [geoms], [g]
        if response is not None:
            response = [response]
    vol = geoms[0].vol_shape
    if f is None or not np.any(f):
        f = np.ones(vol, np.float64)
    else:
        f = np.maximum(_d(f), 0.0)
    R = [np.asarray(r, np.float64) for r in response] if response is not None else None
    ones = [np.ones(G.shape) for G in geoms] if R is None else R
    sens = backproject(geoms, ones, nthreads=nthreads)
    sens[sens == 0.0] = 1.0
    for _ in range(num_iter):
        Pd = project(geoms, f, nthreads=nthreads)
        if R is not None:
            Pd = [p * r for p, r in zip(Pd, R)]
        ratio = [_rdivide(p, gi) for p, gi in zip(Pd, g)]
        if R is not None:
            ratio = [q * r for q, r in zip(ratio, R)]
        d = backproject(geoms, ratio, nthreads=nthreads)
        if beta <= 0.0:
            f = f * _divide(d, sens)
        else:
            tv = rd_gradient(f, delta, beta, nthreads) + sens
            tv = np.maximum(0.1 * sens, tv)
            f = f * _divide(d, tv)
    return f


def project_sub(G, f, first, step, nthreads=0):
    """P f on the views iv0 = first + k step of one planogram (FP64)."""
    p = np.zeros(G.shape, np.float64)
    fc = _d(f)
    lib().oracle_project_sub_f64(ctypes.byref(G), _ptr(fc, ctypes.c_double), _ptr(p, ctypes.c_double), first, step,
                                 nthreads)
    return p


def backproject_sub(G, g, first, step, nthreads=0):
    """P^T g of one planogram using only the views iv0 = first + k step (FP64)."""
    gc = _d(g)
    out = np.zeros(G.vol_shape, np.float64)
    lib().oracle_backproject_sub_f64(ctypes.byref(G), _ptr(gc, ctypes.c_double), _ptr(out, ctypes.c_double), first,
                                     step, nthreads)
    return out


def osem(geoms, g, num_iter, num_subsets, f=None, nthreads=0):
    """Ordered-subsets EM with interleaved subsets over iv0 (subset s holds the
    views iv0 with iv0 % S == s).  With S = 1 it is exactly ``mlem``."""
    if isinstance(geoms, Geom):
        geoms, g = [geoms], [g]
    vol = geoms[0].vol_shape
    f = np.ones(vol, np.float64) if (f is None or not np.any(f)) else np.maximum(_d(f), 0.0)

    def proj_sub(s):
        out = []
        for G in geoms:
            p = np.zeros(G.shape, np.float64)
            fc = _d(f)
            lib().oracle_project_sub_f64(ctypes.byref(G), _ptr(fc, ctypes.c_double), _ptr(p, ctypes.c_double), s,
                                         num_subsets, nthreads)
            out.append(p)
        return out

    def back_sub(gl, s):
        acc = np.zeros(vol, np.float64)
        for G, gi in zip(geoms, gl):
            gc = _d(gi)
            fi = np.zeros(vol, np.float64)
            lib().oracle_backproject_sub_f64(ctypes.byref(G), _ptr(gc, ctypes.c_double), _ptr(fi, ctypes.c_double), s,
                                             num_subsets, nthreads)
            acc += fi
        return acc

    sens = []
    for s in range(num_subsets):
        ss = back_sub([np.ones(G.shape) for G in geoms], s)
        ss[ss == 0.0] = 1.0
        sens.append(ss)
    for _ in range(num_iter):
        for s in range(num_subsets):
            Pd = proj_sub(s)
            ratio = [_rdivide(p, gi) for p, gi in zip(Pd, g)]
            d = back_sub(ratio, s)
            f = f * _divide(d, sens[s])
    return f


def rwls(geoms, g, f, num_iter, delta=1.0, beta=0.0, W=None, sqs=False, nonnegativity=True, response=None,
         p=1.0, nthreads=0):
    """PETLserver.RWLS in FP64 (src/petl_server.py:1691-1877): PCG with a
    restart every 50 iterations, the SQS preconditioner 1 / P^T W P 1 (zeros
    -> 1), step <d, grad> / (<Pd, W Pd> + TV quadratic form); W planograms or
    None; a response R puts R in the projectors (project then multiply by R,
    multiply by R then backproject)."""
    if isinstance(geoms, Geom):
        geoms, g = [geoms], [g]
        W = [W] if W is not None else None
        response = [response] if response is not None else None
    R = [_d(r) for r in response] if response is not None else None

    def P(x):
        out = project(geoms, x, nthreads=nthreads)
        return [o * r for o, r in zip(out, R)] if R is not None else out

    def PT(ys):
        ys = [y * r for y, r in zip(ys, R)] if R is not None else ys
        return backproject(geoms, ys, nthreads=nthreads)

    def dot(a, b, w=None):
        if isinstance(a, list):
            return sum(dot(x, y, None if w is None else wi) for x, y, wi in zip(a, b, w or [None] * len(a)))
        return float(np.sum(a * b * w)) if w is not None else float(np.sum(a * b))

    g = [_d(x) for x in g]
    W = [_d(w) for w in W] if W is not None else None
    f = _d(f).copy()
    if np.any(f):
        if nonnegativity:
            f = np.maximum(f, 0.0)
        Pf = P(f)
    else:
        Pf = [np.zeros_like(x) for x in g]
    resid = [a - b for a, b in zip(Pf, g)]
    Q = None
    if sqs:
        P1 = P(np.ones_like(f))
        if W is not None:
            P1 = [a * w for a, w in zip(P1, W)]
        Q = PT(P1)
        nz = Q != 0.0
        Q[nz] = 1.0 / Q[nz]
        Q[~nz] = 1.0
    d = np.zeros_like(f)
    grad_old = np.zeros_like(f)
    gog = 0.0
    for n in range(num_iter):
        grad = PT([r * w for r, w in zip(resid, W)] if W is not None else resid)
        if beta > 0.0:
            grad = grad + tv_gradient(f, delta, beta, p).reshape(f.shape)
        u = grad * Q if Q is not None else grad.copy()
        if n % 50 == 0:
            d = u.copy()
        else:
            gamma = (dot(u, grad) - dot(u, grad_old)) / gog
            d = u + gamma * d
            if dot(d, grad) <= 0.0:
                d = u.copy()
        gog = dot(u, grad)
        grad_old = grad.copy()
        Pd = P(d)
        num = dot(d, grad)
        den = dot(Pd, Pd, W)
        if beta > 0.0:
            den += tv_quadform(f, d, delta, beta, p)
        step = num / den if abs(den) > 1.0e-16 else 0.0
        if step <= 0.0:
            break
        f = f - step * d
        if nonnegativity:
            f = np.maximum(f, 0.0)
            Pf = P(f)
            resid = [a - b for a, b in zip(Pf, g)]
        else:
            resid = [r - step * pd for r, pd in zip(resid, Pd)]
    return f


def poisson_loglik(g, Pf):
    """sum(g*log(Pf) - Pf) over bins with Pf > 0 (the MLEM objective)."""
    total = 0.0
    for gi, pi in zip(g, Pf):
        m = pi > 0
        total += float(np.sum(gi[m] * np.log(pi[m]) - pi[m]))
    return total

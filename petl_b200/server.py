"""PETLserver: the reference Python operator surface over libpetl.so.

Method names, argument meaning, defaults, return values and error behaviour
follow the reference class ``PETLserver`` (src/petl_server.py:14-2152):
geometry setters raise ValueError when the library returns false, projector
calls raise TypeError, planograms are lists of float32 numpy arrays
[N_v1][N_v0][N_u1][N_u0], volumes are float32 numpy arrays [z][y][x].
Numpy inputs go through the reference-compatible C ABI (host pointers);
torch CUDA tensors (or lists of them) go through the device-resident
operators in petl_b200.ops without leaving the GPU.

Not provided here: scatter simulation (the reference's computes nothing
either) and the napari display.
"""
import ctypes
import os

import numpy as np

from ._lib import c_f, fp, lib

try:  # torch is optional for the host path
    import torch
    _has_torch = True
except Exception:  # pragma: no cover
    torch = None
    _has_torch = False


def _is_dev(x):
    if isinstance(x, list):
        return len(x) > 0 and _is_dev(x[0])
    return _has_torch and isinstance(x, torch.Tensor) and x.is_cuda


def _fp(a):
    return a.ctypes.data_as(fp)


def _pp(arrs):
    return (fp * len(arrs))(*[_fp(a) for a in arrs])


def _to_device(a, device="cuda"):
    """A float32 CUDA tensor with the contents of the host array a (or a
    itself when it already is one), copied through the library's staged
    host copies."""
    if _is_dev(a):
        return a
    a = np.ascontiguousarray(a, np.float32)
    t = torch.empty(a.shape, dtype=torch.float32, device=device)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if a.nbytes and lib().petl_copy_to_device(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(a.ctypes.data),
                                              a.nbytes, st) != 0:
        raise TypeError("copy to the device failed")
    return t


def _to_host_(out, t):
    """Copies the CUDA tensor t into the host array out (float32, C order)."""
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    if out.nbytes and lib().petl_copy_to_host(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(t.data_ptr()),
                                              out.nbytes, st) != 0:
        raise TypeError("copy to the host failed")
    return out


def _copy_back(f, fd):
    """The device result fd into the caller's host array f."""
    if isinstance(f, np.ndarray) and f.dtype == np.float32 and f.flags["C_CONTIGUOUS"]:
        _to_host_(f, fd.contiguous())
    else:
        f[...] = fd.cpu().numpy()


def _check_f32(a, name):
    if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]):
        raise TypeError(f"{name} must be a C-contiguous float32 numpy array")


class PETLserver:
    def __init__(self, param_id=None, lib_dir=""):
        self.libprojectors = lib()
        if param_id is not None:
            self.param_id = param_id
        else:
            self.param_id = self.libprojectors.create_new_model()
        self.set_model()
        self.print_cost = False
        self.print_warnings = True
        self.response = None
        self.include_response_with_projectors = False

    # ------------------------------------------------------------------ model
    def set_model(self, i=None):
        if i is not None:
            self.param_id = i
        return self.libprojectors.set_model(self.param_id)

    def create_new_model(self):
        return self.libprojectors.create_new_model()

    def about(self):
        self.set_model()
        self.libprojectors.about()

    def copy_parameters(self, param_id):
        self.set_model()
        return self.libprojectors.copy_parameters(param_id)

    def clearAll(self):
        self.set_model()
        self.libprojectors.clearAll()

    def print_parameters(self):
        self.set_model()
        self.libprojectors.print_parameters()

    def all_defined(self):
        return self.geometry_defined() and self.volume_defined()

    def volume_defined(self):
        self.set_model()
        return self.libprojectors.volume_defined()

    def geometry_defined(self):
        self.set_model()
        return self.libprojectors.geometry_defined()

    def _getset(self, name, v, setter_type=None):
        self.set_model()
        if v is None:
            return getattr(self.libprojectors, "get_" + name)()
        if getattr(self.libprojectors, "set_" + name)(v):
            return getattr(self.libprojectors, "get_" + name)()
        return None

    def numX(self, N=None):
        return self._getset("numX", N)

    def numY(self, N=None):
        return self._getset("numY", N)

    def numZ(self, N=None):
        return self._getset("numZ", N)

    def voxelWidth(self, w=None):
        return self._getset("voxelWidth", w)

    def voxelHeight(self, h=None):
        return self._getset("voxelHeight", h)

    def offsetX(self, x=None):
        return self._getset("offsetX", x)

    def offsetY(self, y=None):
        return self._getset("offsetY", y)

    def offsetZ(self, z=None):
        return self._getset("offsetZ", z)

    def get_numPlanograms(self):
        self.set_model()
        return self.libprojectors.get_numPlanograms()

    def get_planogramSize(self, n):
        if self.geometry_defined():
            shape = (ctypes.c_int * 4)()
            self.set_model()
            self.libprojectors.get_planogramSize(n, shape)
            return np.array(list(shape), dtype=np.int32)
        return None

    # -------------------------------------------------------------- geometry
    def add_planogram(self, psi, D, L, H, T, v_m0=None, v_m1=None):
        if v_m0 is None:
            v_m0 = 1.0
        if v_m1 is None:
            v_m1 = min(1.0, (H - 1.5 * T) / D)
        self.set_model()
        if not self.libprojectors.add_planogram(psi, D, L, H, v_m0, v_m1, T):
            raise ValueError("Error: add_planogram failed")

    def remove_planogram(self, n):
        self.set_model()
        if not self.libprojectors.remove_planogram(n):
            raise ValueError("Error: remove_planogram failed")

    def keep_only_planogram(self, n):
        self.set_model()
        if not self.libprojectors.keep_only_planogram(n):
            raise ValueError("Error: keep_only_planogram failed")

    def set_default_volume(self, scale=1.0):
        self.set_model()
        if not self.libprojectors.set_default_volume(scale):
            raise ValueError("Error: set_default_volume failed")

    def set_volume(self, numX, numY, numZ, voxelWidth, voxelHeight=0.0, offsetX=0.0, offsetY=0.0, offsetZ=0.0):
        if voxelHeight == 0.0:
            voxelHeight = voxelWidth
        self.set_model()
        if not self.libprojectors.set_volume(numX, numY, numZ, voxelWidth, voxelHeight, offsetX, offsetY, offsetZ):
            raise ValueError("Error: set_volume failed")

    # ----------------------------------------------------------- allocation
    def allocate_projections(self):
        if self.geometry_defined():
            return [np.zeros(tuple(self.get_planogramSize(n)), dtype=np.float32)
                    for n in range(self.get_numPlanograms())]
        return None

    def allocate_rebinned_projections(self):
        if self.geometry_defined():
            return [np.zeros(tuple(self.get_planogramSize(n))[1:], dtype=np.float32)
                    for n in range(self.get_numPlanograms())]
        return None

    def allocate_volume(self):
        if self.volume_defined():
            return np.zeros((self.numZ(), self.numY(), self.numX()), dtype=np.float32)
        print("Error: volume is not defined")
        return None

    def copy_data(self, x):
        if isinstance(x, list):
            return [y.clone() if _is_dev(y) else y.copy() for y in x]
        return x.clone() if _is_dev(x) else x.copy()

    def copyData(self, x):
        return self.copy_data(x)

    # ------------------------------------------------------------ projectors
    def project(self, g, f):
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        self.set_model()
        for a in g:
            _check_f32(a, "g")
        _check_f32(f, "f")
        if not self.libprojectors.project(_pp(g), _fp(f)):
            raise TypeError("project failed")
        if self.response is not None and self.include_response_with_projectors:
            self.multiply(g, self.response)
        return g

    def bin(self, file_name, g=None):
        """Bins a list-mode coincidence file (src/petl_server.py:653-678): the
        planograms are overwritten with the binned data, as the reference's
        C++ does (its docstring's "adds to the data" does not hold there)."""
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        if g is None:
            g = self.allocate_projections()
        self.set_model()
        for a in g:
            _check_f32(a, "g")
        if not self.libprojectors.bin(_pp(g), bytes(str(file_name), "ascii")):
            raise TypeError("bin failed")
        return g

    def backproject(self, g, f=None):
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        if f is None:
            f = self.allocate_volume()
        self.set_model()
        for a in g:
            _check_f32(a, "g")
        _check_f32(f, "f")
        if self.response is not None and self.include_response_with_projectors:
            g = self.multiply(self.copy_data(g), self.response)
        if not self.libprojectors.backproject(_pp(g), _fp(f)):
            raise TypeError("backproject failed")
        return f

    def FBP(self, g, f=None):
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        if f is None:
            f = self.allocate_volume()
        self.set_model()
        if not self.libprojectors.FBP(_pp(g), _fp(f)):
            raise TypeError("FBP failed")
        return f

    def PFDR(self, g, g_reb=None):
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        if g_reb is None:
            g_reb = self.allocate_rebinned_projections()
        self.set_model()
        if not self.libprojectors.PFDR(_pp(g), _pp(g_reb)):
            raise TypeError("PFDR failed")
        return g_reb

    def sensitivity(self, Pstar1=None):
        if Pstar1 is None:
            Pstar1 = self.allocate_volume()
        ones = self.allocate_projections()
        for o in ones:
            o[:] = 1.0
        self.backproject(ones, Pstar1)
        return Pstar1

    # ----------------------------------------------- phantoms and modules
    def add_object(self, typeOfObject, c, r, val, A=None, clip=None):
        """Appends an analytic solid to the phantom (src/petl_server.py:813-875):
        type 0..7 or a name (ball/sphere/ellipsoid, box/parallelepiped,
        can_x, can_y, can_z/can, cone_x, cone_y, cone_z/cone)."""
        from .ops import SOLID_TYPES
        if A is None:
            A = np.eye(3, dtype=np.float32)
        if clip is None:
            clip = np.zeros(3, dtype=np.float32)
        if isinstance(c, (int, float)):
            c = [c, c, c]
        if isinstance(r, (int, float)):
            r = [r, r, r]
        if isinstance(typeOfObject, str):
            if typeOfObject.lower() not in SOLID_TYPES:
                print("Error: unknown object type")
                return False
            typeOfObject = SOLID_TYPES[typeOfObject.lower()]
        c, r = np.ascontiguousarray(c, np.float32), np.ascontiguousarray(r, np.float32)
        A, clip = np.ascontiguousarray(A, np.float32), np.ascontiguousarray(clip, np.float32)
        self.set_model()
        return self.libprojectors.add_object(int(typeOfObject), _fp(c), _fp(r), float(val), _fp(A), _fp(clip))

    def add_module(self, c, r, val=0.0815, A=None):
        """Appends a detector module (a parallelepiped of attenuation val,
        mm^-1) to the stopping-power model (src/petl_server.py:877-910)."""
        if A is None:
            A = np.eye(3, dtype=np.float32)
        if isinstance(c, (int, float)):
            c = [c, c, c]
        if isinstance(r, (int, float)):
            r = [r, r, r]
        c, r = np.ascontiguousarray(c, np.float32), np.ascontiguousarray(r, np.float32)
        A, clip = np.ascontiguousarray(A, np.float32), np.zeros(3, np.float32)
        self.set_model()
        return self.libprojectors.add_module(1, _fp(c), _fp(r), float(val), _fp(A), _fp(clip))

    def clear_phantom(self):
        self.set_model()
        self.libprojectors.clear_phantom()

    def clear_modules(self):
        self.set_model()
        self.libprojectors.clear_modules()

    def scale_phantom(self, c):
        if isinstance(c, (int, float)):
            cx = cy = cz = c
        elif isinstance(c, np.ndarray) and c.size == 3:
            cx, cy, cz = (float(v) for v in c)
        else:
            return False
        self.set_model()
        return self.libprojectors.scale_phantom(cx, cy, cz)

    def voxelize(self, f=None, oversampling=1):
        """Writes the phantom's solids into f (src/petl_server.py:946-965)."""
        if not self.volume_defined():
            raise ValueError("Error: volume parameters not specified")
        if f is None:
            f = self.allocate_volume()
        _check_f32(f, "f")
        self.set_model()
        return f if self.libprojectors.voxelize(_fp(f), int(oversampling)) else None

    def ray_trace(self, g=None, oversampling=1):
        """Analytic line integrals of the phantom (src/petl_server.py:967-993)."""
        if not self.geometry_defined():
            raise ValueError("Error: PET scanner not specified")
        if g is None:
            g = self.allocate_projections()
        for a in g:
            _check_f32(a, "g")
        self.set_model()
        return g if self.libprojectors.ray_trace(_pp(g), int(oversampling)) else None

    def stopping_power(self, g=None, oversampling=1):
        """Detector stopping power of every coincidence line through the
        module model, smoothed by a 0.6571-bin Gaussian as the reference does
        (src/petl_server.py:995-1022)."""
        if not self.geometry_defined():
            raise ValueError("Error: PET scanner not specified")
        if g is None:
            g = self.allocate_projections()
        for a in g:
            _check_f32(a, "g")
        self.set_model()
        if self.libprojectors.stopping_power(_pp(g), int(oversampling)):
            self.gaussian_filter(g, 0.6571)
            return g
        return None

    # ------------------------------------------------------ response / corrections
    def set_response(self, R):
        """Sets the response map (src/petl_server.py:121-135); with
        include_response_with_projectors it multiplies the data after project
        and before backproject, and MLEM/OSEM always include it."""
        self.response = R

    def clear_response(self):
        self.response = None

    def calc_response(self, oversampling=1, mu=None):
        """Response = detector stopping power (oversampling > 0) times the
        solid-angle model, divided by exp(P mu) when mu is given
        (src/petl_server.py:578-605)."""
        if oversampling > 0:
            self.response = self._device_response(oversampling)
        else:
            self.response = self.apply_solid_angle_model(None)
        if mu is not None:
            Pmu = self.allocate_projections()
            self.project(Pmu, mu)
            for a in Pmu:
                np.exp(a, out=a)
            self.divide(self.response, Pmu)
        return self.response

    def _device_response(self, oversampling):
        """The stopping power of the module model (1 without modules), the
        0.6571-bin Gaussian and the solid-angle model, composed on the GPU
        with the same kernels as the host-array calls and copied back once."""
        from . import ops
        from ._lib import petl_solid
        self.set_model()
        geoms = self.geometries_from_model()
        n = lib().petl_model_solids(1, None, 0)
        if n > 0:
            arr = (petl_solid * n)()
            lib().petl_model_solids(1, arr, n)
            R = ops.ray_trace(geoms, list(arr), oversampling=oversampling, stopping_power=True)
        else:
            R = [torch.ones(G.shape, device="cuda", dtype=torch.float32) for G in geoms]
        for r in R:
            ops.gaussian_filter_(r.view(r.shape[0] * r.shape[1], r.shape[2], r.shape[3]), 0.6571, 2)
        ops.solid_angle_(geoms, R, inverse=True)
        out = []
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for r in R:
            h = np.empty(tuple(r.shape), np.float32)
            if lib().petl_copy_to_host(ctypes.c_void_p(h.ctypes.data), ctypes.c_void_p(r.data_ptr()), h.nbytes,
                                       st) != 0:
                raise TypeError("calc_response: copy to the host failed")
            out.append(h)
        return out

    def apply_corrections(self, g, oversampling=1, mu=None):
        """g = g / response with the bad-pixel median in-fill (threshold 0.75
        of each projection's median response), computing the response first
        if none is set (src/petl_server.py:607-639).  Device tensors stay on
        the GPU."""
        if self.response is None:
            self.calc_response(oversampling, mu)
        if self.response is None:
            return g
        if _is_dev(g):
            from . import ops
            R = self.response if _is_dev(self.response) else \
                [_to_device(r, g[0].device) for r in self.response]
            ops.apply_corrections_(self.geometries_from_model(), g, R, 0.75)
            return g
        self.set_model()
        for a, r in zip(g, self.response):
            _check_f32(a, "g")
            _check_f32(r, "response")
        if self.libprojectors.apply_corrections(_pp(g), _pp(self.response), 0.75):
            return g
        return None

    def apply_solid_angle_correction(self, g=None, do_inverse=False):
        """Scales every projection by its solid-angle correction, or its
        inverse (src/petl_server.py:1024-1043); g defaults to ones."""
        if g is None:
            g = self.allocate_projections()
            self.setToOne(g)
        self.set_model()
        if _is_dev(g):
            from . import ops
            ops.solid_angle_(self.geometries_from_model(), g, do_inverse)
            return g
        for a in g:
            _check_f32(a, "g")
        if self.libprojectors.set_solid_angle_correction(_pp(g), bool(do_inverse)):
            return g
        return None

    def apply_solid_angle_model(self, g=None):
        return self.apply_solid_angle_correction(g, True)

    # ------------------------------------------------------- vector helpers
    def _binop4(self, name3, name4, x, y):
        self.set_model()
        xs = x if isinstance(x, list) else [x]
        ys = y if isinstance(y, list) else [y]
        for a, b in zip(xs, ys):
            if a.ndim == 4:
                ok = getattr(self.libprojectors, name4)(_fp(a), _fp(b), *a.shape)
            elif a.ndim == 3:
                ok = getattr(self.libprojectors, name3)(_fp(a), _fp(b), *a.shape)
            else:
                raise ValueError("inputs must be 3D or 4D numpy arrays")
            if not ok:
                return None
        return x

    def multiply(self, x, y):
        return self._binop4("multiply3D", "multiply4D", x, y)

    def divide(self, num, denom):
        return self._binop4("divide3D", "divide4D", num, denom)

    def rdivide(self, denom, num):
        """denom = num / denom (0 where denom == 0)."""
        self.set_model()
        ds = denom if isinstance(denom, list) else [denom]
        ns = num if isinstance(num, list) else [num]
        for d, n in zip(ds, ns):
            if d.ndim == 4:
                ok = self.libprojectors.rdivide4D(_fp(n), _fp(d), *d.shape)
            else:
                ok = self.libprojectors.rdivide3D(_fp(n), _fp(d), *d.shape)
            if not ok:
                return None
        return denom

    def reciprocal(self, x, divide_by_zero_value=0.0):
        self.set_model()
        xs = x if isinstance(x, list) else [x]
        for a in xs:
            if a.ndim == 4:
                self.libprojectors.reciprocal4D(_fp(a), *a.shape, divide_by_zero_value)
            else:
                self.libprojectors.reciprocal3D(_fp(a), *a.shape, divide_by_zero_value)
        return x

    def inner_product(self, x, y, w=None):
        if isinstance(x, list):
            acc = 0.0
            for n in range(len(x)):
                if w is None:
                    acc += self.inner_product(x[n], y[n])
                elif isinstance(w, (int, float)):
                    acc += self.inner_product(x[n], y[n]) * w
                else:
                    acc += self.inner_product(x[n], y[n], w[n])
            return acc
        self.set_model()
        wp = _fp(w) if w is not None else None
        if x.ndim == 4:
            return self.libprojectors.inner_product4D(_fp(x), _fp(y), wp, *x.shape)
        if x.ndim == 3:
            return self.libprojectors.inner_product3D(_fp(x), _fp(y), wp, *x.shape)
        return float(np.sum(x * y * w))

    def innerProd(self, x, y, w=None):
        return self.inner_product(x, y, w)

    def isAllZeros(self, f):
        return not np.any(f)

    def setToConstant(self, x, c=0.0):
        for a in (x if isinstance(x, list) else [x]):
            a[:] = c

    def setToZero(self, x):
        self.setToConstant(x, 0.0)

    def setToOne(self, x):
        self.setToConstant(x, 1.0)

    def clip(self, x, min_val=0.0, max_val=None):
        for a in (x if isinstance(x, list) else [x]):
            np.clip(a, min_val, max_val, out=a)
        return x

    def scale(self, x, c=1.0):
        for a in (x if isinstance(x, list) else [x]):
            a[:] *= c
        return x

    def subtract(self, x, y):
        for a, b in zip(x if isinstance(x, list) else [x], y if isinstance(y, list) else [y]):
            a[:] -= b[:]
        return x

    def scalarAdd(self, x, c, y):
        for a, b in zip(x if isinstance(x, list) else [x], y if isinstance(y, list) else [y]):
            a[:] += c * b[:]
        return x

    def square(self, x):
        return self.multiply(x, x)

    # --------------------------------------------------------- iterations
    def MLEM(self, g, f, numIter, delta=2.0, beta=0.0, mask=None):
        """MLEM / one-step-late RD MLEM (src/petl_server.py:1534-1606).

        Runs device-resident: the planograms are copied to the GPU once, every
        iteration stays there, and f is copied back at the end."""
        return self.OSEM(g, f, numIter, 1, delta=delta, beta=beta, mask=mask)

    def OSEM(self, g, f, numIter, numSubsets, delta=2.0, beta=0.0, mask=None):
        """Ordered-subsets EM with interleaved view subsets (iv0 mod S)."""
        from . import recon
        if mask is not None:
            raise ValueError("mask is not supported by the device-resident MLEM")
        geoms = self.geometries_from_model()
        dev = torch.device("cuda")
        gd = [_to_device(x, dev) for x in g]
        if f is None:
            f = self.allocate_volume()
        fd = _to_device(f, dev)
        R = None
        if self.response is not None:  # MLEM always includes a set response
            R = [_to_device(r, dev) for r in self.response]
        fd, _ = recon.osem(geoms, gd, numIter, numSubsets, f=fd, delta=delta, beta=beta, response=R)
        _copy_back(f, fd)
        return f

    def LS(self, g, f, numIter, preconditioner=None, nonnegativityConstraint=True):
        """Least squares by PCG (src/petl_server.py:1608-1634)."""
        return self.RWLS(g, f, numIter, 1.0, 0.0, 1.0, preconditioner, nonnegativityConstraint)

    def WLS(self, g, f, numIter, W=None, preconditioner=None, nonnegativityConstraint=True):
        """Weighted least squares by PCG (src/petl_server.py:1636-1662)."""
        return self.RWLS(g, f, numIter, 1.0, 0.0, W, preconditioner, nonnegativityConstraint)

    def RLS(self, g, f, numIter, delta=1.0, beta=0.0, preconditioner=None, nonnegativityConstraint=True):
        """Regularized (Huber-TV) least squares by PCG (src/petl_server.py:
        1664-1689)."""
        return self.RWLS(g, f, numIter, delta, beta, 1.0, preconditioner, nonnegativityConstraint)

    def RWLS(self, g, f, numIter, delta=1.0, beta=0.0, W=None, preconditioner=None, nonnegativityConstraint=True,
             include_response_with_projectors=False):
        """Regularized weighted least squares by preconditioned conjugate
        gradient (src/petl_server.py:1691-1845), device-resident.  W None:
        1 / max(gaussian(g, 3), 7), times the response squared when a
        response is set and not in the projectors; a number: no weights; else
        planograms.  preconditioner True or 'SQS': 1 / P^T W P 1.  With a set
        response: in the projectors (include_response_with_projectors), or
        else g is corrected in place first and multiplied by the response at
        the end, as the reference does."""
        from . import recon
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        dev = torch.device("cuda")
        to_dev = lambda a: _to_device(a, dev)  # noqa: E731
        R = [to_dev(r) for r in self.response] if self.response is not None else None
        if W is None:
            Wd = recon.auto_weights([to_dev(x) for x in g])
            if R is not None and not include_response_with_projectors:
                Wd = [w * r * r for w, r in zip(Wd, R)]
        elif isinstance(W, list):
            Wd = [to_dev(w) for w in W]
        else:
            Wd = None
        corrected = R is not None and not include_response_with_projectors
        if corrected:
            self.apply_corrections(g)
        gd = [to_dev(x) for x in g]
        if f is None:
            f = self.allocate_volume()
        fd = to_dev(f)
        pre = "SQS" if preconditioner in (True, "SQS") else None
        fd = recon.rwls(self.geometries_from_model(), gd, fd, numIter, delta=delta, beta=beta, W=Wd,
                        preconditioner=pre, nonnegativity=nonnegativityConstraint,
                        response=R if include_response_with_projectors else None)
        if corrected:
            self.multiply(g, self.response)
        if not _is_dev(f):
            _copy_back(f, fd)
        return f

    def RWLSstepSize(self, f, grad, d, Pd, W, delta, beta, num=None):
        """<d, grad> / (<Pd, W Pd> + TV quadratic form), 0 if the denominator
        vanishes (src/petl_server.py:1847-1877)."""
        if num is None:
            num = self.innerProd(d, grad)
        denom = self.innerProd(Pd, Pd, W) if W is not None else self.innerProd(Pd, Pd)
        if beta > 0.0:
            denom += self.TVquadForm(f, d, delta, beta)
        return num / denom if np.abs(denom) > 1.0e-16 else 0.0

    def simulate_scatter(self, g, mu):
        """As the reference's: validates the model and returns g unchanged
        (src/petl_server.py:679-701)."""
        if not self.all_defined():
            raise ValueError("Error: volume and PET geometry must be defined")
        if g is None:
            g = self.allocate_projections()
        self.set_model()
        if not self.libprojectors.simulate_scatter(_pp(g), _fp(mu)):
            raise TypeError("simulate_scatter failed")
        return g

    # ------------------------------------------------ helpers of the reference
    def floatstarstar(self, g):
        """float** of a list of float32 arrays (src/petl_server.py:641-651)."""
        return _pp(g)

    def as_float_ptr(self, arr):
        if arr is None:
            return None
        arr = np.asarray(arr, dtype=np.float32, order="C")
        return arr.ctypes.data_as(fp)

    def inner_product_helper(self, x, y, w=None):
        return self.inner_product(x, y, w)

    def display(self, x):
        """Shows 3D data with napari when it is installed
        (src/petl_server.py:1118-1134)."""
        try:
            import napari
            napari.view_image(np.squeeze(x) if min(x.shape) == 1 else x, rgb=False)
            napari.run()
        except Exception:
            print("Cannot load napari, to install run this command:")
            print("pip install napari[all]")

    def geometries_from_model(self):
        """Geometry objects equal to this model's planograms and volume."""
        from .geometry import Geometry
        from ._lib import petl_geom
        self.set_model()
        out = []
        for n in range(self.get_numPlanograms()):
            G = Geometry.__new__(Geometry)
            G.args = None
            G.volume_args = None
            G.g = petl_geom()
            if lib().petl_model_geometry(n, ctypes.byref(G.g)) != 0:
                raise ValueError("model geometry unavailable")
            out.append(G)
        return out

    # ------------------------------------------------------- regularizers
    @staticmethod
    def _dims(f):
        if f.ndim == 3:
            return f.shape
        return (1,) + tuple(f.shape)

    def TVcost(self, f, delta, beta=0.0, p=1.0):
        self.set_model()
        if _is_dev(f):
            return self.libprojectors.TV_cost(ctypes.c_void_p(f.data_ptr()), *self._dims(f), delta, beta, p, False)
        return self.libprojectors.TV_cost(f.ctypes.data_as(ctypes.c_void_p), *self._dims(f), delta, beta, p, True)

    def TVgradient(self, f, delta, beta=0.0, p=1.0):
        self.set_model()
        if _is_dev(f):
            Df = f.clone()
            self.libprojectors.TV_gradient(ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(Df.data_ptr()),
                                           *self._dims(f), delta, beta, p, False)
            return Df
        Df = np.zeros(f.shape, dtype=np.float32)
        self.libprojectors.TV_gradient(f.ctypes.data_as(ctypes.c_void_p), Df.ctypes.data_as(ctypes.c_void_p),
                                       *self._dims(f), delta, beta, p, True)
        return Df

    def TVquadForm(self, f, d, delta, beta=0.0, p=1.0):
        self.set_model()
        if _is_dev(f):
            return self.libprojectors.TV_quadForm(ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                                  *self._dims(f), delta, beta, p, False)
        return self.libprojectors.TV_quadForm(f.ctypes.data_as(ctypes.c_void_p), d.ctypes.data_as(ctypes.c_void_p),
                                              *self._dims(f), delta, beta, p, True)

    def diffuse(self, f, delta, numIter, p=1.0):
        self.set_model()
        if _is_dev(f):
            self.libprojectors.diffuse(ctypes.c_void_p(f.data_ptr()), *self._dims(f), delta, p, numIter, False)
        else:
            self.libprojectors.diffuse(f.ctypes.data_as(ctypes.c_void_p), *self._dims(f), delta, p, numIter, True)
        return f

    def TV_denoise(self, f, delta, beta, numIter, p=1.0, meanOverFirstDim=False):
        self.set_model()
        if _is_dev(f):
            self.libprojectors.TV_denoise(ctypes.c_void_p(f.data_ptr()), *self._dims(f), delta, beta, p, numIter,
                                          meanOverFirstDim, False)
        else:
            self.libprojectors.TV_denoise(f.ctypes.data_as(ctypes.c_void_p), *self._dims(f), delta, beta, p, numIter,
                                          meanOverFirstDim, True)
        return f

    def relative_differences_grad(self, f, delta, beta):
        Df = np.zeros(f.shape, dtype=np.float32)
        self.set_model()
        self.libprojectors.relativeDifferences_gradient(_fp(f), _fp(Df), *self._dims(f), delta, beta)
        return Df

    def gaussian_filter(self, f, FWHM=2.0, numDims=3):
        if isinstance(f, list):
            for x in f:
                self.gaussian_filter(x, FWHM, numDims)
            return
        if f.ndim == 4:
            dims = (f.shape[0] * f.shape[1], f.shape[2], f.shape[3])
            numDims = 2
        else:
            dims = self._dims(f)
        self.set_model()
        self.libprojectors.gaussian_filter(_fp(f), *dims, FWHM, numDims)

    # ------------------------------------------------------------- I/O
    def save_data(self, fileName, x, T=1.0, offset_0=0.0, offset_1=0.0, offset_2=0.0, sequence_offset=0):
        if fileName.endswith(".npy"):
            np.save(fileName, x)
            return True
        print("Error: only .npy output is supported by this build")
        return False

    def load_data(self, fileName, x=None, fileRange=None, rowRange=None, colRange=None):
        if not os.path.isfile(fileName) or not fileName.endswith(".npy"):
            print("Error: only .npy input is supported by this build")
            return None
        y = np.load(fileName)
        if x is not None:
            x[:] = y[:]
            return x
        return y


def petx_modules(use_simple_geometry=False):
    """The PET/X crystal blocks as (centre, half sizes) in mm
    (src/petx_server.py:13-42): 8 x 5 blocks on each psi-0 panel and 4 x 5 on
    each psi-90 panel, 30.32 mm blocks with 1.28 mm gaps, 20 mm deep; or four
    slabs (use_simple_geometry)."""
    if use_simple_geometry:
        return [([0.0, 0.5 * 101.0 + 10.0, 0.0], [0.5 * 251.52, 10.0, 0.5 * 156.72]),
                ([0.0, -0.5 * 101.0 - 10.0, 0.0], [0.5 * 251.52, 10.0, 0.5 * 156.72]),
                ([0.5 * 251.52 + 10.0, 0.0, 0.0], [10.0, 0.5 * 101.0 + 20.0, 0.5 * 156.72]),
                ([-0.5 * 251.52 - 10.0, 0.0, 0.0], [10.0, 0.5 * 101.0 + 20.0, 0.5 * 156.72])]
    block, gap, depth = 30.32, 1.28, 20.0
    out = []
    c_y = 101.0 * 0.5
    for m in range(5):
        c_z = (m - 2) * (block + gap)
        for n in range(8):
            c_x = (n - 3.5) * (block + gap)
            half = [0.5 * block, 0.5 * depth, 0.5 * block]
            out.append(([c_x, c_y + 0.5 * depth, c_z], half))
            out.append(([c_x, -c_y - 0.5 * depth, c_z], half))
    c_x = 266.6 * 0.5
    for m in range(5):
        c_z = (m - 2) * (block + gap)
        for n in range(4):
            c_y = (n - 1.5) * (block + gap)
            half = [0.5 * depth, 0.5 * block, 0.5 * block]
            out.append(([c_x + 0.5 * depth, c_y, c_z], half))
            out.append(([-c_x - 0.5 * depth, c_y, c_z], half))
    return out


class PETXserver(PETLserver):
    """The PET/X scanner preset (src/petx_server.py:4-42): two planograms
    (psi 0 and 90 degrees, 1.6 mm pixels), the default volume, and the
    crystal-block module model (petx_modules) for the stopping power."""

    def __init__(self, param_id=None, lib_dir="", use_simple_geometry=False):
        super().__init__(param_id, lib_dir)
        pitch = 1.6
        self.add_planogram(psi=0.0, D=101.0, L=251.52, H=156.72, T=pitch)
        self.add_planogram(psi=90.0, D=266.6, L=125.12, H=156.72, T=pitch)
        self.set_default_volume()
        for c, r in petx_modules(use_simple_geometry):
            self.add_module(c, r)

"""Planogram + volume geometry objects for the device-resident API.

``Geometry`` wraps one ``petl_geom`` (one planogram together with the volume
it projects to).  Its constructor takes the arguments of the reference
``PETLserver.add_planogram`` (src/petl_server.py:484-507: psi in degrees,
panel separation D, full panel length L and height H, bin pitch T, maximum
slopes v_m0 / v_m1 with the same defaults) and ``set_volume``
(src/petl_server.py:534-557, voxelHeight 0 meaning voxelWidth).  The
planogram arithmetic itself runs in the library (petl_geom_init), which
restates src/planogram.cpp:143-186.
"""
import ctypes

from ._lib import check, lib, petl_geom


class Geometry:
    def __init__(self, psi, D, L, H, T, v_m0=None, v_m1=None, volume=None):
        if v_m0 is None:
            v_m0 = 1.0
        if v_m1 is None:
            v_m1 = min(1.0, (H - 1.5 * T) / D)
        self.args = (float(psi), float(D), float(L), float(H), float(T), float(v_m0), float(v_m1))
        self.g = petl_geom()
        if lib().petl_geom_init(ctypes.byref(self.g), float(psi), float(D), float(L), float(H), float(v_m0),
                                float(v_m1), float(T)) != 0:
            raise ValueError("add_planogram failed: " + lib().petl_last_error().decode())
        self.volume_args = None
        if volume is not None:
            self.set_volume(*volume)

    # ------------------------------------------------------------------
    def set_volume(self, numX, numY, numZ, voxelWidth, voxelHeight=0.0, offsetX=0.0, offsetY=0.0, offsetZ=0.0):
        if voxelHeight == 0.0:
            voxelHeight = voxelWidth
        check(lib().petl_geom_set_volume(ctypes.byref(self.g), int(numX), int(numY), int(numZ), float(voxelWidth),
                                         float(voxelHeight), float(offsetX), float(offsetY), float(offsetZ)),
              "set_volume")
        self.volume_args = (int(numX), int(numY), int(numZ), float(voxelWidth), float(voxelHeight), float(offsetX),
                            float(offsetY), float(offsetZ))
        return self

    def copy(self):
        other = Geometry.__new__(Geometry)
        other.args = self.args
        other.volume_args = self.volume_args
        other.g = petl_geom()
        ctypes.pointer(other.g)[0] = self.g
        return other

    def rebinned(self):
        """The geometry after PFDR (src/petl.cpp:379-380): N_v1 = 1, v1_0 = 0."""
        r = self.copy()
        r.g.N_v1 = 1
        r.g.v1_0 = 0.0
        return r

    # ------------------------------------------------------------------
    @property
    def shape(self):
        """Planogram shape (N_v1, N_v0, N_u1, N_u0)."""
        return (self.g.N_v1, self.g.N_v0, self.g.N_u1, self.g.N_u0)

    @property
    def rebinned_shape(self):
        return (self.g.N_v0, self.g.N_u1, self.g.N_u0)

    @property
    def vol_shape(self):
        """Volume shape (numZ, numY, numX)."""
        return (self.g.numZ, self.g.numY, self.g.numX)

    @property
    def n_rays(self):
        s = self.shape
        return s[0] * s[1] * s[2] * s[3]

    @property
    def n_voxels(self):
        v = self.vol_shape
        return v[0] * v[1] * v[2]

    @property
    def ptr(self):
        return ctypes.byref(self.g)

    def __repr__(self):
        return f"Geometry(psi={self.args[0]}, shape={self.shape}, volume={self.vol_shape})"


def as_list(geoms):
    return list(geoms) if isinstance(geoms, (list, tuple)) else [geoms]

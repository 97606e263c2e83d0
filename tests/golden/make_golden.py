"""Generate golden vectors from the reference PETL library itself.

The reference library is compiled from its own sources by ``make -C oracle
ref`` into ``oracle/_ref/libpetl_ref.so``.  Its projector, backprojector,
PFDR, FBP and regularizers exist only as CUDA, so this script has to run on a
machine with a GPU; geometry and the dataCube elementwise rules are CPU code
and run anywhere.

    python tests/golden/make_golden.py --out <dir> [--cpu-only] [--only case ...]

Each case is written as ``<name>.npz`` holding its inputs, the reference
arguments and the reference outputs.  The committed fixtures in this
directory were produced by this script; the tests read them, never the
reference library.

The solid-angle correction is CPU code too; apply_corrections divides on
the host and in-fills bad pixels with a CUDA kernel, so it needs a GPU.

List-mode binning is CPU code in the reference and runs anywhere (it reads
seeded coincidence files this script writes in the reference's formats).

The MLEM case drives the reference C ABI with the same call sequence as the
reference ``PETLserver.MLEM`` loop (src/petl_server.py:1534-1606): project,
rdivide4D, backproject, divide3D, multiply3D, with sensitivity =
backproject(ones) and zeros of the sensitivity replaced by one.
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libpetl_ref.so")

fp = ctypes.POINTER(ctypes.c_float)


class Ref:
    def __init__(self, path=REF_LIB):
        L = ctypes.CDLL(path)
        c_f, c_i, c_b = ctypes.c_float, ctypes.c_int, ctypes.c_bool
        L.create_new_model.restype = c_i
        L.set_model.argtypes = [c_i]
        L.add_planogram.argtypes = [c_f] * 7
        L.add_planogram.restype = c_b
        L.set_volume.argtypes = [c_i, c_i, c_i, c_f, c_f, c_f, c_f, c_f]
        L.set_volume.restype = c_b
        L.get_numPlanograms.restype = c_i
        L.get_planogramSize.argtypes = [c_i, ctypes.POINTER(c_i)]
        L.get_planogramSize.restype = c_b
        for n in ("project", "backproject", "FBP"):
            getattr(L, n).argtypes = [ctypes.POINTER(fp), fp]
            getattr(L, n).restype = c_b
        L.PFDR.argtypes = [ctypes.POINTER(fp), ctypes.POINTER(fp)]
        L.PFDR.restype = c_b
        L.rdivide4D.argtypes = [fp, fp, c_i, c_i, c_i, c_i]
        L.rdivide4D.restype = c_b
        L.divide3D.argtypes = [fp, fp, c_i, c_i, c_i]
        L.divide3D.restype = c_b
        L.multiply3D.argtypes = [fp, fp, c_i, c_i, c_i]
        L.multiply3D.restype = c_b
        L.reciprocal3D.argtypes = [fp, c_i, c_i, c_i, c_f]
        L.reciprocal3D.restype = c_b
        L.inner_product3D.argtypes = [fp, fp, fp, c_i, c_i, c_i]
        L.inner_product3D.restype = c_f
        L.relativeDifferences_gradient.argtypes = [fp, fp, c_i, c_i, c_i, c_f, c_f]
        L.relativeDifferences_gradient.restype = c_b
        L.TV_cost.argtypes = [fp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]
        L.TV_cost.restype = c_f
        L.TV_gradient.argtypes = [fp, fp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]
        L.TV_gradient.restype = c_b
        L.TV_quadForm.argtypes = [fp, fp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]
        L.TV_quadForm.restype = c_f
        L.diffuse.argtypes = [fp, c_i, c_i, c_i, c_f, c_f, c_i, c_b]
        L.diffuse.restype = c_b
        L.TV_denoise.argtypes = [fp, c_i, c_i, c_i, c_f, c_f, c_f, c_i, c_b, c_b]
        L.TV_denoise.restype = c_b
        L.gaussian_filter.argtypes = [fp, c_i, c_i, c_i, c_f, c_i]
        L.gaussian_filter.restype = c_b
        L.bin.argtypes = [ctypes.POINTER(fp), ctypes.c_char_p]
        L.bin.restype = c_b
        for n in ("add_object", "add_module"):
            getattr(L, n).argtypes = [c_i, fp, fp, c_f, fp, fp]
            getattr(L, n).restype = c_b
        L.clear_phantom.restype = c_b
        L.clear_modules.restype = c_b
        L.scale_phantom.argtypes = [c_f, c_f, c_f]
        L.scale_phantom.restype = c_b
        L.voxelize.argtypes = [fp, c_i]
        L.voxelize.restype = c_b
        for n in ("ray_trace", "stopping_power"):
            getattr(L, n).argtypes = [ctypes.POINTER(fp), c_i]
            getattr(L, n).restype = c_b
        L.set_solid_angle_correction.argtypes = [ctypes.POINTER(fp), c_b]
        L.set_solid_angle_correction.restype = c_b
        L.apply_corrections.argtypes = [ctypes.POINTER(fp), ctypes.POINTER(fp), c_f]
        L.apply_corrections.restype = c_b
        self.L = L

    def model(self, planograms, vol):
        m = self.L.create_new_model()
        self.L.set_model(m)
        for p in planograms:
            psi, D, L_, H, T, vm0, vm1 = p
            if not self.L.add_planogram(psi, D, L_, H, vm0, vm1, T):
                raise RuntimeError("add_planogram failed")
        if vol is not None and not self.L.set_volume(*vol):
            raise RuntimeError("set_volume failed")
        return m

    def shapes(self):
        out = []
        for i in range(self.L.get_numPlanograms()):
            s = (ctypes.c_int * 4)()
            self.L.get_planogramSize(i, s)
            out.append(tuple(s))
        return out

    @staticmethod
    def pp(arrs):
        """float** over the arrays; the returned object keeps them alive (a
        pointer taken from a temporary array would dangle once the array is
        freed, and large arrays are unmapped when freed)."""
        arrs = list(arrs)
        a = (fp * len(arrs))(*[x.ctypes.data_as(fp) for x in arrs])
        a._keep = arrs
        return a

    @staticmethod
    def check_device(what):
        """Stop at the first reference call that left the device in error:
        the reference prints a failure and carries on (its copies' return
        values are not checked), so a later call would run on bad pointers."""
        rt = ctypes.CDLL(os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "lib64", "libcudart.so"))
        e = rt.cudaDeviceSynchronize()
        if e == 0:
            e = rt.cudaGetLastError()
        if e != 0:
            raise RuntimeError(f"reference call {what} left CUDA error {e}")


def ptr(a):
    return a.ctypes.data_as(fp)


def ellipsoids(shape, vox, rng, n, vmin=0.1, vmax=1.0, background=0.0, axes=None):
    """Seeded ellipsoid phantom (replace semantics, insertion order); semi-axes
    a fraction of the volume, or uniform in `axes` (mm) when given."""
    nz, ny, nx = shape
    wx, wz = vox
    x = (np.arange(nx) - 0.5 * (nx - 1)) * wx
    y = (np.arange(ny) - 0.5 * (ny - 1)) * wx
    z = (np.arange(nz) - 0.5 * (nz - 1)) * wz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    f = np.full(shape, background, np.float32)
    ext = np.array([nx * wx, ny * wx, nz * wz]) * 0.5
    for _ in range(n):
        if axes is None:
            r = rng.uniform(0.08, 0.3, 3) * ext
        else:
            r = np.minimum(rng.uniform(axes[0], axes[1], 3), ext * 0.95)
        c = rng.uniform(-1, 1, 3) * np.maximum(ext - r, 0)
        val = rng.uniform(vmin, vmax)
        inside = ((X - c[0]) / r[0]) ** 2 + ((Y - c[1]) / r[1]) ** 2 + ((Z - c[2]) / r[2]) ** 2 <= 1.0
        f[inside] = val
    return f


GEOMS = {
    # name: (planograms [(psi, D, L, H, T, v_m0, v_m1)], volume (numX,numY,numZ,vw,vh,ox,oy,oz))
    "g0": ([(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)], (32, 32, 8, 2.0, 2.0, 0.0, 0.0, 0.0)),
    "g90": ([(90.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)], (32, 32, 8, 2.0, 2.0, 0.0, 0.0, 0.0)),
    "g30": ([(30.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)], (32, 32, 8, 2.0, 2.0, 0.0, 0.0, 0.0)),
    "gpitch": ([(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)], (40, 40, 12, 1.5, 1.25, 1.0, -2.0, 0.5)),
    "gpetx": ([(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), (90.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)],
              (32, 32, 8, 2.0, 2.0, 0.0, 0.0, 0.0)),
    "g0t1": ([(0.0, 48.0, 24.0, 16.0, 1.0, 0.5, 0.25)], (48, 48, 16, 1.0, 1.0, 0.0, 0.0, 0.0)),
}


def run_projectors(ref, out):
    for name, (plans, vol) in GEOMS.items():
        rng = np.random.default_rng(sum(map(ord, name)))
        ref.model(plans, vol)
        shapes = ref.shapes()
        vshape = (vol[2], vol[1], vol[0])
        f = ellipsoids(vshape, (vol[3], vol[4]), rng, 6)
        f_noise = rng.random(vshape).astype(np.float32)
        g = [np.zeros(s, np.float32) for s in shapes]
        if not ref.L.project(ref.pp(g), ptr(f)):
            raise RuntimeError("project failed")
        g_noise = [np.zeros(s, np.float32) for s in shapes]
        ref.L.project(ref.pp(g_noise), ptr(f_noise))
        y = [rng.random(s).astype(np.float32) for s in shapes]
        b = np.zeros(vshape, np.float32)
        if not ref.L.backproject(ref.pp(y), ptr(b)):
            raise RuntimeError("backproject failed")
        ones = [np.ones(s, np.float32) for s in shapes]
        sens = np.zeros(vshape, np.float32)
        ref.L.backproject(ref.pp(ones), ptr(sens))
        rec = dict(planograms=np.array(plans, np.float64), volume=np.array(vol, np.float64),
                   f=f, f_noise=f_noise, sens=sens, b=b)
        for i, s in enumerate(shapes):
            rec[f"g{i}"] = g[i]
            rec[f"gnoise{i}"] = g_noise[i]
            rec[f"y{i}"] = y[i]
        np.savez_compressed(os.path.join(out, f"proj_{name}.npz"), **rec)
        print("wrote", name, shapes)


def run_pfdr_fbp(ref, out):
    for name in ("g0", "g0t1"):
        plans, vol = GEOMS[name]
        ref.model(plans, vol)
        shapes = ref.shapes()
        vshape = (vol[2], vol[1], vol[0])
        rng = np.random.default_rng(1234 + len(name))
        f = ellipsoids(vshape, (vol[3], vol[4]), rng, 6)
        g = [np.zeros(s, np.float32) for s in shapes]
        ref.L.project(ref.pp(g), ptr(f))
        fbp = np.zeros(vshape, np.float32)
        if not ref.L.FBP(ref.pp(g), ptr(fbp)):
            raise RuntimeError("FBP failed")
        # PFDR changes the model's planogram (N_v1 -> 1): do it last
        greb = [np.zeros(s[1:], np.float32) for s in shapes]
        if not ref.L.PFDR(ref.pp(g), ref.pp(greb)):
            raise RuntimeError("PFDR failed")
        shapes_after = ref.shapes()
        np.savez_compressed(os.path.join(out, f"pfdr_{name}.npz"), planograms=np.array(plans, np.float64),
                            volume=np.array(vol, np.float64), f=f, g=g[0], g_reb=greb[0], fbp=fbp,
                            shape_after=np.array(shapes_after[0]))
        print("wrote pfdr", name)


def run_mlem(ref, out):
    plans, vol = GEOMS["g0"]
    ref.model(plans, vol)
    shape = ref.shapes()[0]
    vshape = (vol[2], vol[1], vol[0])
    rng = np.random.default_rng(777)
    ftrue = ellipsoids(vshape, (vol[3], vol[4]), rng, 6)
    g = [np.zeros(shape, np.float32)]
    ref.L.project(ref.pp(g), ptr(ftrue))
    g[0] *= np.float32(2e5 / g[0].sum())
    g = [rng.poisson(g[0]).astype(np.float32)]
    rec = dict(planograms=np.array(plans, np.float64), volume=np.array(vol, np.float64), g=g[0])
    for beta, tag in ((0.0, "plain"), (0.05, "rd")):
        f = np.ones(vshape, np.float32)
        ones = [np.ones(shape, np.float32)]
        sens = np.zeros(vshape, np.float32)
        ref.L.backproject(ref.pp(ones), ptr(sens))
        sens[sens == 0.0] = 1.0
        d = np.zeros(vshape, np.float32)
        Pd = [np.zeros(shape, np.float32)]
        iters = []
        for n in range(4):
            ref.L.project(ref.pp(Pd), ptr(f))
            ref.L.rdivide4D(ptr(g[0]), ptr(Pd[0]), *shape)
            ref.L.backproject(ref.pp(Pd), ptr(d))
            if beta <= 0.0:
                ref.L.divide3D(ptr(d), ptr(sens), *vshape)
                ref.L.multiply3D(ptr(f), ptr(d), *vshape)
            else:
                tv = np.zeros(vshape, np.float32)
                ref.L.relativeDifferences_gradient(ptr(f), ptr(tv), *vshape, 2.0, beta)
                tv[:] += sens[:]
                np.maximum(np.float32(0.1) * sens, tv, out=tv)
                ref.L.divide3D(ptr(d), ptr(tv), *vshape)
                ref.L.multiply3D(ptr(f), ptr(d), *vshape)
            iters.append(f.copy())
        rec[f"f_{tag}"] = np.stack(iters)
        rec[f"sens_{tag}"] = sens
    np.savez_compressed(os.path.join(out, "mlem_g0.npz"), **rec)
    print("wrote mlem")


def run_regularizers(ref, out):
    ref.model([GEOMS["g0"][0][0]], GEOMS["g0"][1])
    rng = np.random.default_rng(4242)
    rec = {}
    for tag, shape in (("3d", (10, 12, 14)), ("2d", (1, 16, 18))):
        f = (rng.random(shape) * 2.0).astype(np.float32)
        f[0, 0, :3] = 0.0  # exercise the x == y == 0 branches
        d = rng.standard_normal(shape).astype(np.float32)
        rec[f"f_{tag}"] = f
        rec[f"d_{tag}"] = d
        Df = np.zeros(shape, np.float32)
        ref.L.relativeDifferences_gradient(ptr(f), ptr(Df), *shape, 2.0, 0.01)
        rec[f"rd_grad_{tag}"] = Df
        for delta, p in ((0.05, 1.0), (0.3, 1.2)):
            key = f"{tag}_d{delta}_p{p}"
            Dt = np.zeros(shape, np.float32)
            ref.L.TV_gradient(ptr(f), ptr(Dt), *shape, delta, 0.7, p, True)
            rec[f"tv_grad_{key}"] = Dt
            rec[f"tv_cost_{key}"] = np.float64(ref.L.TV_cost(ptr(f), *shape, delta, 0.7, p, True))
            rec[f"tv_quad_{key}"] = np.float64(ref.L.TV_quadForm(ptr(f), ptr(d), *shape, delta, 0.7, p, True))
        fd = f.copy()
        ref.L.diffuse(ptr(fd), *shape, 0.05, 1.0, 3, True)
        rec[f"diffuse_{tag}"] = fd
        fn = f.copy()
        ref.L.TV_denoise(ptr(fn), *shape, 0.05, 0.5, 1.0, 3, False, True)
        rec[f"tvdenoise_{tag}"] = fn
    np.savez_compressed(os.path.join(out, "regularizers.npz"), **rec)
    print("wrote regularizers")


def run_cpu(ref, out):
    """Geometry and dataCube rules: CPU-only reference code."""
    rec = {}
    calls = [(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25), (0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25),
             (0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25), (30.0, 180.0, 192.0, 144.0, 2.0, 0.2679, 0.2679),
             (0.0, 200.0, 96.0, 64.0, 1.5, 0.5, 0.25), (45.0, 300.0, 256.0, 128.0, 1.7, 0.4, 0.3),
             (0.0, 256.0, 256.0, 128.0, 2.0, 0.5, 0.25), (90.0, 100.0, 50.0, 40.0, 0.8, 1.0, 0.9)]
    shapes = []
    for c in calls:
        ref.model([c], None)
        shapes.append(ref.shapes()[0])
    rec["geom_calls"] = np.array(calls)
    rec["geom_shapes"] = np.array(shapes)
    rng = np.random.default_rng(99)
    a = rng.random((3, 4, 5, 6)).astype(np.float32)
    b = rng.random((3, 4, 5, 6)).astype(np.float32)
    a.flat[::7] = 0.0
    b.flat[::5] = 0.0
    r = b.copy()
    ref.L.rdivide4D(ptr(a), ptr(r), *a.shape)
    rec["rd_num"], rec["rd_den"], rec["rd_out"] = a, b, r
    x3, y3 = a[0].copy(), b[0].copy()
    ref.L.divide3D(ptr(x3), ptr(y3), *x3.shape)
    rec["div_x"], rec["div_y"], rec["div_out"] = a[0], b[0], x3
    rr = b[1].copy()
    ref.L.reciprocal3D(ptr(rr), *rr.shape, 7.0)
    rec["recip_in"], rec["recip_out"] = b[1], rr
    rec["ip"] = np.float64(ref.L.inner_product3D(ptr(a[2]), ptr(b[2]), None, *a[2].shape))
    np.savez_compressed(os.path.join(out, "cpu_rules.npz"), **rec)
    print("wrote cpu rules", shapes)


def run_binning(ref, out):
    """List-mode binning: CPU reference code (src/binning.cpp).  Events are
    seeded coincidences on the panels (petl_b200.listmode), written in the
    reference's two file formats and binned by the reference's bin(); the
    planograms are pre-filled with 7 to record that bin() overwrites them."""
    sys.path.insert(0, ROOT)
    from petl_b200 import listmode
    import tempfile
    cases = {
        # name: (planograms, volume, file format, [(psi of the panels, events)])
        "bin_g0": ([GEOMS["g0"][0][0]], GEOMS["g0"][1], "acq", [(0.0, 4000)]),
        "bin_g0t1": ([GEOMS["g0t1"][0][0]], GEOMS["g0t1"][1], "lst", [(0.0, 4000)]),
        "bin_gpetx": (GEOMS["gpetx"][0], GEOMS["gpetx"][1], "acq", [(0.0, 2000), (90.0, 2000)]),
    }
    rec = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (plans, vol, fmt, srcs) in cases.items():
            rng = np.random.default_rng(sum(map(ord, name)))
            bl, pk = [], []
            for psi_p, n in srcs:
                _, D, L_, H, _, _, _ = plans[0]
                b, p = listmode.coincidences(n, rng, D / 2, L_ / 2, H / 2, psi_deg=psi_p,
                                             box=(0.6 * L_ / 2, 0.6 * L_ / 2, 0.6 * H / 2))
                bl.append(b)
                pk.append(p)
            blue, pink = np.concatenate(bl), np.concatenate(pk)
            path = os.path.join(tmp, name + (".lst" if fmt == "lst" else ".dat"))
            counts = listmode.interaction_counts(len(blue), rng, 0.2)
            if fmt == "lst":
                listmode.write_lst(path, blue, pink)
            else:
                listmode.write_acq(path, blue, pink, counts)
            ref.model(plans, vol)
            gs = [np.full(sh, 7.0, np.float32) for sh in ref.shapes()]
            if not ref.L.bin(ref.pp(gs), path.encode()):
                raise RuntimeError("reference bin failed")
            rec[f"{name}_planograms"] = np.array(plans)
            rec[f"{name}_volume"] = np.array(vol)
            rec[f"{name}_blue"], rec[f"{name}_pink"] = blue, pink
            rec[f"{name}_format"] = np.array(fmt)
            rec[f"{name}_nb"], rec[f"{name}_np"] = counts
            for i, g in enumerate(gs):
                rec[f"{name}_g{i}"] = g
    np.savez_compressed(os.path.join(out, "binning.npz"), **rec)
    print("wrote binning", {k: float(v.sum()) for k, v in rec.items() if k[-3:-1] == "_g"})


# Solids of the phantom cases: (type, centre, radii, value, rotation, clip)
# (types: 0 ellipsoid, 1 box, 2/3/4 cylinder x/y/z, 5/6/7 cone x/y/z; cones
# take (l, r_1, r_2) in the reference's per-axis order)
_C30 = float(np.cos(np.pi / 6)), float(np.sin(np.pi / 6))
PHANTOM = [
    (0, (2.0, -3.0, 1.0), (10.0, 7.0, 4.0), 1.0, None, None),
    (1, (-5.0, 4.0, 0.0), (4.0, 3.0, 2.0), 2.0, None, None),
    (4, (6.0, 6.0, 0.0), (3.0, 3.0, 5.0), 0.5, None, None),
    (2, (0.0, -8.0, 2.0), (8.0, 2.0, 2.0), 1.5, None, None),
    (3, (-8.0, 0.0, -2.0), (2.0, 9.0, 2.0), 0.7, None, None),
    (7, (0.0, 0.0, 0.0), (2.0, 4.0, 5.0), 0.3, None, None),
    (5, (5.0, -5.0, -2.0), (4.0, 1.0, 3.0), 0.9, None, None),
    (6, (-4.0, -6.0, 1.0), (1.0, 5.0, 3.0), 1.2, None, None),
    (0, (10.0, -10.0, 0.0), (6.0, 2.0, 3.0), 0.8,
     ((_C30[0], -_C30[1], 0.0), (_C30[1], _C30[0], 0.0), (0.0, 0.0, 1.0)), None),
    (1, (-10.0, -12.0, 0.0), (5.0, 5.0, 3.0), 1.1, None, (1.0, 0.0, 0.0)),
]


def _rot(axis, deg):
    """Rotation by deg degrees about x (0), y (1) or z (2), as a 3x3 tuple."""
    c, s_ = float(np.cos(np.radians(deg))), float(np.sin(np.radians(deg)))
    R = np.eye(3)
    i, j = [(1, 2), (0, 2), (0, 1)][axis]
    R[i, i], R[i, j], R[j, i], R[j, j] = c, -s_, s_, c
    return tuple(map(tuple, R))


# Rotated cylinders, cones and boxes, clipping on y and z, a negative value
# and overlaps.
PHANTOM2 = [
    (1, (0.0, 0.0, 0.0), (20.0, 18.0, 6.0), 0.2, None, None),
    (4, (-6.0, 4.0, 0.0), (4.0, 3.0, 5.0), 1.3, _rot(0, 40.0), None),
    (5, (8.0, 6.0, 1.0), (6.0, 1.5, 3.5), 0.7, _rot(2, 20.0), None),
    (7, (-8.0, -8.0, -1.0), (1.0, 3.0, 4.0), 0.6, _rot(1, 15.0), None),
    (0, (6.0, -6.0, 0.0), (7.0, 5.0, 4.0), 1.8, None, (0.0, 1.0, 0.0)),
    (2, (0.0, 10.0, 1.0), (9.0, 2.5, 2.5), 0.9, None, (0.0, 0.0, 2.0)),
    (1, (12.0, -12.0, 0.0), (3.0, 4.0, 3.0), -0.5, _rot(1, 30.0), None),
    (3, (-12.0, 0.0, 2.0), (2.0, 8.0, 2.0), 1.1, _rot(2, -25.0), None),
    (6, (0.0, -14.0, 0.0), (2.0, 4.0, 1.0), 0.4, None, None),
]


def _add_solids(fn, solids):
    for t, c, r, v, A, clip in solids:
        c = np.array(c, np.float32)
        r = np.array(r, np.float32)
        A = np.eye(3, dtype=np.float32) if A is None else np.array(A, np.float32)
        clip = np.zeros(3, np.float32) if clip is None else np.array(clip, np.float32)
        if not fn(t, ptr(c), ptr(r), v, ptr(A), ptr(clip)):
            raise RuntimeError("reference rejected a solid")


def _modules(D, L_, H):
    """Four detector slabs around a planogram pair's field of view, as the
    reference's simple PET/X module model (src/petx_server.py:22-27)."""
    return [(1, (0.0, 0.5 * D + 10.0, 0.0), (0.5 * L_, 10.0, 0.5 * H), 0.0815, None, None),
            (1, (0.0, -0.5 * D - 10.0, 0.0), (0.5 * L_, 10.0, 0.5 * H), 0.0815, None, None),
            (1, (0.5 * L_ + 10.0, 0.0, 0.0), (10.0, 0.5 * D + 20.0, 0.5 * H), 0.0815, None, None),
            (1, (-0.5 * L_ - 10.0, 0.0, 0.0), (10.0, 0.5 * D + 20.0, 0.5 * H), 0.0815, None, None)]


def run_voxelize(ref, out):
    """phantom::voxelize (CPU code, src/phantom.cpp:105-335) of the PHANTOM
    solids into a volume pre-filled with 0.25 (values outside every solid are
    kept), with 1 and 3 sub-samples per axis, and after scale_phantom."""
    rec = {}
    vol = (32, 32, 8, 2.0, 2.0, 0.0, 0.0, 0.0)
    ref.model([GEOMS["g0"][0][0]], vol)
    ref.L.clear_phantom()
    _add_solids(ref.L.add_object, PHANTOM)
    for os_ in (1, 3):
        f = np.full((vol[2], vol[1], vol[0]), 0.25, np.float32)
        if not ref.L.voxelize(ptr(f), os_):
            raise RuntimeError("reference voxelize failed")
        rec[f"f_os{os_}"] = f
    ref.L.scale_phantom(1.25, 0.8, 1.1)
    f = np.full((vol[2], vol[1], vol[0]), 0.25, np.float32)
    ref.L.voxelize(ptr(f), 1)
    rec["f_scaled"] = f
    ref.L.clear_phantom()
    _add_solids(ref.L.add_object, PHANTOM2)
    for os_ in (1, 5):
        f = np.zeros((vol[2], vol[1], vol[0]), np.float32)
        ref.L.voxelize(ptr(f), os_)
        rec[f"f2_os{os_}"] = f
    rec["volume"] = np.array(vol)
    np.savez_compressed(os.path.join(out, "voxelize.npz"), **rec)
    print("wrote voxelize", {k: float(v.sum()) for k, v in rec.items() if k.startswith("f_")})


def run_raytrace(ref, out):
    """Analytic ray tracing (rayTracingKernel) of the PHANTOM solids and the
    stopping power (stoppingPowerKernel) of a four-slab module model, CUDA
    code in the reference, so this case needs a GPU."""
    rec = {}
    for name in ("g0", "g30", "gpetx"):
        plans, vol = GEOMS[name]
        ref.model(plans, vol)
        ref.L.clear_phantom()
        ref.L.clear_modules()
        _add_solids(ref.L.add_object, PHANTOM)
        _, D, L_, H, _, _, _ = plans[0]
        _add_solids(ref.L.add_module, _modules(D, L_, H))
        for os_ in (1, 3):
            gs = [np.full(sh, 7.0, np.float32) for sh in ref.shapes()]
            if not ref.L.ray_trace(ref.pp(gs), os_):
                raise RuntimeError("reference ray_trace failed")
            for i, g in enumerate(gs):
                rec[f"{name}_rt{os_}_{i}"] = g
        ref.L.clear_phantom()
        _add_solids(ref.L.add_object, PHANTOM2)
        gs = [np.full(sh, 7.0, np.float32) for sh in ref.shapes()]
        if not ref.L.ray_trace(ref.pp(gs), 1):
            raise RuntimeError("reference ray_trace failed")
        for i, g in enumerate(gs):
            rec[f"{name}_rt2_{i}"] = g
        gs = [np.full(sh, 7.0, np.float32) for sh in ref.shapes()]
        if not ref.L.stopping_power(ref.pp(gs), 1):
            raise RuntimeError("reference stopping_power failed")
        for i, g in enumerate(gs):
            rec[f"{name}_sp_{i}"] = g
        rec[f"{name}_planograms"] = np.array(plans)
        rec[f"{name}_volume"] = np.array(vol)
    np.savez_compressed(os.path.join(out, "raytrace.npz"), **rec)
    print("wrote raytrace", {k: float(v.sum()) for k, v in rec.items() if "_rt" in k or "_sp" in k})


def run_demo(ref, out):
    """The reference's geometry demo (demo/d01_set_geometry.py): six
    planograms at psi = 0, 30, ..., 150 degrees (D 180, L 192, H 144, T 2,
    v_m0 = v_m1 = tan 15 degrees), the default volume, two ellipsoids traced
    analytically and reconstructed by FBP.  CUDA code in the reference, so
    this case needs a GPU; the FBP volume is recorded."""
    t15 = float(np.tan(np.radians(15.0)))
    plans = [(n * 30.0, 180.0, 192.0, 144.0, 2.0, t15, t15) for n in range(6)]
    m = ref.L.create_new_model()
    ref.L.set_model(m)
    for psi, D, L_, H, T, vm0, vm1 in plans:
        if not ref.L.add_planogram(psi, D, L_, H, vm0, vm1, T):
            raise RuntimeError("add_planogram failed")
    ref.L.set_default_volume.argtypes = [ctypes.c_float]
    ref.L.set_default_volume.restype = ctypes.c_bool
    ref.L.set_default_volume(1.0)
    for n in ("get_numX", "get_numY", "get_numZ"):
        getattr(ref.L, n).restype = ctypes.c_int
    ref.L.get_voxelWidth.restype = ctypes.c_float
    ref.L.get_voxelHeight.restype = ctypes.c_float
    vol = (ref.L.get_numX(), ref.L.get_numY(), ref.L.get_numZ(), ref.L.get_voxelWidth(), ref.L.get_voxelHeight())
    ref.L.clear_phantom()
    _add_solids(ref.L.add_object, [(0, (0.0, 0.0, 0.0), (90.0, 80.0, 70.0), 100.0, None, None),
                                   (0, (0.0, 0.0, 0.0), (5.0, 5.0, 5.0), 1000.0, None, None)])
    gs = [np.zeros(sh, np.float32) for sh in ref.shapes()]
    if not ref.L.ray_trace(ref.pp(gs), 1):
        raise RuntimeError("reference ray_trace failed")
    f = np.zeros((vol[2], vol[1], vol[0]), np.float32)
    if not ref.L.FBP(ref.pp(gs), ptr(f)):
        raise RuntimeError("reference FBP failed")
    np.savez_compressed(os.path.join(out, "demo_d01.npz"), planograms=np.array(plans), volume=np.array(vol), f=f,
                        g_sums=np.array([g.sum(dtype=np.float64) for g in gs]))
    print("wrote demo", vol, float(f.sum()))


def run_solid_angle(ref, out):
    """Solid-angle correction (CPU code, src/planogram.cpp:262-302) of all-ones
    planograms: the output is the per-projection factor, recorded as a table
    (N_v1, N_v0) for the correction and for its inverse (the model)."""
    cases = {"sa_g0": GEOMS["g0"], "sa_g0t1": GEOMS["g0t1"], "sa_gpetx": GEOMS["gpetx"],
             "sa_bench": ([(0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)], (256, 256, 128, 1.0, 1.0, 0.0, 0.0, 0.0))}
    rec = {}
    for name, (plans, vol) in cases.items():
        ref.model(plans, vol)
        rec[f"{name}_planograms"] = np.array(plans)
        rec[f"{name}_volume"] = np.array(vol)
        for inv in (False, True):
            gs = [np.ones(sh, np.float32) for sh in ref.shapes()]
            if not ref.L.set_solid_angle_correction(ref.pp(gs), inv):
                raise RuntimeError("reference set_solid_angle_correction failed")
            for i, g in enumerate(gs):
                tab = g[:, :, :1, :1].copy()
                if not np.array_equal(np.broadcast_to(tab, g.shape), g):
                    raise RuntimeError("solid-angle output is not one factor per projection")
                rec[f"{name}_c{int(inv)}_{i}"] = tab[:, :, 0, 0]
            del gs
    np.savez_compressed(os.path.join(out, "solid_angle.npz"), **rec)
    print("wrote solid angle", sorted(k for k in rec if "_c" in k))


def _fov_margin(G, eps):
    """Pixels of planogram G whose field-of-view test (the projector's ray
    mask, src/median_filter.cu:26-39) holds with margin eps in float64
    (eps > 0: surely inside, whatever the float rounding)."""
    v1 = np.arange(G.N_v1) * G.T_v1 + G.v1_0
    v0 = np.arange(G.N_v0) * G.T_v0 + G.v0_0
    u1 = np.arange(G.N_u1) * G.T_u1 + G.u1_0
    u0 = np.arange(G.N_u0) * G.T_u0 + G.u0_0
    a = (np.abs(u0)[None, None, None, :] - 0.5 * G.T_u0) <= G.L + G.R * np.abs(v0)[None, :, None, None] - eps
    b = (np.abs(u1)[None, None, :, None] - 0.5 * G.T_u1) <= G.H - G.R * np.abs(v1)[:, None, None, None] - eps
    return a & b


def run_corrections(ref, out):
    """apply_corrections (src/petl.cpp:163-192): g / r on the host, then the
    bad-pixel median in-fill, a CUDA kernel (src/median_filter.cu), so this
    case needs a GPU.  The reference kernel rewrites g in place while other
    threads read it; the inputs keep every window free of pixels that the
    launch rewrites to a different value, so its result is the same whatever
    the thread order: g is 0 wherever a pixel may lie outside the field of
    view (those are rewritten to 0; bins on the boundary, where rounding
    decides, included), and the bad pixels (r below the
    threshold) are at least 3 apart in (u1, u0).  g holds Poisson counts with
    a rate drawn per projection (many zeros, so windows hold from 0 to 25
    good values), r quantized values in [1, 1.5] with the bad bins planted
    below 0.375 (some at 0); the outputs are stored
    as the entries where they differ from the plain division g / r."""
    sys.path.insert(0, ROOT)
    import oracle as O  # geometry values only
    rec = {}
    for name in ("g0", "g0t1", "gpetx"):
        plans, vol = GEOMS[name]
        rng = np.random.default_rng(sum(map(ord, "corr_" + name)))
        ref.model(plans, vol)
        gs, rs = [], []
        for p, sh in zip(plans, ref.shapes()):
            G = O.make_geom(*p, vol)
            inside = _fov_margin(G, 1e-3)
            lam = rng.uniform(0.05, 3.0, size=sh[:2])[:, :, None, None]
            g = rng.poisson(lam, size=sh).astype(np.float32)
            g[~inside] = 0.0
            # responses in [1, 1.5]: 0.75 of any projection's median stays
            # below 1, so only the planted bins fall under the threshold
            r = (rng.integers(64, 97, size=sh) / 64.0).astype(np.float32)
            bad = np.zeros(sh, bool)
            for iv1 in range(sh[0]):
                for iv0 in range(sh[1]):
                    taken = []
                    for _ in range(sh[2] * sh[3] // 12):
                        j, i = int(rng.integers(sh[2])), int(rng.integers(sh[3]))
                        if all(max(abs(j - a), abs(i - b)) >= 3 for a, b in taken):
                            taken.append((j, i))
                            bad[iv1, iv0, j, i] = True
            kind = rng.integers(0, 3, size=sh)
            r[bad & (kind == 0)] = 0.0
            r[bad & (kind != 0)] = (rng.integers(1, 24, size=int((bad & (kind != 0)).sum())) / 64.0).astype(np.float32)
            thr = 0.75 * np.median(r.reshape(sh[0] * sh[1], -1), axis=1).reshape(sh[:2])[:, :, None, None]
            if not np.array_equal(r < thr, bad):
                raise RuntimeError("bins other than the planted ones fall below the threshold")
            gs.append(g)
            rs.append(r)
        g_in = [g.copy() for g in gs]
        if not ref.L.apply_corrections(ref.pp(gs), ref.pp(rs), 0.75):
            raise RuntimeError("reference apply_corrections failed")
        rec[f"{name}_planograms"] = np.array(plans)
        rec[f"{name}_volume"] = np.array(vol)
        for i, (g0, r, g1) in enumerate(zip(g_in, rs, gs)):
            plain = np.where(r == 0, np.float32(0), g0 / np.where(r == 0, np.float32(1), r)).astype(np.float32)
            idx = np.flatnonzero(g1.ravel() != plain.ravel())
            rec[f"{name}_g{i}"], rec[f"{name}_r{i}"] = g0, r
            rec[f"{name}_idx{i}"], rec[f"{name}_val{i}"] = idx.astype(np.int32), g1.ravel()[idx]
            print("corrections", name, i, "changed", idx.size, "of", g1.size)
    np.savez_compressed(os.path.join(out, "corrections.npz"), **rec)


# The two workloads at their stated sizes: the dual-panel geometry at 2 mm
# (planogram (33, 65, 64, 128), volume 128x128x64) and at 1 mm (planogram
# (65, 129, 128, 256), volume 256x256x128).  Outputs are stored for a few
# views / planes only, so that the fixtures stay small; the inputs are
# stored whole (piecewise-constant phantoms compress well) or regenerated
# from seeds and checked by checksum.
CFG0 = ((0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25), (128, 128, 64, 2.0, 2.0, 0.0, 0.0, 0.0))
CFG1 = ((0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25), (256, 256, 128, 1.0, 1.0, 0.0, 0.0, 0.0))
CFG0_VIEWS = ((0, 0), (0, 32), (8, 20), (16, 32), (16, 64), (24, 45), (32, 32), (32, 64))  # (iv1, iv0)
CFG0_PLANES = (5, 20, 32, 44, 60)
CFG1_VIEWS = ((0, 64), (20, 10), (32, 64), (64, 128))
CFG1_PLANES = (20, 64)
CFG1_REB = (0, 40, 64, 128)


def config_phantom(which):
    """The seeded ellipsoid phantoms of the two workloads: semi-axes 2.5-20 mm
    (axes 5-40 mm), activities 0.1-1.0; twelve ellipsoids at 2 mm, thirty
    plus a uniform background of 1 % of the maximum at 1 mm."""
    plans, vol = (CFG0, CFG1)[which]
    vshape = (vol[2], vol[1], vol[0])
    if which == 0:
        return ellipsoids(vshape, (vol[3], vol[4]), np.random.default_rng(20260), 12, axes=(2.5, 20.0))
    f = ellipsoids(vshape, (vol[3], vol[4]), np.random.default_rng(20261), 30, axes=(2.5, 20.0))
    return f + np.float32(0.01) * f.max()


def config0_counts(f):
    """Poisson data of the 2 mm workload: 5e6 expected counts on the FP64
    oracle projection of the phantom (seeded), float32 counts."""
    sys.path.insert(0, ROOT)
    import oracle as O
    plans, vol = CFG0
    Go = O.make_geom(*plans, vol)
    return config0_counts_from(O.project(Go, f)[0])


def config0_counts_from(lam):
    lam = lam * (5e6 / lam.sum())
    return np.random.default_rng(20262).poisson(lam).astype(np.float32)


def counts_crc(g):
    import zlib
    return np.int64(zlib.crc32(np.ascontiguousarray(g, np.float32).tobytes()))


def run_config0(ref, out):
    plans, vol = CFG0
    ref.model([plans], vol)
    shape = ref.shapes()[0]
    vshape = (vol[2], vol[1], vol[0])
    f = config_phantom(0)
    g = [np.zeros(shape, np.float32)]
    if not ref.L.project(ref.pp(g), ptr(f)):
        raise RuntimeError("project failed")
    ref.check_device("project")
    counts = config0_counts(f)
    b = np.zeros(vshape, np.float32)
    if not ref.L.backproject(ref.pp([counts]), ptr(b)):
        raise RuntimeError("backproject failed")
    ref.check_device("backproject")
    ones = np.ones(shape, np.float32)
    sens = np.zeros(vshape, np.float32)
    ref.L.backproject(ref.pp([ones]), ptr(sens))
    ref.check_device("backproject (sensitivity)")
    sens[sens == 0.0] = 1.0
    # PETLserver.MLEM's call sequence (src/petl_server.py:1534-1606), 20 iterations from f = 1
    x = np.ones(vshape, np.float32)
    Pd = [np.zeros(shape, np.float32)]
    d = np.zeros(vshape, np.float32)
    keep = {}
    for n in range(20):
        ref.L.project(ref.pp(Pd), ptr(x))
        ref.L.rdivide4D(ptr(counts), ptr(Pd[0]), *shape)
        ref.L.backproject(ref.pp(Pd), ptr(d))
        ref.L.divide3D(ptr(d), ptr(sens), *vshape)
        ref.L.multiply3D(ptr(x), ptr(d), *vshape)
        ref.check_device(f"MLEM iteration {n + 1}")
        if n + 1 in (1, 20):
            keep[n + 1] = x[list(CFG0_PLANES)].copy()
    views = np.array(CFG0_VIEWS)
    planes = np.array(CFG0_PLANES)
    np.savez_compressed(os.path.join(out, "config0.npz"), planograms=np.array([plans], np.float64),
                        volume=np.array(vol, np.float64), shape=np.array(shape), f=f, views=views,
                        g_views=g[0][views[:, 0], views[:, 1]], counts_sum=np.float64(counts.sum()),
                        counts_crc=counts_crc(counts), planes=planes, b_planes=b[planes],
                        sens_planes=sens[planes], mlem1_planes=keep[1], mlem20_planes=keep[20])
    print("wrote config0", shape)


def run_config1(ref, out):
    plans, vol = CFG1
    ref.model([plans], vol)
    shape = ref.shapes()[0]
    vshape = (vol[2], vol[1], vol[0])
    f = config_phantom(1)
    g = [np.zeros(shape, np.float32)]
    if not ref.L.project(ref.pp(g), ptr(f)):
        raise RuntimeError("project failed")
    ref.check_device("project")
    b = np.zeros(vshape, np.float32)
    ref.L.backproject(ref.pp(g), ptr(b))
    ref.check_device("backproject")
    fbp = np.zeros(vshape, np.float32)
    if not ref.L.FBP(ref.pp(g), ptr(fbp)):
        raise RuntimeError("FBP failed")
    ref.check_device("FBP")
    greb = [np.zeros(shape[1:], np.float32)]
    if not ref.L.PFDR(ref.pp(g), ref.pp(greb)):  # rewrites the model to N_v1 = 1: last
        raise RuntimeError("PFDR failed")
    ref.check_device("PFDR")
    views = np.array(CFG1_VIEWS)
    planes = np.array(CFG1_PLANES)
    reb = np.array(CFG1_REB)
    np.savez_compressed(os.path.join(out, "config1.npz"), planograms=np.array([plans], np.float64),
                        volume=np.array(vol, np.float64), shape=np.array(shape), views=views,
                        g_views=g[0][views[:, 0], views[:, 1]], planes=planes, b_planes=b[planes],
                        fbp_planes=fbp[planes], reb_views=reb, greb_views=greb[0][reb])
    print("wrote config1", shape)


def run_gaussian(ref, out):
    """gaussian_filter (src/relative_differences.cu:314-411,753-800) along 1, 2
    and 3 dimensions, and the RWLS weight width (FWHM 3) and the response
    smoothing width (FWHM 0.6571) of the reference's Python layer."""
    ref.model([GEOMS["g0"][0][0]], GEOMS["g0"][1])
    rng = np.random.default_rng(5151)
    rec = {}
    shape = (9, 14, 23)
    for numDims in (1, 2, 3):
        for fwhm in (0.6571, 2.0, 3.0):
            f = (rng.random(shape) * 3.0).astype(np.float32)
            out_f = f.copy()
            if not ref.L.gaussian_filter(ptr(out_f), *shape, fwhm, numDims):
                raise RuntimeError("gaussian_filter failed")
            ref.check_device("gaussian_filter")
            rec[f"in_{numDims}_{fwhm}"] = f
            rec[f"out_{numDims}_{fwhm}"] = out_f
    np.savez_compressed(os.path.join(out, "gaussian.npz"), shape=np.array(shape), **rec)
    print("wrote gaussian")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--cpu-only", action="store_true")
    ap.add_argument("--only", nargs="*", default=None,
                    help="run only these cases (cpu, binning, solid_angle, voxelize, corrections, raytrace, demo, "
                         "projectors, pfdr_fbp, mlem, regularizers, config0, config1, gaussian)")
    ap.add_argument("--lib", default=REF_LIB)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    ref = Ref(a.lib)
    runs = [("cpu", run_cpu, False), ("binning", run_binning, False), ("solid_angle", run_solid_angle, False),
            ("voxelize", run_voxelize, False), ("corrections", run_corrections, True),
            ("raytrace", run_raytrace, True), ("demo", run_demo, True), ("projectors", run_projectors, True),
            ("pfdr_fbp", run_pfdr_fbp, True), ("mlem", run_mlem, True), ("regularizers", run_regularizers, True),
            ("config0", run_config0, True), ("config1", run_config1, True), ("gaussian", run_gaussian, True)]
    for name, fn, gpu in runs:
        if (a.only is None or name in a.only) and not (gpu and a.cpu_only):
            fn(ref, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())

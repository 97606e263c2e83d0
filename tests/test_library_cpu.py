"""libpetl.so without a GPU: it loads, exports every declared symbol, and its
host-side logic (geometry, model registry, host elementwise rules) matches
the reference.  No compute call reaches the device here."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, load_golden

import petl_b200
from petl_b200 import Geometry
from petl_b200._lib import API, lib


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    pat = r"\b(?:bool|int|float|void|double|char)\s*\**\s*([A-Za-z_]\w*)\s*\("
    return {m.group(1) for m in re.finditer(pat, text)}


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(petl_b200.LIB_PATH)
    declared = _declared("petl.h") | _declared("petl_device.h")
    assert len(declared) > 90
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding describes every declared function
    bound = {n for n, _, _ in API}
    assert declared <= bound, sorted(declared - bound)


def test_reference_interface_symbols_present():
    # every extern "C" function of the reference interface header
    names = ["set_model", "create_new_model", "about", "copy_parameters", "clearAll", "print_parameters",
             "volume_defined", "geometry_defined", "get_numX", "set_numX", "get_numY", "set_numY", "get_numZ",
             "set_numZ", "get_voxelWidth", "set_voxelWidth", "get_voxelHeight", "set_voxelHeight", "get_offsetX",
             "set_offsetX", "get_offsetY", "set_offsetY", "get_offsetZ", "set_offsetZ", "get_numPlanograms",
             "get_planogramSize", "add_planogram", "remove_planogram", "keep_only_planogram",
             "set_default_volume", "set_volume", "bin", "simulate_scatter", "project", "backproject", "FBP",
             "PFDR", "add_object", "add_module", "clear_phantom", "clear_modules", "scale_phantom", "voxelize",
             "ray_trace", "stopping_power", "set_solid_angle_correction", "apply_corrections", "multiply3D",
             "multiply4D", "divide3D", "divide4D", "rdivide3D", "rdivide4D", "reciprocal3D", "reciprocal4D",
             "inner_product3D", "inner_product4D", "TV_cost", "TV_gradient", "TV_quadForm", "diffuse",
             "TV_denoise", "relativeDifferences_gradient", "gaussian_filter"]
    L = lib()
    for n in names:
        assert hasattr(L, n), n


def test_geometry_matches_reference_and_oracle():
    z = load_golden("cpu_rules.npz")
    for call, shape in zip(z["geom_calls"], z["geom_shapes"]):
        psi, D, L, H, T, vm0, vm1 = call
        G = Geometry(psi, D, L, H, T, vm0, vm1, volume=(16, 16, 8, 1.5))
        assert G.shape == tuple(shape)
        Go = O.make_geom(psi, D, L, H, T, vm0, vm1, (16, 16, 8, 1.5))
        for fld in ("T_v1", "T_v0", "T_u1", "T_u0", "v1_0", "v0_0", "u1_0", "u0_0", "cos_psi", "sin_psi",
                    "R", "L", "H", "v_m1", "x_0", "y_0", "z_0"):
            ours = getattr(G.g, fld)
            theirs = getattr(Go, fld)
            assert ours == theirs, (fld, ours, theirs)


def test_optimal_fft_size_matches_oracle():
    L = lib()
    for n in range(1, 2100):
        assert L.petl_optimal_fft_size(n) == O.optimal_fft_size(n)


def test_cabi_registry_and_geometry():
    from petl_b200 import PETLserver
    s = PETLserver()
    s.add_planogram(0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)
    assert tuple(s.get_planogramSize(0)) == (65, 129, 128, 256)
    s.set_volume(256, 256, 128, 1.0)
    assert s.all_defined()
    assert (s.numX(), s.numY(), s.numZ()) == (256, 256, 128)
    assert s.voxelHeight() == 1.0
    # offsets: the setters accept only positive values, as the reference
    assert s.offsetX(-1.0) is None and s.offsetX(2.0) == 2.0
    # a second model keeps its own parameters; copy_parameters copies
    t = PETLserver()
    assert not t.geometry_defined()
    assert t.copy_parameters(s.param_id)
    assert tuple(t.get_planogramSize(0)) == (65, 129, 128, 256)
    t.keep_only_planogram(0)
    with pytest.raises(ValueError):
        t.remove_planogram(3)
    t.clearAll()
    assert not t.geometry_defined() and not t.volume_defined()
    with pytest.raises(ValueError):
        t.add_planogram(0.0, -1.0, 1.0, 1.0, 1.0)


def test_set_default_volume_fills_fov():
    from petl_b200 import PETLserver
    s = PETLserver()
    s.add_planogram(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25)
    s.set_default_volume()
    # X from L, Y from R (half lengths 64 and 128) at the bin pitch
    assert (s.numX(), s.numY(), s.numZ()) == (64, 128, 64)
    assert s.voxelWidth() == 2.0


def test_host_elementwise_rules_match_reference():
    z = load_golden("cpu_rules.npz")
    from petl_b200 import PETLserver
    s = PETLserver()
    den = z["rd_den"].copy()
    s.rdivide(den, z["rd_num"].copy())
    assert np.array_equal(den, z["rd_out"])
    x = z["div_x"].copy()
    s.divide(x, z["div_y"].copy())
    assert np.array_equal(x, z["div_out"])
    r = z["recip_in"].copy()
    s.reciprocal(r, 7.0)
    assert np.array_equal(r, z["recip_out"])
    a, b = z["rd_num"][2].copy(), z["rd_den"][2].copy()
    assert s.inner_product(a, b) == np.float32(z["ip"])


def test_unsupported_reference_calls_fail_cleanly():
    L = lib()
    assert not L.voxelize(None, 1)
    assert not L.ray_trace(None, 1)
    assert L.clear_phantom()


def test_server_exposes_the_reference_methods():
    """Every public method of the reference PETLserver (src/petl_server.py)
    exists on the mirror class."""
    from petl_b200.server import PETLserver
    names = """about set_response clear_response create_new_model set_model volume_defined geometry_defined
    all_defined print_parameters numX numY numZ voxelWidth voxelHeight offsetX offsetY offsetZ get_numPlanograms
    get_planogramSize allocate_projections allocate_rebinned_projections copy_data copyData allocate_volume
    clearAll add_planogram remove_planogram keep_only_planogram set_default_volume set_volume calc_response
    apply_corrections floatstarstar bin simulate_scatter project backproject FBP PFDR add_object add_module
    clear_phantom clear_modules scale_phantom voxelize ray_trace stopping_power apply_solid_angle_correction
    apply_solid_angle_model save_data load_data display as_float_ptr inner_product_helper inner_product innerProd
    isAllZeros setToConstant setToZero setToOne sensitivity clip scale square subtract scalarAdd multiply divide
    rdivide reciprocal MLEM LS WLS RLS RWLS RWLSstepSize TVcost TVgradient TVquadForm diffuse TV_denoise
    relative_differences_grad gaussian_filter""".split()
    missing = [n for n in names if not callable(getattr(PETLserver, n, None))]
    assert not missing, missing


def test_petx_preset_model():
    """The PET/X preset (src/petx_server.py:4-42): two planograms with the
    reference's shapes, the default volume, 120 crystal blocks."""
    from petl_b200 import PETXserver
    s = PETXserver()
    assert s.get_numPlanograms() == 2
    assert [tuple(int(v) for v in s.get_planogramSize(i)) for i in range(2)] == [(63, 63, 96, 220),
                                                                                 (97, 167, 96, 244)]
    assert s.volume_defined()
    # solids are checked on the host: a bad one is refused, good ones accepted
    assert not s.add_object(9, [0, 0, 0], [1, 1, 1], 1.0)
    assert s.add_object("cone_y", [0, 0, 0], [1, 5, 3], 1.0)


def test_host_logic_of_the_response_and_phantom_calls():
    """Behaviour the reference's C ABI defines before any device work: null
    arguments are refused, the stopping power without a module model is 1
    everywhere (src/petl.cpp:139-147), solids are validated as
    geometricObject::init does, simulate_scatter validates and computes
    nothing (src/petl.cpp:194-202)."""
    import numpy as np
    from petl_b200.server import PETLserver, _pp
    s = PETLserver()
    L = s.libprojectors
    assert not L.set_solid_angle_correction(None, False)
    assert not L.apply_corrections(None, None, 0.75)
    assert not L.voxelize(None, 1)
    assert not L.ray_trace(None, 1)
    s.add_planogram(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)
    g = s.allocate_projections()
    for a in g:
        a[:] = 7.0
    assert L.stopping_power(_pp(g), 1)
    assert all(np.all(a == 1.0) for a in g)
    # the volume is not set: voxelize refuses, scatter refuses
    f = np.zeros((4, 4, 4), np.float32)
    assert not L.voxelize(f.ctypes.data_as(type(_pp([f])[0])), 1)
    c = np.zeros(3, np.float32)
    assert not s.add_object(8, c, c + 1, 1.0)
    assert s.add_object(0, c, c + 1, 1.0) and s.scale_phantom(2.0)
    assert not s.scale_phantom("x")
    try:
        s.simulate_scatter(g, f)
        raised = False
    except ValueError:
        raised = True
    assert raised
    s.set_volume(4, 4, 4, 1.0)
    assert s.simulate_scatter(g, f) is g
    s.clear_phantom()
    s.clear_modules()


def test_server_drops_a_request_past_its_deadline_before_admission():
    """Deadlines are host logic: a request whose deadline has passed when the
    worker looks at it fails without being admitted (no device work), and
    unknown requests cannot be cancelled."""
    from petl_b200 import PetlError
    from petl_b200.serving import ReconServer
    G = Geometry(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25, volume=(32, 32, 8, 2.0))
    g = np.zeros(G.shape, np.float32)
    with ReconServer(hbm_budget_gb=1, max_active=1) as srv:
        rid = srv.submit(G, g, 2, 1, deadline_s=0.0)
        with pytest.raises(PetlError, match="deadline exceeded before admission"):
            srv.wait(rid)
        with pytest.raises(PetlError, match="unknown request"):
            srv.cancel(12345)
        assert srv.stats()["failed"] == 1

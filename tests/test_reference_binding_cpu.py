"""The reference's own, unmodified Python binding (src/petl_server.py) driving
this library.

The binding finds its shared library with a glob for ``*petl*.so`` next to
the module (src/petl_server.py:21-45).  The test copies the binding file and
``petl_b200/libpetl.so`` into a temporary directory (nothing of the
reference is kept in this repository), stubs the ``imageio`` module it
imports for file I/O, and drives the calls that run without a GPU: the model
registry, geometry and volume set-up and queries, array allocation, the
host elementwise rules (against the reference's own outputs in
tests/golden/cpu_rules.npz) and the error behaviour of a compute call on a
machine without a device.  The GPU calls through the same binding are the
same C-ABI entry points that the GPU tests exercise through
``petl_b200.PETLserver``.  Skipped where the reference tree is absent.
"""
import importlib.util
import os
import shutil
import sys
import types

import numpy as np
import pytest

from conftest import ROOT, load_golden

REF_BINDING = os.path.join(os.environ.get("PETL_REFERENCE_DIR", "/root/reference"), "src", "petl_server.py")

pytestmark = pytest.mark.skipif(not os.path.isfile(REF_BINDING), reason="reference binding not present")


@pytest.fixture(scope="module")
def binding(tmp_path_factory):
    d = tmp_path_factory.mktemp("refbinding")
    shutil.copy(REF_BINDING, d / "petl_server.py")
    shutil.copy(os.path.join(ROOT, "petl_b200", "libpetl.so"), d / "libpetl.so")
    sys.modules.setdefault("imageio", types.ModuleType("imageio"))
    spec = importlib.util.spec_from_file_location("reference_petl_server", str(d / "petl_server.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod, str(d / "libpetl.so")


def test_binding_loads_this_library(binding):
    mod, path = binding
    s = mod.PETLserver()
    assert s.libprojectors is not None
    assert os.path.samefile(s.libprojectors._name, path)
    assert s.param_id >= 0


def test_geometry_through_the_reference_binding(binding):
    mod, _ = binding
    z = load_golden("cpu_rules.npz")
    s = mod.PETLserver()
    s.add_planogram(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25)
    s.add_planogram(0.0, 256.0, 128.0, 128.0, 1.0, 0.5, 0.25)
    assert s.get_numPlanograms() == 2
    shapes = [tuple(int(v) for v in s.get_planogramSize(n)) for n in range(2)]
    assert shapes == [(33, 65, 64, 128), (65, 129, 128, 256)]
    assert not s.volume_defined()
    s.set_volume(128, 128, 64, 2.0)
    assert s.all_defined()
    assert (s.numX(), s.numY(), s.numZ(), s.voxelWidth(), s.voxelHeight()) == (128, 128, 64, 2.0, 2.0)
    g = s.allocate_projections()
    assert [x.shape for x in g] == shapes and all(x.dtype == np.float32 for x in g)
    assert [x.shape for x in s.allocate_rebinned_projections()] == [sh[1:] for sh in shapes]
    assert s.allocate_volume().shape == (64, 128, 128)
    s.keep_only_planogram(1)
    assert s.get_numPlanograms() == 1
    assert tuple(int(v) for v in s.get_planogramSize(0)) == shapes[1]
    s.remove_planogram(0)
    assert s.get_numPlanograms() == 0
    with pytest.raises(ValueError):
        s.add_planogram(0.0, -1.0, 128.0, 128.0, 2.0, 0.5, 0.25)
    # the shapes the reference library gives for the same calls
    for k, call in enumerate(z["geom_calls"]):
        t = mod.PETLserver()
        psi, D, L, H, T, vm0, vm1 = (float(v) for v in call)
        t.add_planogram(psi, D, L, H, T, vm0, vm1)
        assert tuple(int(v) for v in t.get_planogramSize(0)) == tuple(int(v) for v in z["geom_shapes"][k])


def test_models_are_independent(binding):
    mod, _ = binding
    a = mod.PETLserver()
    b = mod.PETLserver()
    a.add_planogram(0.0, 256.0, 128.0, 128.0, 2.0, 0.5, 0.25)
    assert a.get_numPlanograms() == 1 and b.get_numPlanograms() == 0
    a.clearAll()
    assert a.get_numPlanograms() == 0


def test_host_elementwise_rules_through_the_reference_binding(binding):
    mod, _ = binding
    z = load_golden("cpu_rules.npz")
    s = mod.PETLserver()
    den = [z["rd_den"].copy()]  # 4-D arrays go in lists, as planograms do
    s.rdivide(den, [z["rd_num"].copy()])
    assert np.array_equal(den[0], z["rd_out"])
    x = z["div_x"].copy()
    s.divide(x, z["div_y"].copy())
    assert np.array_equal(x, z["div_out"])
    r = z["recip_in"].copy()
    s.reciprocal(r, 7.0)
    assert np.array_equal(r, z["recip_out"])
    a, b = z["rd_num"][2].copy(), z["rd_den"][2].copy()
    assert s.inner_product(a, b) == np.float32(z["ip"])


def test_compute_without_a_device_fails_as_the_reference_reports_it(binding):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    mod, _ = binding
    s = mod.PETLserver()
    s.add_planogram(0.0, 64.0, 32.0, 16.0, 2.0, 0.5, 0.25)
    s.set_volume(32, 32, 8, 2.0)
    g = s.allocate_projections()
    f = s.allocate_volume()
    with pytest.raises(TypeError):
        s.project(g, f)

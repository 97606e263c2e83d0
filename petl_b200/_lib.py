"""Loader for the in-tree CUDA library ``libpetl.so``.

The library must exist (``petl_b200.build.build()`` or
``__graft_entry__.build()``); there is no Python fallback for any compute
path, and importing an op without the library raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpetl.so")

_lib = None

c_f, c_i, c_b, c_d, c_ll, c_vp = (ctypes.c_float, ctypes.c_int, ctypes.c_bool, ctypes.c_double,
                                  ctypes.c_longlong, ctypes.c_void_p)
fp = ctypes.POINTER(ctypes.c_float)


class petl_geom(ctypes.Structure):
    """Mirror of ``petl_geom`` (include/petl_device.h)."""
    _fields_ = [(n, c_f) for n in ("psi", "R", "L", "H", "v_m0", "v_m1")] + \
               [(n, c_i) for n in ("N_v1", "N_v0", "N_u1", "N_u0")] + \
               [(n, c_f) for n in ("T_v1", "T_v0", "T_u1", "T_u0", "v1_0", "v0_0", "u1_0", "u0_0",
                                     "cos_psi", "sin_psi")] + \
               [(n, c_i) for n in ("numX", "numY", "numZ")] + \
               [(n, c_f) for n in ("T_x", "T_z", "x_0", "y_0", "z_0")]


class petl_solid(ctypes.Structure):
    """Mirror of ``petl_solid`` (include/petl_device.h)."""
    _fields_ = [("type", c_i), ("centers", c_f * 3), ("radii", c_f * 3), ("val", c_f), ("A", c_f * 9),
                ("clip", (c_f * 4) * 6), ("rotated", c_i), ("num_clip", c_i), ("clip_cone", c_f * 2),
                ("given_c", c_f * 3), ("given_r", c_f * 3)]


# (name, restype, argtypes) of every exported function
_REF_API = [
    ("set_model", c_b, [c_i]), ("create_new_model", c_i, []), ("about", None, []),
    ("copy_parameters", c_b, [c_i]), ("clearAll", None, []), ("print_parameters", None, []),
    ("volume_defined", c_b, []), ("geometry_defined", c_b, []),
    ("get_numX", c_i, []), ("set_numX", c_b, [c_i]), ("get_numY", c_i, []), ("set_numY", c_b, [c_i]),
    ("get_numZ", c_i, []), ("set_numZ", c_b, [c_i]),
    ("get_voxelWidth", c_f, []), ("set_voxelWidth", c_b, [c_f]),
    ("get_voxelHeight", c_f, []), ("set_voxelHeight", c_b, [c_f]),
    ("get_offsetX", c_f, []), ("set_offsetX", c_b, [c_f]), ("get_offsetY", c_f, []), ("set_offsetY", c_b, [c_f]),
    ("get_offsetZ", c_f, []), ("set_offsetZ", c_b, [c_f]),
    ("get_numPlanograms", c_i, []), ("get_planogramSize", c_b, [c_i, ctypes.POINTER(c_i)]),
    ("add_planogram", c_b, [c_f] * 7), ("remove_planogram", c_b, [c_i]), ("keep_only_planogram", c_b, [c_i]),
    ("set_default_volume", c_b, [c_f]), ("set_volume", c_b, [c_i, c_i, c_i, c_f, c_f, c_f, c_f, c_f]),
    ("bin", c_b, [ctypes.POINTER(fp), ctypes.c_char_p]), ("simulate_scatter", c_b, [ctypes.POINTER(fp), fp]),
    ("project", c_b, [ctypes.POINTER(fp), fp]), ("backproject", c_b, [ctypes.POINTER(fp), fp]),
    ("FBP", c_b, [ctypes.POINTER(fp), fp]), ("PFDR", c_b, [ctypes.POINTER(fp), ctypes.POINTER(fp)]),
    ("add_object", c_b, [c_i, fp, fp, c_f, fp, fp]), ("add_module", c_b, [c_i, fp, fp, c_f, fp, fp]),
    ("clear_phantom", c_b, []), ("clear_modules", c_b, []), ("scale_phantom", c_b, [c_f, c_f, c_f]),
    ("voxelize", c_b, [fp, c_i]), ("ray_trace", c_b, [ctypes.POINTER(fp), c_i]),
    ("stopping_power", c_b, [ctypes.POINTER(fp), c_i]),
    ("set_solid_angle_correction", c_b, [ctypes.POINTER(fp), c_b]),
    ("apply_corrections", c_b, [ctypes.POINTER(fp), ctypes.POINTER(fp), c_f]),
    ("multiply3D", c_b, [fp, fp, c_i, c_i, c_i]), ("multiply4D", c_b, [fp, fp, c_i, c_i, c_i, c_i]),
    ("divide3D", c_b, [fp, fp, c_i, c_i, c_i]), ("divide4D", c_b, [fp, fp, c_i, c_i, c_i, c_i]),
    ("rdivide3D", c_b, [fp, fp, c_i, c_i, c_i]), ("rdivide4D", c_b, [fp, fp, c_i, c_i, c_i, c_i]),
    ("reciprocal3D", c_b, [fp, c_i, c_i, c_i, c_f]), ("reciprocal4D", c_b, [fp, c_i, c_i, c_i, c_i, c_f]),
    ("inner_product3D", c_f, [fp, fp, fp, c_i, c_i, c_i]),
    ("inner_product4D", c_f, [fp, fp, fp, c_i, c_i, c_i, c_i]),
    ("TV_cost", c_f, [c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]),
    ("TV_gradient", c_b, [c_vp, c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]),
    ("TV_quadForm", c_f, [c_vp, c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_b]),
    ("diffuse", c_b, [c_vp, c_i, c_i, c_i, c_f, c_f, c_i, c_b]),
    ("TV_denoise", c_b, [c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_i, c_b, c_b]),
    ("relativeDifferences_gradient", c_b, [fp, fp, c_i, c_i, c_i, c_f, c_f]),
    ("gaussian_filter", c_b, [fp, c_i, c_i, c_i, c_f, c_i]),
]

_G = ctypes.POINTER(petl_geom)
_DEV_API = [
    ("petl_last_error", ctypes.c_char_p, []), ("petl_version", c_i, []),
    ("petl_launch_count", ctypes.c_ulonglong, []),
    ("petl_geom_init", c_i, [_G, c_f, c_f, c_f, c_f, c_f, c_f, c_f]),
    ("petl_geom_set_volume", c_i, [_G, c_i, c_i, c_i, c_f, c_f, c_f, c_f, c_f]),
    ("petl_optimal_fft_size", c_i, [c_i]),
    ("petl_model_geometry", c_i, [c_i, _G]),
    ("petl_model_solids", c_i, [c_i, ctypes.POINTER(petl_solid), c_i]),
    ("petl_copy_to_host", c_i, [c_vp, c_vp, c_ll, c_vp]), ("petl_copy_to_device", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_set_dispatch", c_i, [c_i]),
    ("petl_device_error_flag", c_i, []),
    ("petl_force_wait_timeout", c_i, [c_i]),
    ("petl_inject_alloc_failure", c_i, [ctypes.c_longlong]),
    ("petl_scratch_alloc_count", ctypes.c_longlong, []),
    ("petl_scratch_in_use", ctypes.c_longlong, []),
    ("petl_last_projector_path", c_i, []),
    ("petl_project_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_vp]),
    ("petl_project_range_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_project_noalloc_dev", c_i, [_G, c_vp, c_vp, c_vp]),
    ("petl_backproject_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_f, c_i, c_i, c_vp]),
    ("petl_backproject_range_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_f, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_project_ratio_dev", c_i, [_G, c_vp, c_vp, c_vp, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_project_nnz_dev", c_i, [_G, ctypes.POINTER(c_d), c_vp]),
    ("petl_bin_events_dev", c_i, [_G, c_vp, c_vp, c_ll, c_vp, c_i, c_i, c_vp]),
    ("petl_solid_angle_dev", c_i, [_G, c_vp, c_i, c_vp]),
    ("petl_solid_init", c_i, [ctypes.POINTER(petl_solid), c_i, fp, fp, c_f, fp, fp]),
    ("petl_solids_scale", None, [ctypes.POINTER(petl_solid), c_i, c_f, c_f, c_f]),
    ("petl_voxelize_dev", c_i, [ctypes.POINTER(petl_solid), c_i, c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_f, c_f,
                                c_i, c_vp]),
    ("petl_ray_trace_dev", c_i, [_G, ctypes.POINTER(petl_solid), c_i, c_vp, c_i, c_i, c_vp]),
    ("petl_apply_corrections_dev", c_i, [_G, c_vp, c_vp, c_f, c_vp]),
    ("petl_project_bf16_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_project_ratio_bf16_dev", c_i, [_G, c_vp, c_vp, c_vp, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_backproject_bf16_dev", c_i, [_G, c_vp, c_vp, c_i, c_i, c_f, c_i, c_i, c_i, c_i, c_vp]),
    ("petl_mlem_update_bf16_dev", c_i, [c_vp, c_vp, c_vp, c_ll, c_vp]),
    ("petl_to_bf16_dev", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_server_create", c_vp, [c_d, c_i, c_i, c_i]),
    ("petl_server_submit", c_i, [c_vp, _G, c_vp, c_i, c_i, ctypes.POINTER(c_ll)]),
    ("petl_server_submit_deadline", c_i, [c_vp, _G, c_vp, c_i, c_i, c_d, ctypes.POINTER(c_ll)]),
    ("petl_server_cancel", c_i, [c_vp, c_ll]),
    ("petl_server_wait", c_i, [c_vp, c_ll, c_vp, ctypes.POINTER(c_d), ctypes.POINTER(c_d)]),
    ("petl_server_stats", c_i, [c_vp, ctypes.POINTER(c_d)]),
    ("petl_server_set_batching", c_i, [c_vp, c_i]),
    ("petl_server_batch_stats", c_i, [c_vp, ctypes.POINTER(c_d)]),
    ("petl_server_destroy", None, [c_vp]),
    ("petl_pfdr_dev", c_i, [_G, c_vp, c_vp, c_vp]),
    ("petl_ramp_dev", c_i, [_G, c_vp, c_i, c_vp]),
    ("petl_fbp_dev", c_i, [_G, c_vp, c_vp, c_i, c_vp]),
    ("petl_rd_gradient_dev", c_i, [c_vp, c_vp, c_i, c_i, c_i, c_f, c_f, c_vp]),
    ("petl_rd_cost_dev", c_i, [c_vp, c_i, c_i, c_i, c_f, c_f, c_vp, c_vp]),
    ("petl_tv_gradient_dev", c_i, [c_vp, c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_i, c_vp]),
    ("petl_tv_cost_dev", c_i, [c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_i, c_vp, c_vp]),
    ("petl_tv_quadform_dev", c_i, [c_vp, c_vp, c_i, c_i, c_i, c_f, c_f, c_f, c_i, c_vp, c_vp]),
    ("petl_gaussian_filter_dev", c_i, [c_vp, c_i, c_i, c_i, c_f, c_i, c_vp]),
    ("petl_rdivide_dev", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_divide_dev", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_multiply_dev", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_reciprocal_dev", c_i, [c_vp, c_ll, c_f, c_vp]),
    ("petl_dot_dev", c_i, [c_vp, c_vp, c_vp, c_ll, c_vp, c_vp]),
    ("petl_loglik_dev", c_i, [c_vp, c_vp, c_ll, c_vp, c_vp]),
    ("petl_axpby_dev", c_i, [c_vp, c_vp, c_f, c_f, c_ll, c_vp]),
    ("petl_poisson_grad_dev", c_i, [c_vp, c_vp, c_ll, c_vp]),
    ("petl_mlem_update_dev", c_i, [c_vp, c_vp, c_vp, c_ll, c_vp]),
    ("petl_osl_update_dev", c_i, [c_vp, c_vp, c_vp, c_vp, c_ll, c_vp]),
]

API = _REF_API + _DEV_API


class PetlError(RuntimeError):
    pass


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PetlError(f"libpetl.so not found at {LIB_PATH}: build it with petl_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in API:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, what=""):
    if rc != 0:
        msg = lib().petl_last_error()
        raise PetlError(f"{what}: {msg.decode() if msg else 'error ' + str(rc)}")

"""ctypes mirror of include/cudaem_b200.h (structs, enums, function prototypes)."""
from __future__ import annotations

import ctypes as C

MS_NR = 128
MS_MAX_DET = 8
MS_MAX_COEF = 6

# ms_status
MS_OK = 0
MS_ERR_INVALID_ARG = 1
MS_ERR_UNSUPPORTED = 2
MS_ERR_CUDA = 3
MS_ERR_OUT_OF_MEMORY = 4
MS_ERR_TIMEOUT = 5
MS_ERR_NO_DEVICE = 6
MS_ERR_INTERNAL = 7
STATUS_NAMES = {0: "MS_OK", 1: "MS_ERR_INVALID_ARG", 2: "MS_ERR_UNSUPPORTED", 3: "MS_ERR_CUDA",
                4: "MS_ERR_OUT_OF_MEMORY", 5: "MS_ERR_TIMEOUT", 6: "MS_ERR_NO_DEVICE", 7: "MS_ERR_INTERNAL"}

MS_SIM_HRTEM, MS_SIM_ED, MS_SIM_CBED, MS_SIM_STEM = 1, 2, 3, 4
MS_PHONON_STILL, MS_PHONON_FROZEN = 1, 3
MS_IW_PLANE, MS_IW_CONVERGENT, MS_IW_PLANE_TILTED = 1, 2, 3
(MS_POT_DOYLE_0_4, MS_POT_PENG_0_4, MS_POT_PENG_0_12, MS_POT_KIRKLAND_0_12, MS_POT_WEICKENMEIER_0_12,
 MS_POT_LOBATO_0_12, MS_POT_MOLIERE) = range(1, 8)
MS_ILLUM_COHERENT, MS_ILLUM_PARTIAL, MS_ILLUM_TCC = 1, 2, 3
MS_TSI_TEMPORAL_SPATIAL, MS_TSI_TEMPORAL, MS_TSI_SPATIAL, MS_TSI_COHERENT = 1, 2, 3, 4
MS_RECORD_INTENSITY, MS_RECORD_WAVE = 0, 1
MS_EXEC_BATCHED, MS_EXEC_PLAIN, MS_EXEC_GENERAL = 0, 1, 2
MS_BORDER_MIN, MS_BORDER_MAX, MS_BORDER_MIDDLE = 0, 1, 2
MS_INJECT_NONE, MS_INJECT_WAIT_TIMEOUT, MS_INJECT_ALLOC_FAIL = 0, 1, 2


class ms_lens(C.Structure):
    _fields_ = [("m", C.c_int)] + [(n, C.c_double) for n in (
        "c10", "c12", "phi12", "c21", "phi21", "c23", "phi23",
        "c30", "c32", "phi32", "c34", "phi34",
        "c41", "phi41", "c43", "phi43", "c45", "phi45",
        "c50", "c52", "phi52", "c54", "phi54", "c56", "phi56",
        "inner_aper_ang", "outer_aper_ang", "dsf_sigma", "ssf_beta")] + [
        ("dsf_npoints", C.c_int), ("ssf_npoints", C.c_int)]


class ms_element_coef(C.Structure):
    _fields_ = [("Z", C.c_int), ("form", C.c_int), ("cl", C.c_double * MS_MAX_COEF),
                ("cnl", C.c_double * MS_MAX_COEF)]


class ms_atoms(C.Structure):
    _fields_ = [("n", C.c_int64), ("Z", C.POINTER(C.c_int)), ("x", C.POINTER(C.c_float)),
                ("y", C.POINTER(C.c_float)), ("z", C.POINTER(C.c_float)), ("sigma", C.POINTER(C.c_float)),
                ("occ", C.POINTER(C.c_float))]


class ms_params(C.Structure):
    _fields_ = [
        ("simulation_type", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int),
        ("lx", C.c_double), ("ly", C.c_double),
        ("dz", C.c_double),
        ("bwl", C.c_int),
        ("E0", C.c_double),
        ("theta", C.c_double), ("phi", C.c_double),
        ("potential_type", C.c_int),
        ("pot_rmin", C.c_double), ("pot_rmax", C.c_double),
        ("pot_wrap", C.c_int),
        ("element_coefs", C.POINTER(ms_element_coef)),
        ("n_element_coefs", C.c_int),
        ("phonon_model", C.c_int),
        ("pn_nconf", C.c_int),
        ("pn_seed", C.c_uint64),
        ("pn_dim_x", C.c_int), ("pn_dim_y", C.c_int), ("pn_dim_z", C.c_int),
        ("slice_border", C.c_int),
        ("iw_type", C.c_int),
        ("iw_x", C.c_double), ("iw_y", C.c_double),
        ("cond_lens", ms_lens),
        ("obj_lens", ms_lens),
        ("illumination_model", C.c_int),
        ("temporal_spatial_incoh", C.c_int),
        ("data_record", C.c_int),
        ("scan_nx", C.c_int), ("scan_ny", C.c_int),
        ("scan_x0", C.c_double), ("scan_y0", C.c_double),
        ("scan_dx", C.c_double), ("scan_dy", C.c_double),
        ("n_det", C.c_int),
        ("det_inner", C.c_double * MS_MAX_DET),
        ("det_outer", C.c_double * MS_MAX_DET),
        ("thick_det", C.c_int),
        ("exec_mode", C.c_int),
        ("probe_batch", C.c_int),
        ("ckpt_interval", C.c_int),
        ("enable_fine_slicing", C.c_int),
        ("gpu_num", C.c_int),
    ]


class ms_output(C.Structure):
    _fields_ = [
        ("image_intensity", C.POINTER(C.c_float)),
        ("image_real", C.POINTER(C.c_float)),
        ("image_imag", C.POINTER(C.c_float)),
        ("stem_intensity", C.POINTER(C.c_float)),
        ("thickness_frames", C.POINTER(C.c_float)),
        ("thickness_capacity", C.c_int64),
        ("on_device", C.c_int),
        ("row", C.c_int), ("col", C.c_int),
        ("n_slices", C.c_int),
        ("interval_x", C.c_double), ("interval_y", C.c_double),
        ("total_intensity", C.c_double),
    ]


_P = C.POINTER
# name -> (restype, argtypes); every symbol include/cudaem_b200.h declares
PROTOTYPES = {
    "ms_version": (C.c_char_p, []),
    "ms_abi_version": (C.c_int, []),
    "ms_default_params": (None, [_P(ms_params)]),
    "ms_validate_params": (C.c_int, [_P(ms_params)]),
    "ms_create": (C.c_int, [_P(C.c_void_p), C.c_int]),
    "ms_destroy": (C.c_int, [C.c_void_p]),
    "ms_last_error": (C.c_char_p, [C.c_void_p]),
    "ms_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ms_get_stream": (C.c_void_p, [C.c_void_p]),
    "ms_last_device_ms": (C.c_double, [C.c_void_p]),
    "ms_last_launch_count": (C.c_int64, [C.c_void_p]),
    "ms_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_profile_reset": (C.c_int, [C.c_void_p]),
    "ms_profile_get": (C.c_int, [C.c_void_p, C.c_char_p, _P(C.c_int64), _P(C.c_double)]),
    "ms_physics": (C.c_int, [C.c_double, _P(C.c_double), _P(C.c_double), _P(C.c_double)]),
    "ms_set_fault_injection": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_simulate_tem": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), _P(ms_output)]),
    "ms_simulate_tem_defocus_series": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), C.c_int,
                                                 _P(C.c_double), _P(ms_output)]),
    "ms_simulate_cbed": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), _P(ms_output)]),
    "ms_simulate_stem": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), _P(ms_output)]),
    "ms_simulate_thickness": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), _P(ms_output)]),
    "ms_displace_atoms": (C.c_int, [_P(ms_params), _P(ms_atoms), C.c_int, _P(C.c_float), _P(C.c_float),
                                    _P(C.c_float)]),
    "ms_build_slices": (C.c_int, [_P(ms_params), _P(ms_atoms), C.c_int, _P(C.c_int), _P(C.c_float), C.c_int,
                                  _P(C.c_int)]),
    "ms_build_crystal": (C.c_int, [C.c_int, _P(C.c_int), _P(C.c_double), C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _P(C.c_int64), _P(C.c_int),
                                   _P(C.c_float), _P(C.c_float), _P(C.c_float), _P(C.c_float), _P(C.c_float)]),
    "ms_projected_potential": (C.c_int, [C.c_void_p, _P(ms_params), _P(ms_atoms), C.c_int, _P(C.c_float),
                                         C.c_int64, C.c_int, _P(C.c_int)]),
    "ms_stem_forward_potential": (C.c_int, [C.c_void_p, _P(ms_params), _P(C.c_float), C.c_int, C.c_int,
                                            C.c_double, _P(C.c_double), C.c_int, _P(C.c_float)]),
    "ms_stem_forward_potential_noalloc": (C.c_int, [C.c_void_p, _P(ms_params), C.c_void_p, C.c_int, C.c_double,
                                                    _P(C.c_double), C.c_int, C.c_void_p]),
    "ms_stem_backward": (C.c_int, [C.c_void_p, _P(ms_params), _P(C.c_float), C.c_int, C.c_int, C.c_double,
                                   _P(C.c_double), C.c_int, _P(C.c_float), _P(C.c_double), _P(C.c_float),
                                   _P(C.c_double), _P(C.c_double)]),
    "ms_last_probe_batch": (C.c_int, [C.c_void_p]),
    "ms_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_set_pass_kernels": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_set_tile_shape": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_set_transmission_store": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_last_tile_shape": (C.c_int, [C.c_void_p]),
    "ms_set_tune_cache": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ms_set_potential_overlap": (C.c_int, [C.c_void_p, C.c_int]),
    "ms_simulate_many": (C.c_int, [C.c_void_p, C.c_int, _P(ms_params), _P(ms_atoms), _P(ms_output),
                                   _P(C.c_double)]),
}


def bind(lib: C.CDLL) -> C.CDLL:
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib

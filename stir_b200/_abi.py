"""ctypes mirror of include/stir_b200.h and the loader of the CUDA library.

The library is built in-tree (stir_b200/libstir_b200.so) by __graft_entry__.build()
or ``make -C stir_b200/csrc``.  Loading fails loudly if it is missing: there is no
CPU fallback for the projector pair.
"""
from __future__ import annotations

import ctypes
import os

MAX_SEGMENTS = 255

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_OUT_OF_MEMORY = -4
ERR_STATE = -5
ERR_TIMEOUT = -6
ERR_TOO_LARGE = -7

BACKPROJECT_ATOMIC = 0
BACKPROJECT_DETERMINISTIC = 1
BATCH_KERNELS_AUTO = 0
BATCH_KERNELS_PATHS = 1
BATCH_KERNELS_TOF_GROUPED = 2
BATCH_KERNELS_PACKED = 3
BATCH_KERNELS_BASIC_BINS = 4
STATUS_STAGING_TIMEOUT = 1  # b200rt_get_device_status: a forward staging copy's wait ran out

ATTENUATION_FACTORS = 0
ATTENUATION_APPLY = 1
ATTENUATION_UNDO = 2
PRIOR_NONE = 0
PRIOR_QUADRATIC = 1
PRIOR_RELATIVE_DIFFERENCE = 2

MAP_ADDITIVE = 0
MAP_MULTIPLICATIVE = 1

LISTMODE_AUTO = 0
LISTMODE_PER_EVENT = 1
LISTMODE_BINNED = 2


class Geometry(ctypes.Structure):
    """b200rt_geometry"""

    _fields_ = [
        ("num_rings", ctypes.c_int32),
        ("num_detectors_per_ring", ctypes.c_int32),
        ("inner_ring_radius_mm", ctypes.c_float),
        ("average_depth_of_interaction_mm", ctypes.c_float),
        ("ring_spacing_mm", ctypes.c_float),
        ("default_bin_size_mm", ctypes.c_float),
        ("intrinsic_azimuthal_tilt_rad", ctypes.c_float),
        ("timing_resolution_ps", ctypes.c_float),
        ("size_of_timing_pos_ps", ctypes.c_float),
        ("max_num_timing_poss", ctypes.c_int32),
        ("arc_corrected", ctypes.c_int32),
        ("arccorr_bin_size_mm", ctypes.c_float),
        ("num_views", ctypes.c_int32),
        ("num_tangential_poss", ctypes.c_int32),
        ("max_segment_num", ctypes.c_int32),
        ("tof_mash_factor", ctypes.c_int32),
        ("min_ring_diff", ctypes.c_int32 * MAX_SEGMENTS),
        ("max_ring_diff", ctypes.c_int32 * MAX_SEGMENTS),
        ("num_axial_poss", ctypes.c_int32 * MAX_SEGMENTS),
        ("nz", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("min_z", ctypes.c_int32),
        ("min_y", ctypes.c_int32),
        ("min_x", ctypes.c_int32),
        ("voxel_size_z", ctypes.c_float),
        ("voxel_size_y", ctypes.c_float),
        ("voxel_size_x", ctypes.c_float),
        ("origin_z", ctypes.c_float),
        ("origin_y", ctypes.c_float),
        ("origin_x", ctypes.c_float),
        ("num_tangential_LORs", ctypes.c_int32),
        ("restrict_to_cylindrical_FOV", ctypes.c_int32),
        ("do_symmetry_90degrees_min_phi", ctypes.c_int32),
        ("do_symmetry_180degrees_min_phi", ctypes.c_int32),
        ("do_symmetry_swap_segment", ctypes.c_int32),
        ("do_symmetry_swap_s", ctypes.c_int32),
        ("do_symmetry_shift_z", ctypes.c_int32),
        ("tof_kernel_truncation_sigmas", ctypes.c_float),
    ]


class Info(ctypes.Structure):
    """b200rt_info"""

    _fields_ = [
        ("num_bins", ctypes.c_int64),
        ("num_image_voxels", ctypes.c_int64),
        ("num_basic_bins", ctypes.c_int64),
        ("num_row_elements", ctypes.c_int64),
        ("total_nnz", ctypes.c_int64),
        ("num_tof_bins", ctypes.c_int32),
        ("num_basic_views", ctypes.c_int32),
        ("symmetries_used", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class Prior(ctypes.Structure):
    """b200rt_prior"""

    _fields_ = [
        ("type", ctypes.c_int32),
        ("penalisation_factor", ctypes.c_float),
        ("gamma", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("only_2D", ctypes.c_int32),
        ("map_model", ctypes.c_int32),
        ("kappa_dev", ctypes.c_void_p),
    ]


class BatchConfig(ctypes.Structure):
    """b200rt_batch_config"""

    _fields_ = [
        ("ctas_per_sm_forward", ctypes.c_int32),
        ("ctas_per_sm_back", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("kernels", ctypes.c_int32),
    ]


NORM_FACTORS = 0
NORM_APPLY = 1
NORM_UNDO = 2
NORM_PROJDATA = 1
NORM_ATTENUATION = 2


class NormTerm(ctypes.Structure):
    """b200rt_norm_term"""

    _fields_ = [
        ("kind", ctypes.c_int32),
        ("non_tof", ctypes.c_int32),
        ("data_dev", ctypes.c_void_p),
    ]


class LmEvent(ctypes.Structure):
    """b200rt_lm_event"""

    _fields_ = [
        ("segment", ctypes.c_int32),
        ("view", ctypes.c_int32),
        ("axial_pos", ctypes.c_int32),
        ("tangential_pos", ctypes.c_int32),
        ("timing_pos", ctypes.c_int32),
        ("value", ctypes.c_float),
        ("corr", ctypes.c_float),
    ]


STORAGE_SEGMENT_VIEW_AXIAL_TANG = 0
STORAGE_SEGMENT_AXIAL_VIEW_TANG = 1
NUMBER_TYPES = {"schar": 0, "uchar": 1, "short": 2, "ushort": 3, "int": 4, "uint": 5, "float": 6, "double": 7}


class StreamFormat(ctypes.Structure):
    """b200rt_stream_format"""

    _fields_ = [
        ("storage_order", ctypes.c_int32),
        ("number_type", ctypes.c_int32),
        ("swap_bytes", ctypes.c_int32),
        ("scale_factor", ctypes.c_float),
        ("num_segments", ctypes.c_int32),
        ("segment_sequence", ctypes.POINTER(ctypes.c_int32)),
        ("num_axial_poss", ctypes.POINTER(ctypes.c_int32)),
        ("num_timing_poss", ctypes.c_int32),
        ("timing_poss_sequence", ctypes.POINTER(ctypes.c_int32)),
    ]


GIBBS_QUADRATIC = 1
GIBBS_RELATIVE_DIFFERENCE = 2
GIBBS_ARITH_HOST = 0
GIBBS_ARITH_CUDA = 1
LAYOUT_DEVICE = 0  # [y][x][z]
LAYOUT_STIR = 1    # [z][y][x]


class GibbsParams(ctypes.Structure):
    """b200rt_gibbs_params"""

    _fields_ = [
        ("potential", ctypes.c_int32),
        ("penalisation_factor", ctypes.c_float),
        ("gamma", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("nz", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("layout", ctypes.c_int32),
        ("voxel_size_z", ctypes.c_float),
        ("voxel_size_y", ctypes.c_float),
        ("voxel_size_x", ctypes.c_float),
        ("only_2D", ctypes.c_int32),
        ("weights_z", ctypes.c_int32),
        ("weights_y", ctypes.c_int32),
        ("weights_x", ctypes.c_int32),
        ("weights", ctypes.c_void_p),
        ("kappa_dev", ctypes.c_void_p),
    ]


_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libstir_b200.so")

# (name, restype, argtypes) of every entry point declared in include/stir_b200.h
_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
EXPORTS = [
    ("b200rt_create", _I, [ctypes.POINTER(Geometry), _I, ctypes.POINTER(_P)]),
    ("b200rt_destroy", None, [_P]),
    ("b200rt_last_error", ctypes.c_char_p, [_P]),
    ("b200rt_get_info", _I, [_P, ctypes.POINTER(Info)]),
    ("b200rt_projdata_size", _I64, [_P]),
    ("b200rt_image_size", _I64, [_P]),
    ("b200rt_get_row", _I, [_P, _I, _I, _I, _I, _I, _P, _P, _I64, ctypes.POINTER(_I64)]),
    ("b200rt_image_to_device_layout", _I, [_P, _P, _P, _P]),
    ("b200rt_image_from_device_layout", _I, [_P, _P, _P, _P]),
    ("b200rt_projdata_to_device_layout", _I, [_P, _P, _P, _P]),
    ("b200rt_projdata_from_device_layout", _I, [_P, _P, _P, _P]),
    ("b200rt_get_viewgram", _I, [_P, _P, _I, _I, _I, _P, _P]),
    ("b200rt_set_viewgram", _I, [_P, _P, _I, _I, _I, _P, _I, _P]),
    ("b200rt_forward_project_dev", _I, [_P, _P, _P, _I, _I, _P]),
    ("b200rt_back_project_dev", _I, [_P, _P, _P, _I, _I, _I, _P]),
    ("b200rt_sensitivity_dev", _I, [_P, _P, _P, _I, _I, _I, _I, _P]),
    ("b200rt_osmaposl_subiteration_dev", _I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(Prior), ctypes.c_float,
                                              ctypes.c_float, _I, _P, _P]),
    ("b200rt_osmaposl_numerator_dev", _I, [_P, _P, _P, _P, _I, _I, _I, _I, _P, _P]),
    ("b200rt_osmaposl_apply_update_dev", _I, [_P, _P, _P, _P, _I, _I, ctypes.POINTER(Prior), ctypes.c_float, ctypes.c_float,
                                              _P]),
    ("b200rt_get_num_cancelled", _I, [_P, ctypes.POINTER(_I64)]),
    ("b200rt_get_device_status", _I, [_P, ctypes.POINTER(ctypes.c_uint32), _I]),
    ("b200rt_log_likelihood_dev", _I, [_P, _P, _P, _P, _P, _I, _I, _I, ctypes.POINTER(ctypes.c_double), _P]),
    ("b200rt_log_likelihood_gradient_dev", _I, [_P, _P, _P, _P, _P, _I, _I, _I, _I, _P, _P]),
    ("b200rt_prior_value_dev", _I, [_P, ctypes.POINTER(Prior), _P, ctypes.POINTER(ctypes.c_double), _P]),
    ("b200rt_log_likelihood_dev_noalloc", _I, [_P, _P, _P, _P, _P, _I, _I, _I, _P, _P]),
    ("b200rt_prior_gradient_dev", _I, [_P, ctypes.POINTER(Prior), _P, _P, _P]),
    ("b200rt_forward_project", _I, [_P, _P, _P, _I, _I]),
    ("b200rt_back_project", _I, [_P, _P, _P, _I, _I, _I]),
    ("b200rt_attenuation_dev", _I, [_P, _P, _P, _I, _P]),
    ("b200rt_prior_hessian_times_input_dev", _I, [_P, ctypes.POINTER(Prior), _P, _P, _P, _P]),
    ("b200rt_ossps_denominator_dev", _I, [_P, _P, _P, _P, _I, _P]),
    ("b200rt_ossps_subiteration_dev", _I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, ctypes.POINTER(Prior),
                                           ctypes.c_float, ctypes.c_float, ctypes.c_float, _I, _P]),
    ("b200rt_batch_create", _I, [_I, ctypes.POINTER(_P)]),
    ("b200rt_batch_destroy", None, [_P]),
    ("b200rt_batch_last_error", ctypes.c_char_p, [_P]),
    ("b200rt_batch_set_frame_mode", _I, [_P, _I, _I]),
    ("b200rt_batch_add_frame", _I, [_P, _P, _P, _P, _P, ctypes.POINTER(_P), _I, _I, _I, _I, ctypes.POINTER(Prior),
                                    ctypes.c_float, ctypes.c_float, ctypes.POINTER(_I)]),
    ("b200rt_batch_num_frames", _I, [_P]),
    ("b200rt_batch_run", _I, [_P, _I, _I, _I, _P]),
    ("b200rt_batch_autotune", _I, [_P, _I, ctypes.POINTER(BatchConfig)]),
    ("b200rt_batch_set_config", _I, [_P, ctypes.POINTER(BatchConfig)]),
    ("b200rt_batch_get_config", _I, [_P, ctypes.POINTER(BatchConfig)]),
    ("b200rt_batch_get_num_cancelled", _I, [_P, _I, ctypes.POINTER(_I64)]),
    ("b200rt_normalisation_dev", _I, [_P, ctypes.POINTER(NormTerm), _I, _I, _P, _P]),
    ("b200rt_listmode_gradient_dev", _I, [_P, _P, _I64, _P, _I, _I, _I, _P, _I, _P, _P]),
    ("b200rt_listmode_value_dev", _I, [_P, _P, _I64, _P, _I, _I, _I, ctypes.POINTER(ctypes.c_double), _P]),
    ("b200rt_listmode_hessian_times_input_dev", _I, [_P, _P, _I64, _P, _P, _I, _I, _I, _P, _P]),
    ("b200rt_listmode_num_invalid", _I, [_P, ctypes.POINTER(_I64)]),
    ("b200rt_listmode_set_method", _I, [_P, _I]),
    ("b200rt_stream_bytes", _I, [_P, ctypes.POINTER(StreamFormat), ctypes.POINTER(_I64)]),
    ("b200rt_projdata_from_stream_dev", _I, [_P, _P, _I64, ctypes.POINTER(StreamFormat), _P, _P]),
    ("b200rt_projdata_to_stream_dev", _I, [_P, _P, ctypes.POINTER(StreamFormat), _P, _I64, _P]),
    ("b200rt_gibbs_create", _I, [ctypes.POINTER(GibbsParams), _I, ctypes.POINTER(_P)]),
    ("b200rt_gibbs_destroy", None, [_P]),
    ("b200rt_set_view_shard", _I, [_P, _P, _I]),
    ("b200rt_forward_project_batch_dev", _I, [_P, _P, _I64, _P, _I64, _I, _I, _I, _P]),
    ("b200rt_back_project_batch_dev", _I, [_P, _P, _I64, _P, _I64, _I, _I, _I, _I, _P]),
    ("b200rt_log_likelihood_batch_dev", _I, [_P, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _I, _I, _I, _I, _P, _P]),
    ("b200rt_log_likelihood_and_ratio_batch_dev", _I, [_P, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _I, _I, _I, _I,
                                                    ctypes.POINTER(ctypes.c_double), _P, _I64, _P]),
    ("b200rt_log_likelihood_gradient_batch_dev", _I, [_P, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _I, _I, _I, _I, _I,
                                                     _P, _I64, _P]),
    ("b200rt_gibbs_last_error", ctypes.c_char_p, [_P]),
    ("b200rt_gibbs_set_arithmetic", _I, [_P, _I]),
    ("b200rt_gibbs_get_weights", _I, [_P, _P, ctypes.POINTER(ctypes.c_int32)]),
    ("b200rt_gibbs_set_kappa", _I, [_P, _P]),
    ("b200rt_gibbs_value_dev", _I, [_P, _P, ctypes.POINTER(ctypes.c_double), _P]),
    ("b200rt_gibbs_gradient_dev", _I, [_P, _P, _P, _P]),
    ("b200rt_gibbs_gradient_times_input_dev", _I, [_P, _P, _P, ctypes.POINTER(ctypes.c_double), _P]),
    ("b200rt_gibbs_hessian_diagonal_dev", _I, [_P, _P, _P, _P]),
    ("b200rt_gibbs_accumulate_hessian_times_input_dev", _I, [_P, _P, _P, _P, _P]),
    ("b200rt_gibbs_hessian_dev", _I, [_P, _P, _I, _I, _I, _P, _P]),
]

_lib = None


def load_library(path: str | None = None):
    """Load libstir_b200.so and bind every exported entry point.  Raises if missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIBRARY_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"stir_b200: CUDA library {p} not built; run `python -c 'import __graft_entry__ as g; g.build()'` "
            "or `make -C stir_b200/csrc` (there is no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, res, args in EXPORTS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class B200Error(RuntimeError):
    pass


def check(status: int, handle=None, what: str = "", batch=None, gibbs=None):
    if status != OK:
        lib = load_library()
        if gibbs is not None:
            msg = lib.b200rt_gibbs_last_error(gibbs)
        elif batch is not None:
            msg = lib.b200rt_batch_last_error(batch)
        else:
            msg = lib.b200rt_last_error(handle)
        msg = msg.decode() if msg else ""
        raise B200Error(f"{what} failed with status {status}: {msg}")

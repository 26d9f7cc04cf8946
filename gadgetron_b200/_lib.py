"""ctypes binding of libgadgetron_b200.so (the C ABI in include/gadgetron_b200.h).

The library is the product: there is no CPU fallback.  If the shared object is
missing this module raises at import time with the command that builds it.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgadgetron_b200.so")

GB_OK = 0
_STATUS_NAMES = {
    1: "GB_ERR_INVALID_ARGUMENT",
    2: "GB_ERR_TRAJECTORY_RANGE",
    3: "GB_ERR_NOT_PREPROCESSED",
    4: "GB_ERR_CUDA",
    5: "GB_ERR_CUFFT",
    6: "GB_ERR_OUT_OF_MEMORY",
    7: "GB_ERR_DIMENSION_MISMATCH",
    8: "GB_ERR_TIMEOUT",
    9: "GB_ERR_INTERNAL",
}


class GadgetronB200Error(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("%s: %s" % (_STATUS_NAMES.get(status, str(status)), message))
        self.status = status


class TrajectoryRangeError(GadgetronB200Error, ValueError):
    pass


class NotPreprocessedError(GadgetronB200Error):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libgadgetron_b200.so is not built (%s); run `python gadgetron_b200/build.py`" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    u32 = ctypes.c_uint32
    u64 = ctypes.c_uint64
    i32 = ctypes.c_int
    f32 = ctypes.c_float
    sig = {
        "gb_last_error_message": (ctypes.c_char_p, []),
        "gb_version": (ctypes.c_char_p, []),
        "gb_kernel_launch_count": (ctypes.c_uint64, []),
        "gb_nufft_plan_create": (i32, [i32, P, P, f32, u32, P]),
        "gb_nufft_plan_destroy": (i32, [P]),
        "gb_nufft_preprocess": (i32, [P, P, u64, u32, P, i32, P]),
        "gb_nufft_compute": (i32, [P, P, P, P, i32, u32, i32, P]),
        "gb_nufft_mult_MH_M": (i32, [P, P, P, P, u32, P]),
        "gb_nufft_convolve": (i32, [P, P, P, i32, i32, u32, P]),
        "gb_nufft_convolve_nc2c_noalloc": (i32, [P, P, P, i32, u32, P]),
        "gb_nufft_fft": (i32, [P, P, i32, i32, u32, P]),
        "gb_nufft_deapodize": (i32, [P, P, i32, u32, P]),
        "gb_nufft_traj_grad": (i32, [P, P, P, P, P, u32, P]),
        "gb_nufft_traj_grad_from_grid": (i32, [P, P, P, P, u32, P]),
        "gb_nufft_get_info": (i32, [P, P, P, P, P, P, P]),
        "gb_nufft_device_errors": (i32, [P, P, P]),
        "gb_nufft_get_tiling": (i32, [P, P, P]),
        "gb_nufft_time_normal_convolutions": (i32, [P, u32, P, u32, P, u64, P, P, P]),
        "gb_nufft_autotune": (i32, [P, u32, P]),
        "gb_sense_autotune": (i32, [P, P]),
        "gb_nufft_set_tiling": (i32, [P, P, i32]),
        "gb_nufft_set_grid_schedule": (i32, [P, i32]),
        "gb_nufft_get_grid_schedule": (i32, [P, P]),
        "gb_sense_create": (i32, [i32, P, P, f32, u32, P]),
        "gb_sense_destroy": (i32, [P]),
        "gb_sense_preprocess": (i32, [P, P, u64, u32, P, P]),
        "gb_sense_set_csm": (i32, [P, P, u32]),
        "gb_sense_set_dcw": (i32, [P, P]),
        "gb_sense_mult_M": (i32, [P, P, P, i32, P]),
        "gb_sense_mult_MH": (i32, [P, P, P, i32, P]),
        "gb_sense_mult_MH_M": (i32, [P, P, P, i32, P]),
        "gb_sense_get_nufft_plan": (i32, [P, P]),
        "gb_cg_create": (i32, [P]),
        "gb_cg_destroy": (i32, [P]),
        "gb_cg_set_encoding_operator": (i32, [P, P, f32]),
        "gb_cg_set_max_iterations": (i32, [P, u32]),
        "gb_cg_set_tc_tolerance": (i32, [P, f32]),
        "gb_cg_set_x0": (i32, [P, P]),
        "gb_cg_set_preconditioner": (i32, [P, P]),
        "gb_cg_set_identity_regularization": (i32, [P, f32]),
        "gb_cg_set_image_regularization": (i32, [P, P, f32]),
        "gb_image_operator_compute": (i32, [P, u64, i32, P, P, P]),
        "gb_sense_precond_weights": (i32, [P, P, f32, P, P]),
        "gb_radial_trajectory_golden_ratio_2d": (i32, [u32, u32, u32, u32, i32, P, P]),
        "gb_radial_trajectory_fixed_angle_2d": (i32, [u32, u32, u32, f32, P, P]),
        "gb_radial_trajectory_variable_angle_2d": (i32, [P, u32, u32, u32, P, P]),
        "gb_radial_dcw_golden_ratio_2d": (i32, [u32, u32, f32, f32, u32, i32, P, P]),
        "gb_radial_dcw_fixed_angle_2d": (i32, [u32, u32, f32, f32, P, P]),
        "gb_sdc_estimate_dcw": (i32, [i32, P, f32, u32, f32, P, u64, P, P, P]),
        "gb_estimate_b1_map": (i32, [i32, P, u32, i32, P, P, P]),
        "gb_sense_buffer_create": (i32, [P]),
        "gb_sense_buffer_destroy": (i32, [P]),
        "gb_sense_buffer_setup": (i32, [P, i32, P, P, f32, u32, u32, u32, P]),
        "gb_sense_buffer_clear": (i32, [P, P]),
        "gb_sense_buffer_set_dcw": (i32, [P, P]),
        "gb_sense_buffer_set_csm": (i32, [P, P]),
        "gb_sense_buffer_add_frame_data": (i32, [P, P, P, u64, P, P]),
        "gb_sense_buffer_get_accumulated_coil_images": (i32, [P, P, P]),
        "gb_sense_buffer_get_combined_coil_image": (i32, [P, P, P]),
        "gb_sense_buffer_get_normalization_factor": (i32, [P, P]),
        "gb_cg_set_refinements": (i32, [P, u32]),
        "gb_cg_set_use_graph": (i32, [P, i32]),
        "gb_cg_set_frame_independent": (i32, [P, i32]),
        "gb_cg_set_barrier_spin_limit": (i32, [P, u32]),
        "gb_cg_set_row_fusion": (i32, [P, i32]),
        "gb_cg_solve": (i32, [P, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


lib = _load()
EXPORTED = (
    "gb_last_error_message gb_version gb_kernel_launch_count gb_nufft_plan_create gb_nufft_plan_destroy gb_nufft_preprocess "
    "gb_nufft_compute gb_nufft_mult_MH_M gb_nufft_convolve gb_nufft_convolve_nc2c_noalloc gb_nufft_fft gb_nufft_deapodize "
    "gb_nufft_traj_grad gb_nufft_traj_grad_from_grid gb_nufft_get_info gb_nufft_device_errors gb_nufft_get_tiling gb_nufft_autotune "
    "gb_nufft_time_normal_convolutions "
    "gb_nufft_set_tiling gb_nufft_set_grid_schedule gb_nufft_get_grid_schedule gb_sense_create gb_sense_destroy gb_sense_preprocess gb_sense_set_csm "
    "gb_sense_set_dcw gb_sense_mult_M gb_sense_mult_MH gb_sense_mult_MH_M gb_sense_get_nufft_plan gb_sense_autotune "
    "gb_cg_create gb_cg_destroy gb_cg_set_encoding_operator gb_cg_set_max_iterations "
    "gb_cg_set_tc_tolerance gb_cg_set_x0 gb_cg_set_preconditioner gb_cg_set_identity_regularization "
    "gb_cg_set_refinements gb_cg_set_use_graph gb_cg_set_frame_independent gb_cg_set_barrier_spin_limit gb_cg_set_row_fusion gb_cg_solve "
    "gb_cg_set_image_regularization gb_image_operator_compute gb_sense_precond_weights "
    "gb_radial_trajectory_golden_ratio_2d gb_radial_trajectory_fixed_angle_2d gb_radial_trajectory_variable_angle_2d "
    "gb_radial_dcw_golden_ratio_2d gb_radial_dcw_fixed_angle_2d gb_sdc_estimate_dcw "
    "gb_sense_buffer_create gb_sense_buffer_destroy gb_sense_buffer_setup gb_sense_buffer_clear "
    "gb_sense_buffer_set_dcw gb_sense_buffer_set_csm gb_sense_buffer_add_frame_data "
    "gb_sense_buffer_get_accumulated_coil_images gb_sense_buffer_get_combined_coil_image "
    "gb_sense_buffer_get_normalization_factor gb_estimate_b1_map").split()


def check(status: int):
    if status == GB_OK:
        return
    msg = lib.gb_last_error_message().decode(errors="replace")
    if status == 2:
        raise TrajectoryRangeError(status, msg)
    if status == 3:
        raise NotPreprocessedError(status, msg)
    raise GadgetronB200Error(status, msg)

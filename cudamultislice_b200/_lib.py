"""Loader of libmslice_b200.so and the ctypes signatures of include/mslice.h."""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmslice_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "mslice.h")

_lib = None

_i, _f, _d, _p, _s = C.c_int, C.c_float, C.c_double, C.c_void_p, C.c_char_p
_pi, _pf, _pd, _pll = C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_longlong)

# name -> (restype, argtypes), one entry per declaration of include/mslice.h
SIGNATURES = {
    "ms_create": (_i, [_i, C.POINTER(_p)]),
    "ms_destroy": (_i, [_p]),
    "ms_last_error": (_s, [_p]),
    "ms_version": (_s, []),
    "ms_set_option": (_i, [_p, _i, _i]),
    "ms_import_atoms": (_i, [_p, _s]),
    "ms_set_atoms": (_i, [_p, _p, _p, _p, _p, _i]),
    "ms_upload_binned_atoms": (_i, [_p]),
    "ms_upload_binned_atoms_tds": (_i, [_p, C.c_uint64, C.c_uint32, _f]),
    "ms_get_parameterisation": (_i, [_p, _s]),
    "ms_apply_microscope_parameters": (_i, [_p, _f, _f, _f, _f, _f, _f, _f, _f]),
    "ms_set_calculation_variables": (_i, [_p, _f, _f, _i, _i, _f, _f, _f, _f, _f]),
    "ms_stem_set_calculation_variables": (_i, [_p, _f, _f, _i, _i, _f, _f, _f]),
    "ms_precalculate_frequencies": (_i, [_p]),
    "ms_initialise_wavefunctions": (_i, [_p]),
    "ms_initialise_wavefunctions_dz": (_i, [_p, _f]),
    "ms_stem_initialise_wavefunctions": (_i, [_p, _i, _i]),
    "ms_set_fd_dz": (_i, [_p, _f]),
    "ms_multislice_step_fd": (_i, [_p, _i]),
    "ms_multislice_step_conventional": (_i, [_p, _i]),
    "ms_multislice_step_rs": (_i, [_p, _i]),
    "ms_get_size_x": (_i, [_p, _pf]),
    "ms_get_size_y": (_i, [_p, _pf]),
    "ms_get_size_z": (_i, [_p, _pf]),
    "ms_get_slices": (_i, [_p, _i, _pi]),
    "ms_get_kmax": (_i, [_p, _pf]),
    "ms_get_exit_wave": (_i, [_p]),
    "ms_get_stem_exit_wave": (_i, [_p]),
    "ms_free_exit_wave": (_i, [_p]),
    "ms_get_ew_value_abs": (_i, [_p, _i, _i, _pf]),
    "ms_get_ew_value_re": (_i, [_p, _i, _i, _pf]),
    "ms_get_ew_value_im": (_i, [_p, _i, _i, _pf]),
    "ms_get_ew_min": (_i, [_p, _pf]),
    "ms_get_ew_max": (_i, [_p, _pf]),
    "ms_alloc_tds": (_i, [_p]),
    "ms_add_tds_waves": (_i, [_p]),
    "ms_get_tds_min": (_i, [_p, _pf]),
    "ms_get_tds_max": (_i, [_p, _pf]),
    "ms_get_tds_val": (_i, [_p, _i, _i, _pf]),
    "ms_alloc_host_image": (_i, [_p]),
    "ms_simulate_image": (_i, [_p, _f]),
    "ms_get_im_value": (_i, [_p, _i, _i, _pf]),
    "ms_get_dqe_im_value": (_i, [_p, _i, _i, _pf]),
    "ms_get_im_min": (_i, [_p, _pf]),
    "ms_get_im_max": (_i, [_p, _pf]),
    "ms_get_image_contrast": (_i, [_p, _i, _i, _i, _i, _pf]),
    "ms_copy_exit_wave": (_i, [_p, _p]),
    "ms_copy_image": (_i, [_p, _p]),
    "ms_copy_tds": (_i, [_p, _p]),
    "ms_get_grid": (_i, [_p, _pi, _pi]),
    "ms_build_potential_stack": (_i, [_p, _pi]),
    "ms_run_conventional": (_i, [_p, _pi]),
    "ms_run_fd": (_i, [_p, _i, _pi]),
    "ms_get_slice_loop": (_i, [_p, _pi, _pi, _pi]),
    "ms_get_potential_sum": (_i, [_p, _pi, _pi]),
    "ms_get_raster_tuning": (_i, [_p, _pi, _pi]),
    "ms_annular_detector": (_i, [_p, _f, _f, _pd]),
    "ms_stem_raster": (_i, [_p, _p, _p, _i, _f, _f, _i, _p]),
    "ms_get_binned_counts": (_i, [_p, _pi, _pi]),
    "ms_copy_binned": (_i, [_p, _p, _p, _p, _p, _p]),
    "ms_copy_potential_slice": (_i, [_p, _i, _i, _p]),
    "ms_fft2": (_i, [_p, _p, _p, _i, _i, _i]),
    "ms_time_slices": (_i, [_p, _i, _i, _pf, _pf, _pf]),
    "ms_get_fft_plan": (_i, [_p, _i, _pi, _pi]),
    "ms_focal_series": (_i, [_p, _p, _i, _p, _i, _pd, _p]),
    "ms_focal_series_grad": (_i, [_p, _p, _i, _p, _i, _pd, _p, _p]),
    "ms_get_last_device_ms": (_i, [_p, _pf]),
    "ms_time_pass": (_i, [_p, _i, _i, _i, _i, _i, _pf]),
    "ms_frozen_phonon": (_i, [_p, C.c_uint64, C.c_uint32, _i, _f, _i, _p, _p]),
    "ms_simulate_image_series": (_i, [_p, _p, _p, _i, _p]),
    "ms_set_detector": (_i, [_p, _p, _p, _i, _i, _f, _f, _f, C.c_uint64]),
    "ms_write_tiff": (_i, [_p, _i, _s]),
    "ms_write_tiff_f32": (_i, [_s, _p, _i, _i]),
    "ms_stem_raster_concurrent": (_i, [_p, _i, _p, _p, _p, _f, _f, _i, _p]),
    "ms_get_launch_count": (_i, [_p, _pll]),
    "ms_build_atom_index_noalloc": (_i, [_p, _p, _p, _p, _i, _p, _p, _p, _i, _pi, _p]),
}


class MultisliceError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[ms_status {code}] {message}")
        self.code = code


def lib(path: str | None = None):
    """Load the engine library; fails loudly when it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python -m cudamultislice_b200.build` "
            "(the engine has no CPU implementation)")
    L = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L

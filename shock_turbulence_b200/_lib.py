"""ctypes binding of ``libst_b200.so`` (declarations in include/st_b200.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
import ctypes
import os

from .params import StParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libst_b200.so")

_dp = ctypes.c_void_p          # array arguments are raw addresses (host or device)
_ctx = ctypes.c_void_p

# name -> argument types (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "st_create": [ctypes.POINTER(StParams), ctypes.POINTER(ctypes.c_void_p)],
    "st_destroy": [_ctx],
    "st_last_error": [_ctx],
    "st_status_string": [ctypes.c_int],
    "st_default_params": [ctypes.POINTER(StParams), ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "st_set_state": [_ctx, _dp, _dp],
    "st_get_state": [_ctx, _dp, _dp],
    "st_set_tstep": [_ctx, ctypes.c_double],
    "st_get_tstep": [_ctx, ctypes.POINTER(ctypes.c_double)],
    "st_get_common": [_ctx, ctypes.c_char_p, _dp],
    "st_set_common": [_ctx, ctypes.c_char_p, _dp],
    "st_tridiagonal": [_ctx, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "st_pentadiagonal": [_ctx, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "st_tridiagonal_noalloc": [_ctx, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "st_compact_filter": [_ctx, _dp, _dp, ctypes.c_int],
    "st_gaussian_filter": [_ctx, _dp, _dp, ctypes.c_int],
    "st_compute_gamma": [_ctx, _dp],
    "st_rhs": [_ctx, _dp, _dp, _dp],
    "st_compute_hyper": [_ctx, _dp, _dp],
    "st_hyper_rhs": [_ctx, _dp, _dp, _dp],
    "st_species_rhs": [_ctx, _dp, _dp, _dp, _dp],
    "st_bc_rhs": [_ctx, _dp, _dp, _dp, _dp, ctypes.c_double],
    "st_sponge_forcing": [_ctx, _dp, _dp, _dp, _dp],
    "st_fix_pressure": [_ctx, _dp, _dp],
    "st_compute_cfl": [_ctx, _dp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
    "st_compute_tstep": [_ctx, _dp, _dp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
    "st_lddrk4": [_ctx, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)],
    "st_step": [_ctx, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)],
    "st_get_monitors": [_ctx, _dp],
    "st_compute_grad": [_ctx, _dp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
    "st_shell_count": [_ctx, ctypes.POINTER(ctypes.c_int)],
    "st_compute_srm_stats": [_ctx] + [ctypes.POINTER(ctypes.c_double)] * 4,
    "st_generate_shock_surface": [_ctx] + [ctypes.POINTER(ctypes.c_double)] * 2,
    "st_make_padded_arrays": [_ctx, _dp, _dp, _dp, _dp, _dp],
    "st_write_visual": [_ctx, _dp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_int],
    "st_sync": [_ctx],
    "st_step_async": [_ctx, ctypes.c_int],
    "st_get_time": [_ctx, ctypes.POINTER(ctypes.c_double)],
    "st_set_time": [_ctx, ctypes.c_double],
    "st_query": [_ctx],
    "st_memory": [_ctx, ctypes.POINTER(ctypes.c_longlong)],
    "st_set_stream": [_ctx, ctypes.c_void_p],
    "st_get_stream": [_ctx, ctypes.POINTER(ctypes.c_void_p)],
    "st_profile": [_ctx, ctypes.c_int],
    "st_profile_report": [_ctx, ctypes.c_char_p, ctypes.c_int],
    "st_launch_count": [_ctx, ctypes.POINTER(ctypes.c_longlong)],
    # batches of same-size cases
    "st_create_batch": [ctypes.POINTER(StParams), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)],
    "st_batch_info": [_ctx, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)],
    "st_set_active": [_ctx, ctypes.c_int],
    "st_case_start": [_ctx, ctypes.c_int, _dp, _dp, ctypes.c_double],
    "st_case_get": [_ctx, ctypes.c_int, _dp, _dp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)],
    "st_case_move": [_ctx, ctypes.c_int, ctypes.c_int],
    "st_batch_step_async": [_ctx],
    # 1-D spherical-radial batch (handle in place of the context)
    "st_radial_create": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_void_p)],
    "st_radial_destroy": [_ctx],
    "st_radial_last_error": [_ctx],
    "st_radial_num_points": [_ctx, ctypes.POINTER(ctypes.c_longlong)],
    "st_radial_set_state": [_ctx, _dp],
    "st_radial_get_state": [_ctx, _dp],
    "st_radial_get_hyper": [_ctx, _dp],
    "st_radial_get_time": [_ctx, _dp, _dp],
    "st_radial_step": [_ctx, ctypes.c_int],
    "st_radial_step_async": [_ctx, ctypes.c_int],
    "st_radial_set_stream": [_ctx, ctypes.c_void_p],
    "st_radial_config": [_ctx, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int],
    "st_radial_tune": [_ctx, ctypes.POINTER(ctypes.c_double)],
    "st_radial_dfdx": [_ctx, _dp, _dp, ctypes.c_int, ctypes.c_double],
    "st_radial_d2fdx2": [_ctx, _dp, _dp, _dp, ctypes.c_int],
    "st_radial_compact_filter_x": [_ctx, _dp, _dp],
    "st_radial_gaussian_filter_x": [_ctx, _dp, _dp],
    "st_radial_rhs": [_ctx, _dp, _dp],
    "st_radial_rhs_hyper": [_ctx, _dp, _dp],
    "st_radial_launch_count": [_ctx, ctypes.POINTER(ctypes.c_longlong)],
}
for _d in ("x", "y", "z"):
    for _s in ("sym", "asym"):
        SIGNATURES[f"st_df{_d.join(['d', ''])}_{_s}"] = [_ctx, _dp, _dp, ctypes.c_int, ctypes.c_double]
        SIGNATURES[f"st_d2fd{_d}2_{_s}"] = [_ctx, _dp, _dp, _dp, ctypes.c_int]
        SIGNATURES[f"st_compact_filter_{_d}_{_s}"] = [_ctx, _dp, _dp]
    SIGNATURES[f"st_gaussian_filter_{_d}"] = [_ctx, _dp, _dp]
    SIGNATURES[f"st_df{_d.join(['d', ''])}"] = [_ctx, _dp, _dp, ctypes.c_int, ctypes.c_double]
    SIGNATURES[f"st_d2fd{_d}2"] = [_ctx, _dp, _dp, _dp, ctypes.c_int]
    SIGNATURES[f"st_compact_filter_{_d}"] = [_ctx, _dp, _dp]

_RESTYPES = {"st_last_error": ctypes.c_char_p, "st_status_string": ctypes.c_char_p,
             "st_radial_last_error": ctypes.c_char_p,
             "st_default_params": None}

_lib = None


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with shock_turbulence_b200.build.build() "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib

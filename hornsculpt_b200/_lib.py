"""ctypes binding of libhs_bem.so (include/hs_bem.h). Loading fails loudly
when the library is missing: there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
import pathlib
import re

PKG = pathlib.Path(__file__).resolve().parent
LIBRARY = PKG / "libhs_bem.so"
HEADER = PKG.parent / "include" / "hs_bem.h"

HS_OK, HS_E_INVALID, HS_E_CUDA, HS_E_NUMERIC, HS_E_NOCONVERGE, HS_E_NOMEM, HS_E_CANCELLED, HS_E_UNSUPPORTED = range(8)


class hs_numerics(C.Structure):
    _fields_ = [("quadrature_order", C.c_uint32), ("singular_order", C.c_uint32),
                ("near_distance_ratio", C.c_double), ("near_relative_tolerance", C.c_double),
                ("near_maximum_depth", C.c_uint32), ("relative_residual_tolerance", C.c_double),
                ("maximum_refinement_steps", C.c_uint32), ("acceleration", C.c_uint32), ("precision", C.c_uint32),
                ("fmm_leaf_support_capacity", C.c_uint32), ("fmm_separation_ratio", C.c_double),
                ("fmm_maximum_iterations", C.c_uint32), ("fmm_restart_length", C.c_uint32),
                ("fmm_preconditioner_block_width", C.c_uint32)]


class hs_request(C.Structure):
    _fields_ = [("density", C.c_double), ("sound_speed", C.c_double),
                ("frequencies", C.POINTER(C.c_double)), ("frequency_count", C.c_size_t),
                ("plan_frequencies", C.POINTER(C.c_double)), ("plan_frequency_count", C.c_size_t),
                ("excitation_count", C.c_size_t), ("excitation_face_offsets", C.POINTER(C.c_size_t)),
                ("excitation_face_ids", C.POINTER(C.c_uint32)), ("excitation_velocities", C.POINTER(C.c_double)),
                ("observers", C.POINTER(C.c_double)), ("observer_count", C.c_size_t),
                ("far_field", C.c_int32), ("far_origin", C.c_double * 3), ("far_reference_distance", C.c_double),
                ("numerics", hs_numerics)]


class hs_progress(C.Structure):
    _fields_ = [("completed_frequencies", C.c_size_t), ("total_frequencies", C.c_size_t),
                ("frequency", C.c_double), ("phase", C.c_uint32)]


class hs_excitation_info(C.Structure):
    _fields_ = [("boundary_residual", C.c_double), ("refinement_steps", C.c_uint32), ("iterations", C.c_uint32),
                ("field_comparison_degree", C.c_uint32), ("field_verification_degree", C.c_uint32),
                ("field_discrepancy", C.c_double), ("impedance_count", C.c_size_t)]


class hs_face_impedance(C.Structure):
    _fields_ = [("face_id", C.c_uint32), ("area", C.c_double), ("mean_pressure", C.c_double * 2),
                ("volume_velocity", C.c_double * 2), ("volume_impedance", C.c_double * 2)]


class hs_frequency_info(C.Structure):
    _fields_ = [("frequency", C.c_double), ("assembly_ms", C.c_double), ("factorization_ms", C.c_double),
                ("triangular_solve_ms", C.c_double), ("solve_ms", C.c_double), ("field_ms", C.c_double),
                ("residual_check_ms", C.c_double), ("interaction_plan_ms", C.c_double),
                ("interaction_plan_reused", C.c_int32)]


class hs_serve_options(C.Structure):
    _fields_ = [("workers", C.c_uint32), ("memory_fraction", C.c_double), ("resident_meshes", C.c_uint32),
                ("planning_frequency", C.c_double), ("max_batch_frequencies", C.c_uint32)]


class hs_serve_timing(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double),
                ("footprint_bytes", C.c_size_t), ("batched_requests", C.c_uint32)]


class hs_field_settings(C.Structure):
    _fields_ = [("minimum_boundary_distance", C.c_double), ("relative_quadrature_tolerance", C.c_double),
                ("maximum_quadrature_depth", C.c_uint32)]


PROGRESS_FN = C.CFUNCTYPE(None, C.POINTER(hs_progress), C.c_void_p)
NETWORK_FN = C.CFUNCTYPE(C.c_int, C.c_double, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_double),
                         C.POINTER(C.c_double), C.c_void_p)
_P = C.c_void_p
_lib = None


def declared_symbols() -> list[str]:
    """Function names declared by include/hs_bem.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hs_[a-z_]+)\s*\(", text)) - {"hs_progress_fn", "hs_status"})


def load():
    """Loads libhs_bem.so and declares its signatures; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIBRARY.exists():
        raise ImportError(f"{LIBRARY} is missing; build it with `python -m hornsculpt_b200.build` "
                          "(the solver has no CPU fallback)")
    lib = C.CDLL(str(LIBRARY))
    sig = {
        "hs_last_error": (C.c_char_p, []),
        "hs_numerics_default": (None, [C.POINTER(hs_numerics)]),
        "hs_bem_session_create": (C.c_int, [_P, C.c_size_t, _P, _P, _P, C.c_size_t, C.c_uint32, C.POINTER(_P)]),
        "hs_bem_session_destroy": (None, [_P]),
        "hs_bem_session_set_stream": (C.c_int, [_P, _P]),
        "hs_bem_solve": (C.c_int, [_P, C.POINTER(hs_request), _P, PROGRESS_FN, _P, C.POINTER(_P)]),
        "hs_result_frequency_count": (C.c_size_t, [_P]),
        "hs_result_excitation_count": (C.c_size_t, [_P]),
        "hs_result_triangle_count": (C.c_size_t, [_P]),
        "hs_result_pressure_dof_count": (C.c_size_t, [_P]),
        "hs_result_observer_count": (C.c_size_t, [_P]),
        "hs_result_peak_device_bytes": (C.c_size_t, [_P]),
        "hs_result_frequency_info": (C.c_int, [_P, C.c_size_t, C.POINTER(hs_frequency_info)]),
        "hs_result_excitation_info": (C.c_int, [_P, C.c_size_t, C.c_size_t, C.POINTER(hs_excitation_info)]),
        "hs_result_pressure_trace": (C.c_int, [_P, C.c_size_t, C.c_size_t, _P]),
        "hs_result_surface_pressure": (C.c_int, [_P, C.c_size_t, C.c_size_t, _P]),
        "hs_result_normal_derivative": (C.c_int, [_P, C.c_size_t, C.c_size_t, _P]),
        "hs_result_observer_pressure": (C.c_int, [_P, C.c_size_t, C.c_size_t, _P]),
        "hs_result_impedances": (C.c_int, [_P, C.c_size_t, C.c_size_t, _P]),
        "hs_result_copy_all": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(hs_excitation_info),
                                         C.POINTER(hs_frequency_info)]),
        "hs_result_free": (None, [_P]),
        "hs_device_description": (C.c_int, [C.c_char_p, C.c_size_t]),
        "hs_bem_session_set_profiling": (C.c_int, [_P, C.c_int32]),
        "hs_bem_session_profile": (C.c_int, [_P, C.c_char_p, C.c_size_t, _P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
        "hs_bem_session_work": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
        "hs_bem_session_set_graphs": (C.c_int, [_P, C.c_int32]),
        "hs_bem_solve_coupled": (C.c_int, [_P, C.POINTER(hs_request), NETWORK_FN, _P, _P, C.POINTER(_P)]),
        "hs_result_coupling": (C.c_int, [_P, C.c_size_t, _P, _P, _P, C.POINTER(C.c_size_t)]),
        "hs_autotune_set_enabled": (C.c_int, [C.c_int32]),
        "hs_autotune_clear": (C.c_int, []),
        "hs_autotune_report": (C.c_int, [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
        "hs_bem_session_graph_launches": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
        "hs_bem_debug_plan": (C.c_int, [_P, C.c_size_t, _P, C.c_size_t, C.POINTER(hs_numerics), C.c_double, _P, _P,
                                        _P, _P, _P, _P, _P]),
        "hs_bem_debug_plan_device": (C.c_int, [_P, C.c_size_t, _P, C.c_size_t, C.POINTER(hs_numerics), C.c_double,
                                               C.c_uint32, _P, _P, _P, _P, _P, _P, _P, _P]),
        "hs_bem_observer_field_noalloc": (C.c_int, [_P, C.c_size_t, _P, C.c_size_t, _P, _P, _P, C.c_size_t, C.c_double,
                                                    C.c_uint32, C.c_int32, _P, C.c_double, C.c_double, C.c_uint32,
                                                    _P, _P]),
        "hs_bem_debug_assemble": (C.c_int, [_P, C.POINTER(hs_numerics), C.c_double, C.c_double, _P, _P, _P]),
        "hs_bem_debug_fmm_far": (C.c_int, [_P, C.POINTER(hs_numerics), C.c_double, C.c_double, _P, _P, _P, _P,
                                           C.c_size_t, C.POINTER(C.c_size_t), _P, C.c_size_t,
                                           C.POINTER(C.c_size_t)]),
        "hs_bem_debug_fmm_selftest": (C.c_int, [C.POINTER(C.c_double)]),
        "hs_bem_session_set_plane_wave_threshold": (C.c_int, [_P, C.c_double]),
        "hs_bem_session_set_fmm_grouped_m2l": (C.c_int, [_P, C.c_int]),
        "hs_bem_session_set_planner": (C.c_int, [_P, C.c_uint32]),
        "hs_bem_session_plan_stats": (C.c_int, [_P, _P]),
        "hs_bem_session_set_fmm_audit": (C.c_int, [_P, C.c_uint32]),
        "hs_bem_session_fmm_audit_counts": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "hs_bem_debug_lu": (C.c_int, [C.c_uint32, C.c_size_t, C.c_size_t, _P, _P, _P, C.POINTER(C.c_int32)]),
        "hs_bem_debug_fmm_tree": (C.c_int, [_P, C.c_size_t, _P, C.c_size_t, C.c_uint32, C.c_double, C.c_double, _P,
                                            _P, C.c_size_t]),
        "hs_field_settings_default": (C.c_int, [C.POINTER(hs_field_settings)]),
        "hs_bem_pressure_field": (C.c_int, [_P, C.c_double, C.c_double, _P, _P, _P, C.c_size_t,
                                            C.POINTER(hs_field_settings), _P, _P]),
        "hs_serve_options_default": (None, [C.POINTER(hs_serve_options)]),
        "hs_serve_create": (C.c_int, [C.POINTER(hs_serve_options), C.POINTER(_P)]),
        "hs_serve_submit": (C.c_int, [_P, _P, C.c_size_t, _P, _P, _P, C.c_size_t, C.POINTER(hs_request),
                                      C.POINTER(C.c_uint64)]),
        "hs_serve_wait": (C.c_int, [_P, C.c_uint64, C.POINTER(_P), C.POINTER(hs_serve_timing)]),
        "hs_serve_destroy": (None, [_P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class BemError(RuntimeError):
    """std::runtime_error counterpart; `status` is the hs_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class BemCancelled(BemError):
    pass


class BemUnsupported(BemError):
    pass


def check(status: int) -> None:
    if status == HS_OK:
        return
    message = load().hs_last_error().decode()
    if status == HS_E_INVALID:
        raise ValueError(message)
    if status == HS_E_CANCELLED:
        raise BemCancelled(status, message)
    if status == HS_E_UNSUPPORTED:
        raise BemUnsupported(status, message)
    raise BemError(status, message)

"""B200-native candidate-audit engine for BlitzRemesher.

Python mirror of the C ABI in ``include/blitz_audit.h``. The compute path is
the CUDA library ``libblitz_b200.so``; there is no CPU fallback: loading fails
loudly if the library is missing and every audit call reports
``BLITZ_UNAVAILABLE`` without a GPU.

Names follow the reference: ``evaluate`` mirrors ``blitz::evaluate``
(src/evaluate.cpp:353) and ``AuditSession.candidates`` mirrors the four-gate
gate of src/neural/generate.cpp:365-388 applied to GpuActionState trials.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import synthetic  # noqa: F401

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libblitz_b200.so"

BLITZ_OK, BLITZ_INVALID_ARGUMENT, BLITZ_OUT_OF_MEMORY, BLITZ_INTERNAL_ERROR = 0, 1, 2, 3
BLITZ_CANCELLED, BLITZ_BUDGET_LIMITED, BLITZ_UNAVAILABLE = 4, 5, 6
ABI_VERSION = 5


class BlitzError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"blitz status {status}: {message}")
        self.status = status


class Stream(C.Structure):
    _fields_ = [("data", C.c_void_p), ("count", C.c_size_t), ("stride", C.c_size_t)]


class BlitzMesh(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("abi_version", C.c_uint32), ("positions", Stream),
                ("normals", Stream), ("uv", Stream), ("colors", Stream), ("tangents", Stream),
                ("indices", C.c_void_p), ("index_count", C.c_size_t), ("materials", C.c_void_p),
                ("material_count", C.c_size_t), ("double_sided", C.c_void_p), ("double_sided_count", C.c_size_t)]


class NeuralOptionsV2(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("version", C.c_uint32), ("device", C.c_int32),
                ("memory_mib", C.c_uint32), ("action_trials", C.c_uint32), ("ranking_seed", C.c_uint32),
                ("exact_position_bps", C.c_uint16), ("action_batch", C.c_uint8), ("origin", C.c_uint8),
                ("ranking", C.c_uint8), ("confirmation", C.c_uint8), ("raster_backend", C.c_uint8),
                ("vertex_storage", C.c_uint8), ("preserve_uv", C.c_uint8), ("overdraw_tiebreak", C.c_uint8),
                ("cache_rasters", C.c_uint8), ("mask_only_coverage", C.c_uint8), ("direct_targets", C.c_uint8),
                ("view_batch", C.c_uint8), ("candidate_batch", C.c_uint8), ("reserved", C.c_uint8 * 3)]


class NeuralInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("encode_ns", C.c_uint64), ("inference_ns", C.c_uint64),
                ("decode_ns", C.c_uint64), ("gpu_audit_ns", C.c_uint64), ("reference_audit_ns", C.c_uint64),
                ("decoded", C.c_uint64), ("legal_collapses", C.c_uint64), ("rejected_collapses", C.c_uint64),
                ("reference_rejections", C.c_uint64), ("fallback_levels", C.c_uint32)]


class CurvePoint(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class Settings(C.Structure):
    """blitz_settings (blitz.h:38-63)."""
    _fields_ = [("struct_size", C.c_uint32), ("abi_version", C.c_uint32), ("levels", C.c_uint8),
                ("profile", C.c_uint8), ("triangle_overhead_bps", C.c_uint16),
                ("max_added_vertex_bytes_bps", C.c_uint32), ("objective", C.c_uint8), ("beam_width", C.c_uint8),
                ("search_supersample", C.c_uint8), ("audit_supersample", C.c_uint8), ("max_supersample", C.c_uint8),
                ("prune", C.c_uint8), ("force_scalar", C.c_uint8), ("coupled_wedges", C.c_uint8),
                ("candidate_budget", C.c_uint16), ("search_ortho", C.c_uint16), ("search_perspective", C.c_uint16),
                ("audit_ortho", C.c_uint16), ("audit_perspective", C.c_uint16), ("search_seed", C.c_uint32),
                ("audit_seed", C.c_uint32), ("pixels_per_meter", C.c_double), ("meters_per_unit", C.c_double),
                ("base_pixels", C.c_double), ("last_pixels", C.c_double), ("max_lod0_delta_px", C.c_double),
                ("normal_weight", C.c_double), ("color_weight", C.c_double), ("material_weight", C.c_double),
                ("max_changed_area", C.c_double), ("transition", C.c_void_p), ("transition_count", C.c_size_t),
                ("normal_importance", C.c_void_p), ("normal_importance_count", C.c_size_t),
                ("attribute_importance", C.c_void_p), ("attribute_importance_count", C.c_size_t),
                ("cancelled", C.c_void_p), ("user_data", C.c_void_p)]


class LodInfo(C.Structure):
    """blitz_lod_info (blitz.h:64-73)."""
    _fields_ = [("struct_size", C.c_uint32), ("mesh", BlitzMesh), ("screen_pixels", C.c_double),
                ("transition_limit", C.c_double), ("source_limit", C.c_double), ("transition_error", C.c_double),
                ("source_error", C.c_double), ("transition_worst_view", C.c_uint32), ("source_worst_view", C.c_uint32),
                ("shared_vertices", C.c_uint8), ("passed", C.c_uint8), ("reference_triangles", C.c_uint32),
                ("transition_changed_area", C.c_double), ("source_changed_area", C.c_double),
                ("transition_changed_area_worst_view", C.c_uint32), ("source_changed_area_worst_view", C.c_uint32)]


class StorageInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("source_vertex_bytes", C.c_uint64), ("added_vertex_bytes", C.c_uint64),
                ("index_bytes", C.c_uint64), ("total_bytes", C.c_uint64), ("added_vertex_budget_bytes", C.c_uint64),
                ("max_added_vertex_bytes_bps", C.c_uint32)]


class RuntimeLodStorage(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("scheduled_index", C.c_uint8), ("added_vertex_bytes", C.c_uint64),
                ("index_bytes", C.c_uint64), ("cumulative_added_vertex_bytes", C.c_uint64)]


class NeuralOptionsV1(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("version", C.c_uint32), ("device", C.c_int32),
                ("memory_mib", C.c_uint32), ("overdraw_tiebreak", C.c_uint8), ("reserved", C.c_uint8 * 3)]


class ActionProposal(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("version", C.c_uint32), ("start_triangles", C.c_uint32),
                ("target_triangles", C.c_uint32), ("final_triangles", C.c_uint32), ("trial_budget", C.c_uint32),
                ("trials", C.c_uint32), ("accepted_batches", C.c_uint32), ("screen_pixels", C.c_double),
                ("origin", C.c_uint8), ("output", C.c_uint8), ("stop_reason", C.c_uint8), ("reserved", C.c_uint8 * 5)]


class EvalSettings(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("profile", C.c_uint8), ("supersample", C.c_uint8),
                ("max_supersample", C.c_uint8), ("force_two_sided", C.c_uint8), ("conservative_screen", C.c_uint8),
                ("reserved", C.c_uint8 * 1), ("views_orthographic", C.c_uint16), ("views_perspective", C.c_uint16),
                ("views_seed", C.c_uint32), ("screen_size", C.c_double), ("limit", C.c_double),
                ("max_changed_area", C.c_double)]


class Measurement(C.Structure):
    _fields_ = [("error", C.c_double), ("coverage", C.c_double), ("coverage_upper", C.c_double),
                ("changed_area", C.c_double), ("normal_degrees", C.c_double), ("worst_view", C.c_uint32),
                ("changed_area_worst_view", C.c_uint32), ("views_evaluated", C.c_uint32),
                ("supersample", C.c_uint8), ("complete", C.c_uint8), ("passed", C.c_uint8),
                ("resource_limited", C.c_uint8), ("cancelled", C.c_uint8), ("reserved", C.c_uint8 * 3)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Collapse(C.Structure):
    _fields_ = [("from_", C.c_uint32), ("to", C.c_uint32), ("placement", C.c_uint32), ("position", C.c_float * 3)]


class Verdict(C.Structure):
    _fields_ = [("accepted", C.c_uint8), ("failed_gate", C.c_uint8), ("exact_path", C.c_uint8),
                ("reserved", C.c_uint8), ("removed", C.c_uint32)]


COLLAPSE_DTYPE = np.dtype([("from", "<u4"), ("to", "<u4"), ("placement", "<u4"), ("position", "<f4", (3,))])
VERDICT_DTYPE = np.dtype([("accepted", "u1"), ("failed_gate", "u1"), ("exact_path", "u1"), ("reserved", "u1"),
                          ("removed", "<u4")])
MEASUREMENT_DTYPE = np.dtype([("error", "<f8"), ("coverage", "<f8"), ("coverage_upper", "<f8"),
                              ("changed_area", "<f8"), ("normal_degrees", "<f8"), ("worst_view", "<u4"),
                              ("changed_area_worst_view", "<u4"), ("views_evaluated", "<u4"),
                              ("supersample", "u1"), ("complete", "u1"), ("passed", "u1"),
                              ("resource_limited", "u1"), ("cancelled", "u1"), ("reserved", "u1", (3,))],
                             align=True)
assert COLLAPSE_DTYPE.itemsize == C.sizeof(Collapse)
assert VERDICT_DTYPE.itemsize == C.sizeof(Verdict)
assert MEASUREMENT_DTYPE.itemsize == C.sizeof(Measurement)

_lib = None

EXPORTS = {
    "blitz_abi_version": ([], C.c_uint32),
    "blitz_neural_options_v2_init": ([C.POINTER(NeuralOptionsV2), C.c_size_t], C.c_int),
    "blitz_eval_settings_init": ([C.POINTER(EvalSettings), C.c_size_t], C.c_int),
    "blitz_audit_session_create": ([C.POINTER(BlitzMesh), C.POINTER(NeuralOptionsV2), C.POINTER(C.c_void_p),
                                    C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_session_destroy": ([C.c_void_p], None),
    "blitz_audit_bind_reference": ([C.c_void_p, C.POINTER(BlitzMesh), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_evaluate": ([C.c_void_p, C.POINTER(BlitzMesh), C.POINTER(BlitzMesh), C.POINTER(EvalSettings),
                              C.POINTER(Measurement), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_actions": ([C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t],
                            C.c_int),
    "blitz_audit_raster": ([C.c_void_p, C.POINTER(BlitzMesh), C.c_double, C.c_uint8, C.c_uint16, C.c_uint16,
                            C.c_uint32, C.c_uint32, C.c_uint8, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32),
                            C.POINTER(C.c_uint8), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_candidates": ([C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(EvalSettings), C.c_void_p,
                                C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_candidates_device": ([C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(EvalSettings), C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_session_info": ([C.c_void_p, C.POINTER(NeuralInfo)], C.c_int),
    "blitz_audit_coverage_distance": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint8,
                                       C.c_int, C.POINTER(C.c_double), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_profile_enable": ([C.c_void_p, C.c_int], C.c_int),
    "blitz_audit_execute": ([C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(EvalSettings), C.c_void_p, C.c_size_t,
                             C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_execute_ex": ([C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(EvalSettings), C.c_void_p,
                                C.c_void_p, C.c_size_t, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_execute_options_init": ([C.c_void_p], None),
    "blitz_surrogate_create": ([C.c_int, C.c_uint32, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_surrogate_destroy": ([C.c_void_p], None),
    "blitz_surrogate_load": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t],
                             C.c_int),
    "blitz_surrogate_save": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t],
                             C.c_int),
    "blitz_surrogate_score": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t],
                              C.c_int),
    "blitz_surrogate_gradients": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                   C.POINTER(C.c_float), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_surrogate_train_step": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_float,
                                    C.POINTER(C.c_float), C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_surrogate_features": ([C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_attach_surrogate": ([C.c_void_p, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_chain_settings_init": ([C.c_void_p], None),
    "blitz_audit_chain": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_char_p,
                           C.c_size_t], C.c_int),
    "blitz_audit_batch_create": ([C.c_void_p, C.c_size_t, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_batch_destroy": ([C.c_void_p], None),
    "blitz_audit_batch_candidates": ([C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(EvalSettings), C.c_void_p,
                                      C.c_uint32, C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_batch_candidates_host": ([C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(EvalSettings), C.c_void_p,
                                           C.c_uint32, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_batch_read_info": ([C.c_void_p, C.c_void_p], C.c_int),
    "blitz_settings_init": ([C.POINTER(Settings), C.c_size_t], C.c_int),
    "blitz_generate": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_neural_options_init": ([C.POINTER(NeuralOptionsV1), C.c_size_t], C.c_int),
    "blitz_neural_model_load": ([C.c_char_p, C.POINTER(NeuralOptionsV1), C.POINTER(C.c_void_p), C.c_char_p,
                                 C.c_size_t], C.c_int),
    "blitz_neural_model_load_v2": ([C.c_char_p, C.POINTER(NeuralOptionsV2), C.POINTER(C.c_void_p), C.c_char_p,
                                    C.c_size_t], C.c_int),
    "blitz_neural_model_destroy": ([C.c_void_p], None),
    "blitz_neural_model_sha256": ([C.c_void_p], C.c_char_p),
    "blitz_generate_neural": ([C.POINTER(BlitzMesh), C.POINTER(Settings), C.c_void_p, C.POINTER(C.c_void_p),
                               C.c_char_p, C.c_size_t], C.c_int),
    "blitz_result_lod_count": ([C.c_void_p], C.c_size_t),
    "blitz_result_runtime_lod_count": ([C.c_void_p], C.c_size_t),
    "blitz_result_runtime_lod_index": ([C.c_void_p, C.c_size_t], C.c_size_t),
    "blitz_result_lod": ([C.c_void_p, C.c_size_t, C.POINTER(LodInfo)], C.c_int),
    "blitz_result_storage": ([C.c_void_p, C.POINTER(StorageInfo)], C.c_int),
    "blitz_result_runtime_lod_storage": ([C.c_void_p, C.c_size_t, C.POINTER(RuntimeLodStorage)], C.c_int),
    "blitz_result_destroy": ([C.c_void_p], None),
    "blitz_result_neural_info": ([C.c_void_p, C.POINTER(NeuralInfo)], C.c_int),
    "blitz_result_neural_action_proposal_count": ([C.c_void_p], C.c_size_t),
    "blitz_result_neural_action_proposal": ([C.c_void_p, C.c_size_t, C.POINTER(ActionProposal)], C.c_int),
    "blitz_audit_state_materials": ([C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32), C.c_char_p,
                                     C.c_size_t], C.c_int),
    "blitz_mesh_file_load": ([C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(BlitzMesh), C.c_char_p, C.c_size_t],
                             C.c_int),
    "blitz_mesh_file_destroy": ([C.c_void_p], None),
    "blitz_mesh_save_ply": ([C.POINTER(BlitzMesh), C.c_char_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_result_save_chain": ([C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_state": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32),
                           C.c_char_p, C.c_size_t], C.c_int),
    "blitz_mesh_bounds": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_char_p, C.c_size_t], C.c_int),
    "blitz_view_cameras": ([C.c_void_p, C.c_double, C.c_double, C.c_uint16, C.c_uint16, C.c_uint32, C.c_void_p,
                           C.c_size_t, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_chain_schedule": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t],
                             C.c_int),
    "blitz_audit_state_uv": ([C.c_void_p, C.c_void_p, C.c_size_t, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_reset": ([C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "blitz_audit_profile_read": ([C.c_void_p, C.c_void_p], C.c_int),
}


class Execution(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("commits", C.c_uint32), ("trials", C.c_uint32),
                ("final_faces", C.c_uint32), ("audited", C.c_uint64), ("stop_reason", C.c_uint8),
                ("fallbacks", C.c_uint8), ("reserved", C.c_uint8 * 6)]


class ExecuteOptions(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("batch", C.c_uint32), ("keep_permille", C.c_uint32),
                ("ranking", C.c_uint32), ("reserved", C.c_uint32 * 4)]


class ChainSettings(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("levels", C.c_uint32), ("base_pixels", C.c_double),
                ("last_pixels", C.c_double), ("max_lod0_delta_px", C.c_double), ("transition_curve", C.c_float * 16),
                ("transition_points", C.c_uint32), ("search_orthographic", C.c_uint16),
                ("search_perspective", C.c_uint16), ("search_seed", C.c_uint32), ("audit_orthographic", C.c_uint16),
                ("audit_perspective", C.c_uint16), ("audit_seed", C.c_uint32), ("search_supersample", C.c_uint8),
                ("audit_supersample", C.c_uint8), ("max_supersample", C.c_uint8), ("force_two_sided", C.c_uint8),
                ("max_changed_area", C.c_double), ("batch", C.c_uint32), ("keep_permille", C.c_uint32),
                ("trial_budget", C.c_uint32), ("min_faces", C.c_uint32), ("ranking", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class ChainLevel(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("level", C.c_uint32), ("pixels", C.c_double),
                ("transition", C.c_double), ("source_bound", C.c_double), ("faces", C.c_uint32),
                ("commits", C.c_uint32), ("trials", C.c_uint32), ("stop_reason", C.c_uint8),
                ("confirmed", C.c_uint8), ("reserved", C.c_uint8 * 2), ("source_audit", Measurement),
                ("transition_audit", Measurement), ("seconds", C.c_double)]


CHAIN_EMIT = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(C.c_float),
                         C.c_uint32)


def chain_settings(levels: int, base_pixels: float, last_pixels: float, curve=((0.0, 2.0), (1.0, 3.0)),
                   max_lod0_delta_px: float = 2.0, search_views=(42, 12, 0xB1172024), audit_views=(642, 64, 0xB1172026),
                   search_supersample: int = 4, audit_supersample: int = 8, max_supersample: int = 32,
                   max_changed_area: float = 1.0, batch: int = 64, keep_permille: int = 0,
                   trial_budget: int = 1 << 30, min_faces: int = 1, ranking: int = 3) -> ChainSettings:
    c = ChainSettings()
    load().blitz_chain_settings_init(C.byref(c))
    c.levels, c.base_pixels, c.last_pixels, c.max_lod0_delta_px = levels, base_pixels, last_pixels, max_lod0_delta_px
    for i, (x, y) in enumerate(curve):
        c.transition_curve[2 * i], c.transition_curve[2 * i + 1] = x, y
    c.transition_points = len(curve)
    c.search_orthographic, c.search_perspective, c.search_seed = search_views
    c.audit_orthographic, c.audit_perspective, c.audit_seed = audit_views
    c.search_supersample, c.audit_supersample, c.max_supersample = search_supersample, audit_supersample, max_supersample
    c.max_changed_area, c.batch, c.keep_permille = max_changed_area, batch, keep_permille
    c.trial_budget, c.min_faces, c.ranking = trial_budget, min_faces, ranking
    return c


class ViewCamera(C.Structure):
    _fields_ = [("right", C.c_float * 3), ("up", C.c_float * 3), ("forward", C.c_float * 3),
                ("distance", C.c_double), ("focal", C.c_double), ("scale", C.c_double),
                ("perspective", C.c_uint32), ("pad", C.c_uint32)]


def mesh_bounds(mesh):
    """(center float32[3], radius) of a mesh, as every audit projects with
    (blitz_mesh_bounds; no GPU needed)."""
    h = _MeshHold(mesh)
    center = np.zeros(3, np.float32)
    radius = C.c_double()
    err = C.create_string_buffer(512)
    _check(load().blitz_mesh_bounds(C.byref(h.c), center.ctypes.data, C.byref(radius), err, 512), err)
    return center, radius.value


def view_cameras(center, radius: float, screen: float, views: tuple) -> list:
    """The camera set (ortho, persp, seed) at `screen` (blitz_view_cameras)."""
    ortho, persp, seed = views
    c = np.ascontiguousarray(center, np.float32)
    out = (ViewCamera * max(1, ortho + persp))()
    err = C.create_string_buffer(512)
    _check(load().blitz_view_cameras(c.ctypes.data, radius, screen, ortho, persp, seed, out, ortho + persp, err, 512),
           err)
    return list(out[: ortho + persp])


def chain_schedule(settings: ChainSettings):
    """The chain's per-level (pixels, transition bound, LOD0 bound), index 0
    the source (blitz_chain_schedule; no GPU needed)."""
    n = settings.levels
    p, t, b = (np.zeros(n) for _ in range(3))
    err = C.create_string_buffer(512)
    _check(load().blitz_chain_schedule(C.byref(settings), p.ctypes.data, t.ctypes.data, b.ctypes.data, n, err, 512),
           err)
    return p, t, b


class BatchInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("sessions", C.c_uint32), ("tier", C.c_uint32), ("tuned", C.c_uint32),
                ("graph_captured", C.c_uint32), ("tune_ms", C.c_float * 4), ("graph_launches", C.c_uint64),
                ("exact_candidates", C.c_uint64), ("audit_ms", C.c_float), ("units", C.c_uint64),
                ("region_samples", C.c_uint64), ("changed_samples", C.c_uint64),
                ("tier_units", C.c_uint64 * 4), ("tier_cycles", C.c_uint64 * 4), ("phase_cycles", C.c_uint64 * 3),
                ("flipped_samples", C.c_uint64), ("region_split", C.c_uint64 * 15), ("face_samples", C.c_uint64), ("tier_max_cycles", C.c_uint64 * 4), ("tier_ms", C.c_float * 3)]


BATCH_GRAPH, BATCH_AUTOTUNE, BATCH_PROFILE, BATCH_TIMING = 1, 2, 4, 8


class AuditProfile(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("enabled", C.c_uint32), ("launches", C.c_uint64),
                ("audit_launches", C.c_uint64), ("audit_ms", C.c_double), ("prepare_ms", C.c_double),
                ("verdict_ms", C.c_double), ("units", C.c_uint64), ("region_samples", C.c_uint64),
                ("changed_samples", C.c_uint64), ("record_bytes", C.c_uint64)]


def library_path() -> Path:
    return LIB_PATH


def load() -> C.CDLL:
    """Loads the CUDA library (building it if sources are newer). Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    from . import build as _build

    if _build.needs_build():
        try:
            _build.build()
        except Exception as exc:  # pragma: no cover - explicit failure, never a fallback
            if not LIB_PATH.exists():
                raise RuntimeError(f"libblitz_b200.so is missing and could not be built: {exc}") from exc
    if not LIB_PATH.exists():
        raise RuntimeError("libblitz_b200.so is missing; run blitzremesher_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    for name, (args, res) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


class _MeshHold:
    """Keeps numpy arrays alive while a BlitzMesh borrows them."""

    def __init__(self, mesh):
        self.pos = np.ascontiguousarray(mesh.positions, dtype=np.float32)
        self.idx = np.ascontiguousarray(mesh.indices, dtype=np.uint32).reshape(-1)
        self.uv = None if mesh.uv is None else np.ascontiguousarray(mesh.uv, dtype=np.float32)
        self.mat = None if mesh.materials is None else np.ascontiguousarray(mesh.materials, dtype=np.uint16)
        self.ds = None if mesh.double_sided is None else np.ascontiguousarray(mesh.double_sided, dtype=np.uint8)
        m = BlitzMesh()
        m.struct_size = C.sizeof(BlitzMesh)
        m.abi_version = ABI_VERSION
        m.positions = Stream(self.pos.ctypes.data, self.pos.shape[0], 12)
        if self.uv is not None:
            m.uv = Stream(self.uv.ctypes.data, self.uv.shape[0], 8)
        m.indices = self.idx.ctypes.data
        m.index_count = self.idx.size
        if self.mat is not None:
            m.materials, m.material_count = self.mat.ctypes.data, self.mat.size
        if self.ds is not None:
            m.double_sided, m.double_sided_count = self.ds.ctypes.data, self.ds.size
        self.c = m


def eval_settings(screen: float, limit: float, views: Sequence[int] = (32, 0, 0xB1172026), supersample: int = 8,
                  max_supersample: int = 8, max_changed_area: float = 1.0, force_two_sided: bool = False,
                  conservative_screen: bool = False) -> EvalSettings:
    s = EvalSettings()
    load().blitz_eval_settings_init(C.byref(s), C.sizeof(s))
    s.screen_size, s.limit, s.max_changed_area = screen, limit, max_changed_area
    s.views_orthographic, s.views_perspective, s.views_seed = int(views[0]), int(views[1]), int(views[2])
    s.supersample, s.max_supersample = supersample, max_supersample
    s.force_two_sided, s.conservative_screen = int(force_two_sided), int(conservative_screen)
    return s


def neural_options(**kw) -> NeuralOptionsV2:
    o = NeuralOptionsV2()
    load().blitz_neural_options_v2_init(C.byref(o), C.sizeof(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _check(status: int, err) -> None:
    if status != BLITZ_OK:
        raise BlitzError(status, err.value.decode(errors="replace"))


class AuditSession:
    """Owns the device-resident source, previous LOD, state topology and plans."""

    def __init__(self, source, options: Optional[NeuralOptionsV2] = None):
        self.lib = load()
        self._source = _MeshHold(source)
        self.handle = C.c_void_p()
        err = C.create_string_buffer(512)
        opts = C.byref(options) if options is not None else None
        _check(self.lib.blitz_audit_session_create(C.byref(self._source.c), opts, C.byref(self.handle), err, 512), err)
        self._previous = None

    def close(self) -> None:
        if self.handle:
            self.lib.blitz_audit_session_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def bind_reference(self, previous=None) -> None:
        err = C.create_string_buffer(512)
        self._previous = None if previous is None else _MeshHold(previous)
        ptr = None if previous is None else C.byref(self._previous.c)
        _check(self.lib.blitz_audit_bind_reference(self.handle, ptr, err, 512), err)

    def evaluate(self, reference, candidate, settings: EvalSettings) -> Measurement:
        r, c = _MeshHold(reference), _MeshHold(candidate)
        out = Measurement()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_evaluate(self.handle, C.byref(r.c), C.byref(c.c), C.byref(settings),
                                             C.byref(out), err, 512), err)
        return out

    def rasterize(self, mesh, screen: float, supersample: int, views: Sequence[int], view: int,
                  force_two_sided: bool = False):
        """Packed coverage mask (u64 words), clipped flag and raster side."""
        h = _MeshHold(mesh)
        size = int(np.ceil(screen + 8)) * supersample
        words = np.zeros((size * size + 63) // 64, dtype=np.uint64)
        out_size, clipped = C.c_uint32(), C.c_uint8()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_raster(self.handle, C.byref(h.c), screen, supersample, int(views[0]),
                                           int(views[1]), int(views[2]), view, int(force_two_sided),
                                           words.ctypes.data, words.size, C.byref(out_size), C.byref(clipped),
                                           err, 512), err)
        return words, bool(clipped.value), int(out_size.value)

    def coverage_distance(self, a, b, width: int, height: int, supersample: int) -> float:
        """Coverage distance of two packed host masks (u64 words)."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = C.c_double()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_coverage_distance(self.handle, a.ctypes.data, b.ctypes.data, width, height,
                                                      supersample, 0, C.byref(out), err, 512), err)
        return out.value

    def actions(self) -> np.ndarray:
        count = C.c_size_t()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_actions(self.handle, None, 0, C.byref(count), err, 512), err)
        out = np.zeros(count.value, dtype=COLLAPSE_DTYPE)
        _check(self.lib.blitz_audit_actions(self.handle, out.ctypes.data, out.size, C.byref(count), err, 512), err)
        return out

    def candidates(self, collapses: np.ndarray, gates: Sequence[EvalSettings], measurements: bool = False):
        collapses = np.ascontiguousarray(collapses, dtype=COLLAPSE_DTYPE)
        n = collapses.size
        verdicts = np.zeros(n, dtype=VERDICT_DTYPE)
        meas = np.zeros((n, 4), dtype=MEASUREMENT_DTYPE) if measurements else None
        g = (EvalSettings * 4)(*gates)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_candidates(self.handle, collapses.ctypes.data, n, g, verdicts.ctypes.data,
                                               None if meas is None else meas.ctypes.data, err, 512), err)
        return (verdicts, meas) if measurements else verdicts

    def candidates_device(self, collapses_ptr: int, n: int, gates: Sequence[EvalSettings], verdicts_ptr: int,
                          measurements_ptr: int = 0, stream: int = 0) -> None:
        g = (EvalSettings * 4)(*gates)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_candidates_device(self.handle, collapses_ptr, n, g, verdicts_ptr,
                                                      measurements_ptr or None, stream or None, err, 512), err)

    def execute(self, target_faces: int, trial_budget: int, gates: Sequence[EvalSettings], batch: int = 1,
                keep_permille: int = 0, ranking: int = 3) -> dict:
        """Greedy LOD step on the current state (ShortestEdge ranking), with
        batches of up to `batch` independent collapses per audited trial; with
        `keep_permille` the attached surrogate prunes the ranked edits first."""
        commits = np.zeros(2 * max(16, self._source.idx.size // 3), dtype=np.uint32)
        out = Execution()
        out.struct_size = C.sizeof(Execution)
        g = (EvalSettings * 4)(*gates)
        err = C.create_string_buffer(512)
        if batch == 1 and not keep_permille and ranking == 3:
            _check(self.lib.blitz_audit_execute(self.handle, target_faces, trial_budget, g, commits.ctypes.data,
                                                commits.size // 2, C.byref(out), err, 512), err)
        else:
            opts = ExecuteOptions()
            self.lib.blitz_execute_options_init(C.byref(opts))
            opts.batch = batch
            opts.keep_permille = keep_permille
            opts.ranking = ranking
            _check(self.lib.blitz_audit_execute_ex(self.handle, target_faces, trial_budget, g, C.byref(opts),
                                                   commits.ctypes.data, commits.size // 2, C.byref(out), err, 512),
                   err)
        n = out.commits
        return {"commits": commits[: 2 * n].reshape(-1, 2).copy(), "trials": out.trials,
                "final_faces": out.final_faces, "audited": out.audited, "stop": out.stop_reason,
                "fallbacks": out.fallbacks}

    def chain(self, settings: ChainSettings, meshes: bool = True):
        """LOD chain from the source (blitz_audit_chain): per-level records and,
        with `meshes`, each level's (indices, positions), plus its uv when the
        source has uv (read inside the callback, where the state is the level)."""
        out = (ChainLevel * (settings.levels - 1))()
        emitted = []
        with_uv = self._source.uv is not None

        def on_level(user, level, idx, faces, pos, nv):
            mesh = (np.ctypeslib.as_array(idx, shape=(faces * 3,)).copy(),
                    np.ctypeslib.as_array(pos, shape=(nv * 3,)).reshape(-1, 3).copy())
            emitted.append(mesh + (self.state_uv(),) if with_uv else mesh)

        cb = CHAIN_EMIT(on_level) if meshes else None
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_chain(self.handle, C.byref(settings), out, len(out),
                                          C.cast(cb, C.c_void_p) if cb else None, None, err, 512), err)
        levels = []
        for l in out:
            d = {k: getattr(l, k) for k, _ in l._fields_ if k not in ("struct_size", "reserved", "source_audit",
                                                                      "transition_audit")}
            d["source_audit"] = l.source_audit
            d["transition_audit"] = l.transition_audit
            levels.append(d)
        return levels, emitted

    def surrogate_features(self, screen: float, screen2: float):
        """Features (torch CUDA tensor n x 48) of the current state's legal
        edits, with those edits as midpoint collapses (numpy)."""
        import torch
        count = C.c_size_t()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_surrogate_features(self.handle, screen, screen2, None, None, 0, C.byref(count),
                                                       err, 512), err)
        n = count.value
        feats = torch.zeros((max(n, 1), SURROGATE_FEATURES), dtype=torch.float32, device="cuda")
        cols = np.zeros(max(n, 1), dtype=COLLAPSE_DTYPE)
        _check(self.lib.blitz_audit_surrogate_features(self.handle, screen, screen2, feats.data_ptr(),
                                                       cols.ctypes.data, n, C.byref(count), err, 512), err)
        torch.cuda.synchronize()
        return feats[:n], cols[:n]

    def attach_surrogate(self, model: Optional["Surrogate"]) -> None:
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_attach_surrogate(self.handle, model.handle if model is not None else None,
                                                     err, 512), err)
        self._surrogate = model

    def state(self):
        """Current state: (indices, positions)."""
        faces = C.c_uint32()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_state(self.handle, None, 0, None, 0, C.byref(faces), err, 512), err)
        idx = np.zeros(3 * faces.value, np.uint32)
        pos = np.zeros((self._source.pos.shape[0], 3), np.float32)
        _check(self.lib.blitz_audit_state(self.handle, idx.ctypes.data, idx.size, pos.ctypes.data, pos.size,
                                          C.byref(faces), err, 512), err)
        return idx, pos

    def state_uv(self) -> np.ndarray:
        """Current state's uv per vertex slot (uv transported by commits)."""
        err = C.create_string_buffer(512)
        uv = np.zeros((self._source.pos.shape[0], 2), np.float32)
        _check(self.lib.blitz_audit_state_uv(self.handle, uv.ctypes.data, uv.size, err, 512), err)
        return uv

    def reset(self) -> None:
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_reset(self.handle, err, 512), err)

    def profile(self, enable: Optional[int] = None) -> dict:
        """Enables kernel profiling (1 or True: device times and work counters;
        2: device times only, kernels without counters), disables it (0), or
        reads it (None). Enabling resets the totals."""
        if enable is not None:
            assert self.lib.blitz_audit_profile_enable(self.handle, int(enable)) == BLITZ_OK
        p = AuditProfile()
        p.struct_size = C.sizeof(AuditProfile)
        assert self.lib.blitz_audit_profile_read(self.handle, C.byref(p)) == BLITZ_OK
        return {k: getattr(p, k) for k, _ in p._fields_ if k != "struct_size"}

    def info(self) -> dict:
        i = NeuralInfo()
        i.struct_size = C.sizeof(NeuralInfo)
        assert self.lib.blitz_audit_session_info(self.handle, C.byref(i)) == BLITZ_OK
        return {k: getattr(i, k) for k, _ in i._fields_ if k != "struct_size"}


class AuditBatch:
    """Several sessions audited together: one persistent audit launch per plan
    slot over all their (candidate, view) units, optionally replayed from a
    captured CUDA graph and with the warp tier picked by timing both."""

    def __init__(self, sessions: Sequence[AuditSession]):
        self.lib = load()
        self.sessions = list(sessions)
        arr = (C.c_void_p * len(self.sessions))(*[s.handle for s in self.sessions])
        self.handle = C.c_void_p()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_batch_create(arr, len(self.sessions), C.byref(self.handle), err, 512), err)

    def close(self) -> None:
        if self.handle:
            self.lib.blitz_audit_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def candidates_device(self, collapses_ptr: int, counts: Sequence[int], gates: Sequence[EvalSettings],
                          verdicts_ptr: int, flags: int = 0, stream: int = 0) -> None:
        cnt = (C.c_size_t * len(counts))(*counts)
        g = (EvalSettings * 4)(*gates)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_batch_candidates(self.handle, collapses_ptr, cnt, g, verdicts_ptr, flags,
                                                     stream or None, err, 512), err)

    def candidates(self, collapses: Sequence[np.ndarray], gates: Sequence[EvalSettings], flags: int = 0):
        """Host convenience: per-session collapse arrays in, per-session verdicts out."""
        import torch
        counts = [int(c.size) for c in collapses]
        cat = np.concatenate([np.ascontiguousarray(c, dtype=COLLAPSE_DTYPE) for c in collapses])
        dev = torch.from_numpy(cat.view(np.uint8).copy()).cuda()
        out = torch.zeros(max(1, cat.size) * VERDICT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        self.candidates_device(dev.data_ptr(), counts, gates, out.data_ptr(), flags)
        v = out.cpu().numpy().view(VERDICT_DTYPE)[: cat.size]
        return np.split(v, np.cumsum(counts)[:-1])

    def candidates_host(self, collapses: np.ndarray, counts: Sequence[int], gates: Sequence[EvalSettings],
                        out: np.ndarray, flags: int = 0) -> np.ndarray:
        """Host entry point: concatenated collapses (COLLAPSE_DTYPE) in, verdicts
        (VERDICT_DTYPE, same length) written to `out`; pinned arrays copy fastest."""
        assert collapses.dtype == COLLAPSE_DTYPE and out.dtype == VERDICT_DTYPE and out.size >= collapses.size
        cnt = (C.c_size_t * len(counts))(*counts)
        g = (EvalSettings * 4)(*gates)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_audit_batch_candidates_host(self.handle, collapses.ctypes.data, cnt, g,
                                                          out.ctypes.data, flags, err, 512), err)
        return out

    def info(self) -> dict:
        i = BatchInfo()
        i.struct_size = C.sizeof(BatchInfo)
        assert self.lib.blitz_audit_batch_read_info(self.handle, C.byref(i)) == BLITZ_OK
        d = {k: getattr(i, k) for k, _ in i._fields_ if k != "struct_size"}
        for k in ("tune_ms", "tier_units", "tier_cycles", "phase_cycles", "region_split", "tier_max_cycles", "tier_ms"):
            d[k] = list(getattr(i, k))
        return d


SURROGATE_FEATURES = 48
SURROGATE_PARAMS = 26896


class Surrogate:
    """The learned audit surrogate (48 -> 128 -> 128 -> 2 BF16 MLP) on one GPU.
    Device arrays are torch CUDA tensors (float32, contiguous)."""

    def __init__(self, seed: int = 1, device: int = 0):
        self.lib = load()
        self.handle = C.c_void_p()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_create(device, seed, C.byref(self.handle), err, 512), err)

    def close(self) -> None:
        if self.handle:
            self.lib.blitz_surrogate_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def parameters(self):
        p = np.zeros(SURROGATE_PARAMS, np.float32)
        mean = np.zeros(SURROGATE_FEATURES, np.float32)
        inv = np.zeros(SURROGATE_FEATURES, np.float32)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_save(self.handle, p.ctypes.data, p.size, mean.ctypes.data, inv.ctypes.data,
                                             err, 512), err)
        return p, mean, inv

    def load(self, params, mean=None, inv_std=None) -> None:
        p = np.ascontiguousarray(params, np.float32)
        m = None if mean is None else np.ascontiguousarray(mean, np.float32)
        v = None if inv_std is None else np.ascontiguousarray(inv_std, np.float32)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_load(self.handle, p.ctypes.data, p.size, None if m is None else m.ctypes.data,
                                             None if v is None else v.ctypes.data, err, 512), err)

    def score(self, features):
        import torch
        n = features.shape[0]
        out = torch.empty((max(n, 1), 2), dtype=torch.float32, device=features.device)
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_score(self.handle, features.data_ptr(), n, out.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream, err, 512), err)
        return out[:n]

    def gradients(self, features, labels):
        g = np.zeros(SURROGATE_PARAMS, np.float32)
        loss = C.c_float()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_gradients(self.handle, features.data_ptr(), labels.data_ptr(),
                                                  features.shape[0], g.ctypes.data, g.size, C.byref(loss), err, 512),
               err)
        return g, loss.value

    def train_step(self, features, labels, lr: float) -> float:
        import torch
        loss = C.c_float()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_surrogate_train_step(self.handle, features.data_ptr(), labels.data_ptr(),
                                                   features.shape[0], lr, C.byref(loss),
                                                   torch.cuda.current_stream().cuda_stream, err, 512), err)
        return loss.value


def evaluate(reference, candidate, settings: EvalSettings, session: Optional[AuditSession] = None) -> Measurement:
    """blitz::evaluate on the GPU. The session supplies bounds (of its source)."""
    own = session is None
    s = session or AuditSession(reference)
    try:
        return s.evaluate(reference, candidate, settings)
    finally:
        if own:
            s.close()


def midpoint_collapses(actions: np.ndarray) -> np.ndarray:
    out = np.zeros(actions.size, dtype=COLLAPSE_DTYPE)
    out["from"], out["to"] = actions["from"], actions["to"]
    return out


def four_gates(search: EvalSettings, audit: EvalSettings, source_limit: float, transition_limit: float):
    """Gate settings in the reference order: source@search, previous@search,
    source@audit, previous@audit (generate.cpp:365-388); the search gates use
    max_changed_area = 1 (chain.cpp:187)."""
    gates = []
    for base, is_audit in ((search, False), (audit, True)):
        for limit in (source_limit, transition_limit):
            g = EvalSettings()
            C.memmove(C.byref(g), C.byref(base), C.sizeof(EvalSettings))
            g.limit = limit
            if not is_audit:
                g.max_changed_area = 1.0
            gates.append(g)
    return gates


def settings(**kw) -> Settings:
    """blitz_settings with the reference's defaults, fields overridden by `kw`
    (`transition` as a sequence of (x, y) points)."""
    c = Settings()
    if load().blitz_settings_init(C.byref(c), C.sizeof(c)) != BLITZ_OK:
        raise BlitzError(BLITZ_INVALID_ARGUMENT, "blitz_settings_init")
    curve = kw.pop("transition", None)
    for k, v in kw.items():
        setattr(c, k, v)
    if curve is not None:
        pts = (CurvePoint * len(curve))(*[CurvePoint(float(x), float(y)) for x, y in curve])
        c._curve = pts  # kept alive with the settings
        c.transition, c.transition_count = C.cast(pts, C.c_void_p), len(curve)
    return c


class NeuralModel:
    """A BLZNET policy file loaded through blitz_neural_model_load_v2."""

    def __init__(self, path, options: Optional[NeuralOptionsV2] = None):
        self.lib = load()
        self.handle = C.c_void_p()
        opts = options if options is not None else neural_options()
        err = C.create_string_buffer(512)
        _check(self.lib.blitz_neural_model_load_v2(str(path).encode(), C.byref(opts), C.byref(self.handle), err, 512),
               err)

    @property
    def sha256(self) -> str:
        return self.lib.blitz_neural_model_sha256(self.handle).decode()

    def close(self) -> None:
        if self.handle:
            self.lib.blitz_neural_model_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_neural(mesh, config: Settings, model: NeuralModel, save_to=None) -> dict:
    """blitz_generate_neural: every scheduled level (0 = the source) with its
    lod info, indices and positions; runtime levels, storage, diagnostics and
    per-level action proposals. With `save_to`, the chain is also exported
    there (blitz_result_save_chain: chain.gltf, chain.bin, lods.json)."""
    lib = load()
    hold = _MeshHold(mesh)
    res = C.c_void_p()
    err = C.create_string_buffer(512)
    _check(lib.blitz_generate_neural(C.byref(hold.c), C.byref(config), model.handle, C.byref(res), err, 512), err)
    try:
        if save_to is not None:
            _check(lib.blitz_result_save_chain(res, str(save_to).encode(), err, 512), err)
        lods = []
        for i in range(lib.blitz_result_lod_count(res)):
            info = LodInfo()
            info.struct_size = C.sizeof(LodInfo)
            assert lib.blitz_result_lod(res, i, C.byref(info)) == BLITZ_OK
            m = info.mesh
            idx = np.ctypeslib.as_array(C.cast(m.indices, C.POINTER(C.c_uint32)), shape=(m.index_count,)).copy()
            pos = np.ctypeslib.as_array(C.cast(m.positions.data, C.POINTER(C.c_float)),
                                        shape=(m.positions.count * 3,)).reshape(-1, 3).copy()
            d = {k: getattr(info, k) for k, _ in info._fields_ if k not in ("struct_size", "mesh")}
            d["indices"], d["positions"] = idx, pos
            lods.append(d)
        runtime = [lib.blitz_result_runtime_lod_index(res, i) for i in range(lib.blitz_result_runtime_lod_count(res))]
        st = StorageInfo()
        st.struct_size = C.sizeof(StorageInfo)
        assert lib.blitz_result_storage(res, C.byref(st)) == BLITZ_OK
        ni = NeuralInfo()
        ni.struct_size = C.sizeof(NeuralInfo)
        assert lib.blitz_result_neural_info(res, C.byref(ni)) == BLITZ_OK
        props = []
        for i in range(lib.blitz_result_neural_action_proposal_count(res)):
            a = ActionProposal()
            a.struct_size, a.version = C.sizeof(ActionProposal), 1
            assert lib.blitz_result_neural_action_proposal(res, i, C.byref(a)) == BLITZ_OK
            props.append({k: getattr(a, k) for k, _ in a._fields_ if k not in ("struct_size", "reserved")})
        return {"lods": lods, "runtime": runtime,
                "storage": {k: getattr(st, k) for k, _ in st._fields_ if k != "struct_size"},
                "info": {k: getattr(ni, k) for k, _ in ni._fields_ if k != "struct_size"}, "proposals": props}
    finally:
        lib.blitz_result_destroy(res)


def _stream_array(stream, dtype, width):
    if not stream.data or not stream.count:
        return None
    n = stream.count * stream.stride // np.dtype(dtype).itemsize
    raw = np.ctypeslib.as_array(C.cast(stream.data, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))), shape=(n,))
    return raw.reshape(stream.count, stream.stride // np.dtype(dtype).itemsize)[:, :width].copy()


def load_mesh(path) -> dict:
    """blitz_mesh_file_load: OBJ, PLY or STL as numpy arrays (positions,
    indices, and normals / uv / colors / materials when the file has them)."""
    lib = load()
    handle = C.c_void_p()
    d = BlitzMesh()
    err = C.create_string_buffer(512)
    _check(lib.blitz_mesh_file_load(str(path).encode(), C.byref(handle), C.byref(d), err, 512), err)
    try:
        out = {"positions": _stream_array(d.positions, np.float32, 3),
               "indices": np.ctypeslib.as_array(C.cast(d.indices, C.POINTER(C.c_uint32)), shape=(d.index_count,)).copy(),
               "normals": _stream_array(d.normals, np.float32, 3), "uv": _stream_array(d.uv, np.float32, 2),
               "colors": _stream_array(d.colors, np.uint8, 4), "materials": None}
        if d.materials:
            out["materials"] = np.ctypeslib.as_array(C.cast(d.materials, C.POINTER(C.c_uint16)),
                                                     shape=(d.material_count,)).copy()
        return out
    finally:
        lib.blitz_mesh_file_destroy(handle)


def save_ply(mesh, path) -> None:
    """blitz_mesh_save_ply of a synthetic.Mesh-like object."""
    hold = _MeshHold(mesh)
    err = C.create_string_buffer(512)
    _check(load().blitz_mesh_save_ply(C.byref(hold.c), str(path).encode(), err, 512), err)

"""ctypes declarations of the two C-ABI libraries (include/jgs2.h and
include/jgs2_scene.h).  The structures mirror the C records field by field."""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int,
                    c_int32, c_int64, c_size_t, c_uint8, c_uint32, c_uint64,
                    c_void_p)

PACKAGE_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.environ.get("JGS2_LIB_DIR") or os.path.join(PACKAGE_ROOT, "lib")

STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "INFEASIBLE_INPUT", 3: "OUT_OF_MEMORY",
    4: "DEVICE_ERROR", 5: "TIMEOUT", 6: "DESTROYED", 7: "UNSUPPORTED",
    8: "NOT_READY",
}


class JGS2Error(RuntimeError):
    """A non-OK jgs2_status with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class ClothInput(Structure):
    _fields_ = [
        ("vertex_count", c_uint32), ("triangle_count", c_uint32),
        ("hinge_count", c_uint32), ("reserved0", c_uint32),
        ("triangle_indices", POINTER(c_uint32)),
        ("triangle_inverse_rest_bases", POINTER(c_float)),
        ("triangle_rest_areas", POINTER(c_float)),
        ("hinge_indices", POINTER(c_uint32)),
        ("hinge_rest_angles", POINTER(c_float)),
        ("hinge_rest_edge_lengths", POINTER(c_float)),
        ("young_modulus", c_float), ("poisson_ratio", c_float),
        ("thickness", c_float), ("bending_stiffness", c_float),
    ]


class ContactSurface(Structure):
    _fields_ = [
        ("triangle_count", c_uint32), ("reserved0", c_uint32),
        ("triangles", POINTER(c_uint32)), ("candidate_capacity", c_uint64),
    ]


LAUNCH_SHAPES = 3


class LaunchShape(Structure):
    _fields_ = [("shape", c_uint32), ("solve_vertices_per_block", c_uint32), ("tuning", c_uint32),
                ("samples", c_uint32), ("frame_ms", c_double * LAUNCH_SHAPES)]


class OracleDiagnostics(Structure):
    _fields_ = [(name, c_double) for name in (
        "energy", "inertia", "elasticity", "external_force", "quadratic_target", "floor_contact",
        "inertia_gradient_norm", "material_gradient_norm", "external_force_gradient_norm", "target_gradient_norm",
        "contact_gradient_norm", "gradient_norm", "gradient_squared_norm", "residual_denominator",
        "relative_residual", "maximum_update", "minimum_deformation_determinant", "minimum_contact_distance")] + [
        (name, c_uint32) for name in (
            "active_vertex_count", "active_contact_count", "relative_residual_valid", "gradient_valid",
            "maximum_update_valid", "minimum_deformation_determinant_valid", "minimum_contact_distance_valid",
            "finite")]


class Input(Structure):
    _fields_ = [
        ("vertex_count", c_uint32), ("tet_count", c_uint32),
        ("cubature_k", c_uint32), ("reserved0", c_uint32),
        ("positions", POINTER(c_float)), ("velocities", POINTER(c_float)),
        ("vertex_rest", POINTER(c_float)), ("vertex_colors", POINTER(c_float)),
        ("vertex_info", POINTER(c_uint32)),
        ("external_forces", POINTER(c_float)),
        ("target_positions", POINTER(c_float)),
        ("target_stiffnesses", POINTER(c_float)),
        ("tet_indices", POINTER(c_uint32)), ("tet_inverse_dm", POINTER(c_float)),
        ("tet_meta", POINTER(c_float)), ("tet_rest_stiffness", POINTER(c_float)),
        ("adjacency", POINTER(c_uint32)), ("adjacency_length", c_uint64),
        ("cubature_tet_ids", POINTER(c_uint32)),
        ("cubature_weights", POINTER(c_float)),
        ("cubature_basis", POINTER(c_float)),
        ("cloth", POINTER(ClothInput)),
        ("contact_indices", POINTER(c_uint32)),
        ("contact_vertex_triangle_count", c_uint32),
        ("contact_edge_edge_count", c_uint32),
        ("contact_surface", POINTER(ContactSurface)),
    ]


SETTINGS_FIELDS = [
    ("schedule", c_uint32), ("iterations", c_uint32), ("timestep", c_float),
    ("gravity", c_float * 3), ("floor_height", c_float),
    ("floor_stiffness", c_float), ("velocity_damping", c_float),
    ("regularization", c_float), ("rotation_epsilon", c_float),
    ("max_step", c_float), ("residual_tolerance", c_float),
    ("normalized_update_tolerance", c_float),
    ("contact_tangential_damping", c_float), ("contact_margin", c_float),
    ("ipc_activation_distance", c_float), ("ipc_minimum_distance", c_float),
    ("ipc_barrier_stiffness", c_float), ("ipc_friction_coefficient", c_float),
    ("ipc_friction_velocity_epsilon", c_float), ("ipc_step_safety", c_float),
    ("horizontal_body_correction", c_uint32), ("parity_mode", c_uint32),
]


class Settings(Structure):
    _fields_ = SETTINGS_FIELDS


# Bit i of an override mask selects SETTINGS_FIELDS[i].
SETTINGS_BITS = {name: 1 << i for i, (name, _t) in enumerate(SETTINGS_FIELDS)}


class Info(Structure):
    _fields_ = [
        ("vertex_count", c_uint32), ("tet_count", c_uint32),
        ("cubature_k", c_uint32), ("body_count", c_uint32),
        ("schedule_color_count", c_uint32), ("globalization_enabled", c_uint32),
        ("objective_flags", c_uint32), ("external_force_vertex_count", c_uint32),
        ("quadratic_target_vertex_count", c_uint32),
        ("objective_revision", c_uint32),
        ("last_submitted_iterations", c_uint32), ("history_count", c_uint32),
        ("scene_scale", c_float), ("preprocessing_timestep", c_float),
        ("current_position_buffer", c_uint32), ("cloth_triangle_count", c_uint32),
        ("contact_candidate_count", c_uint32), ("contact_candidate_capacity", c_uint32),
    ]


PROFILE_KINDS = 9


class KernelProfile(Structure):
    _fields_ = [
        ("kinds", c_uint32), ("launches", c_uint32 * PROFILE_KINDS),
        ("milliseconds", c_double * PROFILE_KINDS), ("names", (ctypes.c_char * 24) * PROFILE_KINDS),
    ]


class ServerOptions(Structure):
    _fields_ = [("device", c_int), ("memory_budget_bytes", c_uint64), ("max_scenes_per_wave", c_uint32),
                ("max_waves", c_uint32)]


class RequestResult(Structure):
    _fields_ = [
        ("id", c_uint64), ("status", c_int), ("frames", c_uint32), ("vertex_count", c_uint32),
        ("wave_scenes", c_uint32), ("submit_seconds", c_double), ("admit_seconds", c_double),
        ("finish_seconds", c_double), ("mean_frame_ms", c_double), ("max_frame_ms", c_double),
    ]


class ServerStats(Structure):
    _fields_ = [
        ("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64),
        ("waves_created", c_uint64), ("rounds", c_uint64),
        ("resident_bytes", c_uint64), ("peak_resident_bytes", c_uint64),
        ("waves_in_flight", c_uint32), ("queued", c_uint32), ("busy_seconds", c_double),
    ]


class PrecomputeOptions(Structure):
    _fields_ = [
        ("timestep", c_double), ("cubature_k", c_uint32), ("method", c_uint32),
        ("patch_radius", c_uint32), ("threads", c_uint32),
        ("mode_count", c_uint32), ("inverse_iterations", c_uint32),
        ("training_amplitude", c_double), ("refinement_passes", c_uint32),
        ("exact_complement", c_uint32), ("selection_device", c_uint32),
    ]


class PrecomputeStats(Structure):
    _fields_ = [
        ("source_vertices", c_uint32), ("training_classes", c_uint32),
        ("records_written", c_uint32), ("max_records_per_vertex", c_uint32),
        ("max_residual", c_double), ("mean_residual", c_double),
        ("vertices_over_tolerance", c_uint32),
        ("reduced_amplitude_classes", c_uint32), ("seconds", c_double),
        ("selection_on_gpu", c_uint32), ("selection_batches", c_uint32),
        ("training_seconds", c_double), ("selection_seconds", c_double),
    ]


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(LIB_DIR, name)
    if not os.path.exists(path):
        raise OSError(
            f"{path} is missing; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` "
            "from the repository root")
    return ctypes.CDLL(path)


_scene_lib = None
_step_lib = None


def scene_lib() -> ctypes.CDLL:
    global _scene_lib
    if _scene_lib is None:
        lib = _load("libjgs2_scene.so")
        lib.jgs2_scene_new.restype = c_void_p
        lib.jgs2_scene_destroy.argtypes = [c_void_p]
        lib.jgs2_scene_last_error.argtypes = [c_void_p]
        lib.jgs2_scene_last_error.restype = c_char_p
        lib.jgs2_default_precompute_options.argtypes = [POINTER(PrecomputeOptions)]
        lib.jgs2_scene_add_material.argtypes = [c_void_p, c_double, c_double, c_double, c_uint32]
        lib.jgs2_scene_add_material.restype = c_int32
        lib.jgs2_scene_add_cuboid.argtypes = [c_void_p, POINTER(c_uint32), POINTER(c_double),
                                              POINTER(c_double), c_uint32, c_uint32, c_uint32]
        lib.jgs2_scene_add_cuboid.restype = c_int64
        lib.jgs2_scene_add_mesh.argtypes = [c_void_p, c_uint32, POINTER(c_double), c_uint32,
                                            POINTER(c_uint32), POINTER(c_uint32), c_uint32,
                                            POINTER(c_uint8), c_uint32]
        lib.jgs2_scene_add_mesh.restype = c_int64
        lib.jgs2_scene_add_cloth.argtypes = [c_void_p, c_uint32, POINTER(c_double), c_uint32,
                                             POINTER(c_uint32), POINTER(c_uint8), c_uint32, c_double,
                                             c_double, c_double, c_double, c_double]
        lib.jgs2_scene_add_cloth.restype = c_int64
        lib.jgs2_scene_cloth_triangle_count.argtypes = [c_void_p]
        lib.jgs2_scene_cloth_triangle_count.restype = c_uint32
        lib.jgs2_scene_set_rest_positions.argtypes = [c_void_p, POINTER(c_double)]
        lib.jgs2_scene_set_contact.argtypes = [c_void_p, c_uint32]
        lib.jgs2_scene_set_contact_capacity.argtypes = [c_void_p, c_uint64]
        lib.jgs2_build_static_contact_candidates.argtypes = [c_uint32, POINTER(c_uint32), c_uint32,
                                                             POINTER(c_uint32), c_uint64, POINTER(c_uint32),
                                                             POINTER(c_uint32)]
        lib.jgs2_build_static_contact_candidates.restype = c_int64
        lib.jgs2_scene_set_pinned.argtypes = [c_void_p, POINTER(c_uint8)]
        lib.jgs2_scene_vertex_count.argtypes = [c_void_p]
        lib.jgs2_scene_vertex_count.restype = c_uint32
        lib.jgs2_scene_tet_count.argtypes = [c_void_p]
        lib.jgs2_scene_tet_count.restype = c_uint32
        lib.jgs2_scene_rest_positions.argtypes = [c_void_p, POINTER(c_double)]
        lib.jgs2_scene_precompute.argtypes = [c_void_p, POINTER(PrecomputeOptions),
                                              POINTER(PrecomputeStats)]
        lib.jgs2_scene_set_initial_state.argtypes = [c_void_p, POINTER(c_float),
                                                     POINTER(c_float), c_uint32]
        lib.jgs2_scene_set_objectives.argtypes = [c_void_p, POINTER(c_float),
                                                  POINTER(c_float), POINTER(c_float)]
        lib.jgs2_scene_pack.argtypes = [c_void_p, POINTER(Input)]
        _scene_lib = lib
    return _scene_lib


def step_lib() -> ctypes.CDLL:
    global _step_lib
    if _step_lib is None:
        lib = _load("libjgs2.so")
        vp = c_void_p
        S = POINTER(Settings)
        lib.jgs2_version.restype = c_uint32
        lib.jgs2_build_string.restype = c_char_p
        lib.jgs2_global_last_error.restype = c_char_p
        lib.jgs2_default_settings.argtypes = [S]
        lib.jgs2_resolve_settings.argtypes = [S, S, c_uint32, S]
        lib.jgs2_validate_input.argtypes = [POINTER(Input)]
        lib.jgs2_build_vertex_coloring.argtypes = [POINTER(Input), POINTER(c_uint32),
                                                   POINTER(c_uint32)]
        lib.jgs2_create.argtypes = [POINTER(Input), S, c_uint32, c_int, POINTER(vp)]
        lib.jgs2_destroy.argtypes = [vp]
        lib.jgs2_destroy.restype = None
        lib.jgs2_last_error.argtypes = [vp]
        lib.jgs2_last_error.restype = c_char_p
        lib.jgs2_get_info.argtypes = [vp, POINTER(Info)]
        lib.jgs2_get_default_settings.argtypes = [vp, S]
        lib.jgs2_get_last_submitted_settings.argtypes = [vp, S]
        lib.jgs2_step.argtypes = [vp, S, c_uint32]
        lib.jgs2_step_frames.argtypes = [vp, c_uint32, S, c_uint32]
        lib.jgs2_step_exact_iterations.argtypes = [vp, c_uint32, S, c_uint32]
        lib.jgs2_step_frames_exact_iterations.argtypes = [vp, c_uint32, c_uint32, S, c_uint32]
        lib.jgs2_sync.argtypes = [vp]
        lib.jgs2_step_with_gpu_timestamps.argtypes = [vp, c_uint32, c_uint32, S, c_uint32,
                                                      POINTER(KernelProfile)]
        lib.jgs2_set_external_force.argtypes = [vp, c_uint32, POINTER(c_float)]
        lib.jgs2_replace_external_forces.argtypes = [vp, POINTER(c_float)]
        lib.jgs2_clear_external_forces.argtypes = [vp]
        lib.jgs2_set_quadratic_target.argtypes = [vp, c_uint32, POINTER(c_float), c_float]
        lib.jgs2_replace_quadratic_targets.argtypes = [vp, POINTER(c_float), POINTER(c_float)]
        lib.jgs2_release_quadratic_target.argtypes = [vp, c_uint32]
        lib.jgs2_release_all_quadratic_targets.argtypes = [vp]
        for name in ("jgs2_read_positions", "jgs2_read_velocities",
                     "jgs2_read_predicted_positions",
                     "jgs2_read_final_iteration_updates",
                     "jgs2_read_vertex_rotations"):
            getattr(lib, name).argtypes = [vp, POINTER(c_float), c_size_t]
        lib.jgs2_read_globalization.argtypes = [vp, POINTER(c_float), c_size_t,
                                                POINTER(c_float), POINTER(c_float),
                                                c_size_t, POINTER(c_uint32)]
        lib.jgs2_device_positions.argtypes = [vp, POINTER(c_void_p), POINTER(c_void_p)]
        lib.jgs2_export_state.argtypes = [vp, vp, c_size_t, POINTER(c_size_t)]
        lib.jgs2_read_positions_async.argtypes = [vp, POINTER(c_float), c_size_t]
        lib.jgs2_wait_reads.argtypes = [vp]
        lib.jgs2_import_state.argtypes = [vp, vp, c_size_t]
        lib.jgs2_evaluate_contact_features.argtypes = [POINTER(c_float), POINTER(c_uint32), c_uint32,
                                                       POINTER(c_float), POINTER(c_uint32), c_int]
        lib.jgs2_read_contact_candidates.argtypes = [vp, POINTER(c_uint32), c_uint64, POINTER(c_uint64)]
        lib.jgs2_read_oracle_diagnostics.argtypes = [vp, POINTER(OracleDiagnostics), POINTER(c_float), c_size_t,
                                                     POINTER(c_float), c_size_t]
        lib.jgs2_minimum_contact_distance.argtypes = [POINTER(Input), c_double, POINTER(c_double)]
        lib.jgs2_contact_superset_size.argtypes = [POINTER(Input), POINTER(c_uint64)]
        lib.jgs2_evaluate_assembled_candidate.argtypes = [vp, POINTER(c_float), POINTER(c_float), S, c_uint32,
                                                          POINTER(c_float), POINTER(c_float), POINTER(c_float)]
        lib.jgs2_kernel_launch_count.argtypes = [vp]
        lib.jgs2_kernel_launch_count.restype = c_uint64
        for prefix in ("jgs2_", "jgs2_batch_"):
            getattr(lib, prefix + "autotune").argtypes = [vp, c_uint32]
            getattr(lib, prefix + "get_launch_shape").argtypes = [vp, POINTER(LaunchShape)]
            getattr(lib, prefix + "set_launch_shape").argtypes = [vp, c_uint32]
        lib.jgs2_batch_create.argtypes = [POINTER(POINTER(Input)), c_uint32, S, POINTER(c_uint32), c_int,
                                          POINTER(vp)]
        lib.jgs2_batch_destroy.argtypes = [vp]
        lib.jgs2_batch_destroy.restype = None
        lib.jgs2_batch_last_error.argtypes = [vp]
        lib.jgs2_batch_last_error.restype = c_char_p
        lib.jgs2_batch_scene_count.argtypes = [vp]
        lib.jgs2_batch_scene_count.restype = c_uint32
        lib.jgs2_batch_vertex_count.argtypes = [vp]
        lib.jgs2_batch_vertex_count.restype = c_uint32
        lib.jgs2_batch_step_frames.argtypes = [vp, c_uint32, c_uint32, S, POINTER(c_uint32)]
        lib.jgs2_batch_sync.argtypes = [vp]
        lib.jgs2_batch_get_info.argtypes = [vp, c_uint32, POINTER(Info)]
        for name in ("jgs2_batch_read_positions", "jgs2_batch_read_velocities"):
            getattr(lib, name).argtypes = [vp, c_uint32, POINTER(c_float), c_size_t]
        lib.jgs2_batch_read_globalization.argtypes = [vp, c_uint32, POINTER(c_float), c_size_t,
                                                      POINTER(c_float), POINTER(c_float), c_size_t,
                                                      POINTER(c_uint32)]
        lib.jgs2_batch_read_all_positions.argtypes = [vp, POINTER(c_float), c_size_t]
        lib.jgs2_batch_kernel_launch_count.argtypes = [vp]
        lib.jgs2_batch_kernel_launch_count.restype = c_uint64
        lib.jgs2_batch_stream.argtypes = [vp]
        lib.jgs2_batch_stream.restype = c_void_p
        lib.jgs2_batch_set_scene_active.argtypes = [vp, c_uint32, c_uint32]
        lib.jgs2_estimate_device_bytes.argtypes = [POINTER(Input)]
        lib.jgs2_estimate_device_bytes.restype = c_uint64
        lib.jgs2_server_create.argtypes = [POINTER(ServerOptions), POINTER(vp)]
        lib.jgs2_server_destroy.argtypes = [vp]
        lib.jgs2_server_destroy.restype = None
        lib.jgs2_server_last_error.argtypes = [vp]
        lib.jgs2_server_last_error.restype = c_char_p
        lib.jgs2_server_submit.argtypes = [vp, POINTER(Input), S, c_uint32, c_uint32, c_uint32, POINTER(c_uint64)]
        lib.jgs2_server_wait.argtypes = [vp, c_uint64, POINTER(c_float), c_size_t, POINTER(c_float), c_size_t,
                                         POINTER(RequestResult)]
        lib.jgs2_server_drain.argtypes = [vp]
        lib.jgs2_server_get_stats.argtypes = [vp, POINTER(ServerStats)]
        _step_lib = lib
    return _step_lib


def fptr(array):
    """float* of a contiguous float32 numpy array, or NULL for None."""
    if array is None:
        return ctypes.cast(None, POINTER(c_float))
    return array.ctypes.data_as(POINTER(c_float))


def uptr(array):
    if array is None:
        return ctypes.cast(None, POINTER(c_uint32))
    return array.ctypes.data_as(POINTER(c_uint32))


def dptr(array):
    if array is None:
        return ctypes.cast(None, POINTER(c_double))
    return array.ctypes.data_as(POINTER(c_double))

"""Host-side mirror of the reference's `class JGS2GpuSolver`
(src/simulation/gpu/jgs2-solver.ts:905-3051) over the C-ABI in include/jgs2.h.

Method names, argument meaning and error conditions follow the reference:
`JGS2GpuSolver.create(input, settings)`, `step(overrides)`,
`stepFrames(n, overrides)`, `stepExactIterations(n, overrides)`,
`stepFramesExactIterations(frames, n, overrides)`, the objective setters,
`readPositions()` and the other reads, `awaitIdle()` and `destroy()`.  Where
the reference throws RangeError/TypeError this raises `JGS2RangeError`
(a ValueError); device failures raise `JGS2Error`.
"""
from __future__ import annotations

import ctypes
import dataclasses
from ctypes import byref, c_float, c_size_t, c_uint32, c_void_p
from typing import Optional

import numpy as np

from . import _ffi

DEFAULT_SETTINGS_KEYS = [name for name, _t in _ffi.SETTINGS_FIELDS]
SCHEDULES = {"jacobi": 0, "graph-colored-gauss-seidel": 1}
# Settings keys in the reference's camelCase spelling.
CAMEL = {
    "schedule": "schedule", "timestep": "timestep", "gravity": "gravity", "iterations": "iterations",
    "floorHeight": "floor_height", "floorStiffness": "floor_stiffness",
    "velocityDamping": "velocity_damping", "regularization": "regularization",
    "rotationEpsilon": "rotation_epsilon", "maxStep": "max_step",
    "residualTolerance": "residual_tolerance", "normalizedUpdateTolerance": "normalized_update_tolerance",
    "contactTangentialDamping": "contact_tangential_damping", "contactMargin": "contact_margin",
    "ipcActivationDistance": "ipc_activation_distance", "ipcMinimumDistance": "ipc_minimum_distance",
    "ipcBarrierStiffness": "ipc_barrier_stiffness", "ipcFrictionCoefficient": "ipc_friction_coefficient",
    "ipcFrictionVelocityEpsilon": "ipc_friction_velocity_epsilon", "ipcStepSafety": "ipc_step_safety",
    "horizontalBodyCorrection": "horizontal_body_correction", "parityMode": "parity_mode",
}


class JGS2RangeError(_ffi.JGS2Error, ValueError):
    """Invalid argument, input or state (the reference's RangeError/TypeError)."""


def _raise(status: int, message: str):
    if status in (1, 2, 6, 7, 8):
        raise JGS2RangeError(status, message)
    raise _ffi.JGS2Error(status, message)


def settings_struct(overrides: Optional[dict]):
    """(jgs2_settings, mask) for a Partial<JGS2StepSettings> dict."""
    rec = _ffi.Settings()
    mask = 0
    for key, value in (overrides or {}).items():
        name = CAMEL.get(key, key)
        if name not in _ffi.SETTINGS_BITS:
            raise JGS2RangeError(1, f"Unknown JGS2 setting: {key}.")
        if name == "schedule" and isinstance(value, str):
            if value not in SCHEDULES:
                raise JGS2RangeError(1, f"Unknown JGS2 schedule: {value}.")
            value = SCHEDULES[value]
        if name == "gravity":
            rec.gravity[:] = [float(x) for x in value]
        elif name in ("horizontal_body_correction", "parity_mode"):
            if not isinstance(value, (bool, int, np.bool_)):
                raise JGS2RangeError(1, f"{key} must be a boolean.")
            setattr(rec, name, 1 if value else 0)
        elif name in ("schedule", "iterations"):
            value = int(value)
            if value < 0:
                raise JGS2RangeError(1, f"{key} must be nonnegative; got {value}.")
            setattr(rec, name, value)
        else:
            setattr(rec, name, float(value))
        mask |= _ffi.SETTINGS_BITS[name]
    return rec, mask


def settings_dict(rec) -> dict:
    out = {}
    for name, _t in _ffi.SETTINGS_FIELDS:
        value = getattr(rec, name)
        out[name] = list(value) if name == "gravity" else value
    return out


def default_settings() -> dict:
    rec = _ffi.Settings()
    _ffi.step_lib().jgs2_default_settings(byref(rec))
    return settings_dict(rec)


def resolve_settings(overrides: Optional[dict] = None, defaults: Optional[dict] = None) -> dict:
    L = _ffi.step_lib()
    base = None
    if defaults is not None:
        base, _m = settings_struct(defaults)
    o, mask = settings_struct(overrides)
    out = _ffi.Settings()
    st = L.jgs2_resolve_settings(byref(base) if base is not None else None, byref(o), mask, byref(out))
    if st != 0:
        _raise(st, L.jgs2_global_last_error().decode())
    return settings_dict(out)


def build_vertex_coloring(scene_input):
    """buildJGS2InputVertexColoring: (colors uint32[V], colorCount)."""
    L = _ffi.step_lib()
    rec = scene_input.as_ctypes()
    colors = np.zeros(scene_input.vertex_count, dtype=np.uint32)
    count = c_uint32(0)
    st = L.jgs2_build_vertex_coloring(byref(rec), colors.ctypes.data_as(ctypes.POINTER(c_uint32)), byref(count))
    if st != 0:
        _raise(st, L.jgs2_global_last_error().decode())
    return colors, int(count.value)


def minimum_contact_distance(scene_input, positions=None, cutoff=1.0) -> float:
    """The exact (double) minimum distance over the scene's IPC candidates at
    `positions` (4 floats per vertex; default the input's), restricted for a
    contact surface to pairs whose boxes come within `cutoff` (inf if none)."""
    L = _ffi.step_lib()
    inp = scene_input
    if positions is not None:
        inp = dataclasses.replace(scene_input, positions=np.ascontiguousarray(positions, dtype=np.float32).reshape(-1))
    rec = inp.as_ctypes()
    out = ctypes.c_double(0.0)
    st = L.jgs2_minimum_contact_distance(byref(rec), float(cutoff), byref(out))
    if st != 0:
        _raise(st, L.jgs2_global_last_error().decode())
    return float(out.value)


def contact_superset_size(scene_input) -> int:
    """Candidates of the static superset of the input's contact surface."""
    L = _ffi.step_lib()
    rec = scene_input.as_ctypes()
    out = ctypes.c_uint64(0)
    st = L.jgs2_contact_superset_size(byref(rec), byref(out))
    if st != 0:
        _raise(st, L.jgs2_global_last_error().decode())
    return int(out.value)


def validate_input(scene_input):
    L = _ffi.step_lib()
    rec = scene_input.as_ctypes()
    st = L.jgs2_validate_input(byref(rec))
    if st != 0:
        _raise(st, L.jgs2_global_last_error().decode())


class JGS2GpuSolver:
    """One solver = one CUDA stream and its device memory."""

    def __init__(self, handle, lib, vertex_count):
        self._h = handle
        self._L = lib
        self.vertexCount = vertex_count
        self._destroyed = False

    # ---- lifetime ----------------------------------------------------------------
    @classmethod
    def create(cls, scene_input, settings: Optional[dict] = None, device: int = 0) -> "JGS2GpuSolver":
        L = _ffi.step_lib()
        rec = scene_input.as_ctypes()
        s, mask = settings_struct(settings)
        h = c_void_p()
        st = L.jgs2_create(byref(rec), byref(s), mask, int(device), byref(h))
        if st != 0:
            _raise(st, L.jgs2_global_last_error().decode())
        return cls(h, L, scene_input.vertex_count)

    def destroy(self):
        if not self._destroyed and self._h:
            self._L.jgs2_destroy(self._h)
        self._destroyed = True
        self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            msg = self._L.jgs2_last_error(self._h).decode() if self._h else "destroyed"
            _raise(st, msg)

    def _usable(self):
        if self._destroyed:
            raise JGS2RangeError(6, "JGS2GpuSolver has been destroyed.")

    # ---- info ----------------------------------------------------------------------
    def info(self) -> dict:
        self._usable()
        out = _ffi.Info()
        self._check(self._L.jgs2_get_info(self._h, byref(out)))
        return {name: getattr(out, name) for name, _t in _ffi.Info._fields_}

    @property
    def scheduleColorCount(self) -> int:
        return self.info()["schedule_color_count"]

    @property
    def globalizationEnabled(self) -> bool:
        return bool(self.info()["globalization_enabled"])

    @property
    def clothTriangleCount(self) -> int:
        return self.info()["cloth_triangle_count"]

    @property
    def globalizationElementCount(self) -> int:
        """Tets plus cloth triangles (jgs2-solver.ts:959)."""
        i = self.info()
        return i["tet_count"] + i["cloth_triangle_count"]

    @property
    def objectiveActivity(self) -> dict:
        i = self.info()
        return {"flags": i["objective_flags"], "externalForces": bool(i["objective_flags"] & 1),
                "quadraticTargets": bool(i["objective_flags"] & 2),
                "externalForceVertexCount": i["external_force_vertex_count"],
                "quadraticTargetVertexCount": i["quadratic_target_vertex_count"]}

    @property
    def lastSubmittedIterationCount(self) -> int:
        return self.info()["last_submitted_iterations"]

    @property
    def defaultStepSettings(self) -> dict:
        self._usable()
        out = _ffi.Settings()
        self._check(self._L.jgs2_get_default_settings(self._h, byref(out)))
        return settings_dict(out)

    @property
    def lastSubmittedSettings(self) -> dict:
        self._usable()
        out = _ffi.Settings()
        self._check(self._L.jgs2_get_last_submitted_settings(self._h, byref(out)))
        return settings_dict(out)

    def kernelLaunchCount(self) -> int:
        return int(self._L.jgs2_kernel_launch_count(self._h)) if self._h else 0

    # Launch shapes (include/jgs2.h): vertices per block of the local-solve
    # kernel; every shape gives bit-identical results.
    def autotune(self, rounds: int = 3):
        """Time the next rounds x 3 frames stepped, one shape per frame in
        turn, then keep the fastest shape."""
        self._usable()
        self._check(getattr(self._L, "jgs2_" + "autotune")(self._h, int(rounds)))

    def launchShape(self) -> dict:
        self._usable()
        out = _ffi.LaunchShape()
        self._check(getattr(self._L, "jgs2_" + "get_launch_shape")(self._h, byref(out)))
        return dict(shape=int(out.shape), solveVerticesPerBlock=int(out.solve_vertices_per_block),
                    tuning=int(out.tuning), samples=int(out.samples), frameMs=list(out.frame_ms))

    def setLaunchShape(self, shape: int):
        self._usable()
        self._check(getattr(self._L, "jgs2_" + "set_launch_shape")(self._h, int(shape)))

    def exportState(self) -> bytes:
        """The solver's between-frame state as a byte image (positions,
        velocities, objectives, frame records); see jgs2_export_state."""
        self._usable()
        n = c_size_t(0)
        self._check(self._L.jgs2_export_state(self._h, None, 0, byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._check(self._L.jgs2_export_state(self._h, buf, n.value, byref(n)))
        return buf.raw

    def importState(self, image: bytes):
        """Restore an image from exportState of a solver over the same input."""
        self._usable()
        buf = ctypes.create_string_buffer(bytes(image), len(image))
        self._check(self._L.jgs2_import_state(self._h, buf, len(image)))

    def devicePositions(self):
        """(device pointer, cudaStream_t) of the canonical position array."""
        self._usable()
        p, s = c_void_p(), c_void_p()
        self._check(self._L.jgs2_device_positions(self._h, byref(p), byref(s)))
        return p.value, s.value

    # ---- stepping --------------------------------------------------------------------
    def step(self, overrides: Optional[dict] = None):
        self._usable()
        o, m = settings_struct(overrides)
        self._check(self._L.jgs2_step(self._h, byref(o), m))

    def stepFrames(self, frameCount: int, overrides: Optional[dict] = None):
        self._usable()
        o, m = settings_struct(overrides)
        self._check(self._L.jgs2_step_frames(self._h, int(frameCount), byref(o), m))

    def stepExactIterations(self, iterations: int, overrides: Optional[dict] = None):
        self._usable()
        if int(iterations) < 1:
            raise JGS2RangeError(1, f"iterations must be a positive safe integer; got {iterations}.")
        o, m = settings_struct(overrides)
        self._check(self._L.jgs2_step_exact_iterations(self._h, int(iterations), byref(o), m))

    def stepFramesExactIterations(self, frameCount: int, iterations: int, overrides: Optional[dict] = None):
        self._usable()
        if int(iterations) < 1:
            raise JGS2RangeError(1, f"iterations must be a positive safe integer; got {iterations}.")
        o, m = settings_struct(overrides)
        self._check(self._L.jgs2_step_frames_exact_iterations(self._h, int(frameCount), int(iterations),
                                                              byref(o), m))

    def stepWithGpuTimestamps(self, frameCount: int, iterations: int, overrides: Optional[dict] = None) -> dict:
        """Step frames with CUDA events around every kernel; returns
        {kind: (launches, milliseconds)} (waits for the frames)."""
        self._usable()
        o, m = settings_struct(overrides)
        prof = _ffi.KernelProfile()
        self._check(self._L.jgs2_step_with_gpu_timestamps(self._h, int(frameCount), int(iterations), byref(o), m,
                                                          byref(prof)))
        return {prof.names[k].value.decode(): (int(prof.launches[k]), float(prof.milliseconds[k]))
                for k in range(prof.kinds)}

    def awaitIdle(self):
        self._usable()
        self._check(self._L.jgs2_sync(self._h))

    # ---- objectives ---------------------------------------------------------------------
    def setExternalForce(self, vertex: int, force):
        self._usable()
        f = (c_float * 3)(*[float(x) for x in force])
        self._check(self._L.jgs2_set_external_force(self._h, int(vertex), f))

    def replaceExternalForces(self, forces):
        self._usable()
        a = np.ascontiguousarray(forces, dtype=np.float32).reshape(-1)
        if a.size != 3 * self.vertexCount:
            raise JGS2RangeError(1, f"External forces must contain {3 * self.vertexCount} values; got {a.size}.")
        self._check(self._L.jgs2_replace_external_forces(self._h, _ffi.fptr(a)))

    def clearExternalForces(self):
        self._usable()
        self._check(self._L.jgs2_clear_external_forces(self._h))

    def setQuadraticTarget(self, vertex: int, target, stiffness: float):
        self._usable()
        t = (c_float * 3)(*[float(x) for x in target])
        self._check(self._L.jgs2_set_quadratic_target(self._h, int(vertex), t, float(stiffness)))

    def replaceQuadraticTargets(self, targetPositions, targetStiffnesses):
        self._usable()
        p = np.ascontiguousarray(targetPositions, dtype=np.float32).reshape(-1)
        k = np.ascontiguousarray(targetStiffnesses, dtype=np.float32).reshape(-1)
        if p.size != 3 * self.vertexCount:
            raise JGS2RangeError(1, f"Quadratic target positions must contain {3 * self.vertexCount} values; "
                                    f"got {p.size}.")
        if k.size != self.vertexCount:
            raise JGS2RangeError(1, f"Quadratic target stiffnesses must contain {self.vertexCount} values; "
                                    f"got {k.size}.")
        self._check(self._L.jgs2_replace_quadratic_targets(self._h, _ffi.fptr(p), _ffi.fptr(k)))

    def releaseQuadraticTarget(self, vertex: int):
        self._usable()
        self._check(self._L.jgs2_release_quadratic_target(self._h, int(vertex)))

    def releaseAllQuadraticTargets(self):
        self._usable()
        self._check(self._L.jgs2_release_all_quadratic_targets(self._h))

    # ---- reads -----------------------------------------------------------------------------
    def _read(self, fn, per_vertex):
        self._usable()
        out = np.empty(per_vertex * self.vertexCount, dtype=np.float32)
        self._check(fn(self._h, _ffi.fptr(out), out.size))
        return out

    def readOracleDiagnostics(self) -> dict:
        """readOracleDiagnostics: the exact all-element implicit-Euler oracle
        at the current pose (summary in the reference's field names, plus
        'vertexRecords' (V, 9, 4) and 'tetRecords' (T, 4) float32)."""
        self._usable()
        info = self.info()
        V, T = info["vertex_count"], info["tet_count"]
        out = _ffi.OracleDiagnostics()
        vrec = np.zeros(36 * max(V, 1), dtype=np.float32)
        trec = np.zeros(4 * max(T, 1), dtype=np.float32)
        self._check(self._L.jgs2_read_oracle_diagnostics(self._h, byref(out), _ffi.fptr(vrec), vrec.size,
                                                         _ffi.fptr(trec), trec.size))
        d = {name: getattr(out, name) for name, _t in _ffi.OracleDiagnostics._fields_}
        summary = {
            "energy": d["energy"],
            "components": {"inertia": d["inertia"], "elasticity": d["elasticity"],
                           "externalForce": d["external_force"], "quadraticTarget": d["quadratic_target"],
                           "floorContact": d["floor_contact"]},
            "componentGradientNorms": {"inertia": d["inertia_gradient_norm"],
                                       "material": d["material_gradient_norm"],
                                       "externalForce": d["external_force_gradient_norm"],
                                       "target": d["target_gradient_norm"], "contact": d["contact_gradient_norm"]},
            "gradientNorm": d["gradient_norm"], "residualNumerator": d["gradient_norm"],
            "relativeResidual": d["relative_residual"], "relativeResidualValid": bool(d["relative_residual_valid"]),
            "residualDenominator": d["residual_denominator"], "gradientSquaredNorm": d["gradient_squared_norm"],
            "gradientValid": bool(d["gradient_valid"]), "maximumUpdate": d["maximum_update"],
            "maximumUpdateValid": bool(d["maximum_update_valid"]),
            "minimumDeformationDeterminant": d["minimum_deformation_determinant"],
            "minimumDeformationDeterminantValid": bool(d["minimum_deformation_determinant_valid"]),
            "minimumContactDistance": d["minimum_contact_distance"],
            "minimumContactDistanceValid": bool(d["minimum_contact_distance_valid"]),
            "activeContactCount": d["active_contact_count"], "activeVertexCount": d["active_vertex_count"],
            "finite": bool(d["finite"]),
            "vertexRecords": vrec[:36 * V].reshape(V, 9, 4), "tetRecords": trec[:4 * T].reshape(T, 4),
        }
        return summary

    @property
    def contactCandidateCount(self) -> int:
        """Static candidates, or the broad phase's listing of the last iteration."""
        return self.info()["contact_candidate_count"]

    def readContactCandidates(self) -> np.ndarray:
        """The IPC candidates of the last iteration, (n, 4) uint32 in
        canonical order (vertex-triangle rows first)."""
        self._usable()
        n = ctypes.c_uint64(0)
        self._check(self._L.jgs2_read_contact_candidates(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(4 * max(n.value, 1), dtype=np.uint32)
        self._check(self._L.jgs2_read_contact_candidates(self._h, _ffi.uptr(out), n.value, ctypes.byref(n)))
        return out[:4 * n.value].reshape(-1, 4)

    def readPositions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Positions (4 floats per vertex); `out` may be a caller-owned
        (e.g. pinned) float32 array to read into."""
        if out is None:
            return self._read(self._L.jgs2_read_positions, 4)
        self._usable()
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < 4 * self.vertexCount:
            raise JGS2RangeError(1, "out must be a contiguous float32 array with 4 floats per vertex.")
        self._check(self._L.jgs2_read_positions(self._h, _ffi.fptr(out), out.size))
        return out

    def readPositionsAsync(self, out: np.ndarray) -> np.ndarray:
        """Enqueue a read of the positions into `out` (contiguous float32,
        4 floats per vertex, ideally page-locked) after the submitted work
        and return at once; `out` holds the positions after awaitReads()."""
        self._usable()
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < 4 * self.vertexCount:
            raise JGS2RangeError(1, "out must be a contiguous float32 array with 4 floats per vertex.")
        self._check(self._L.jgs2_read_positions_async(self._h, _ffi.fptr(out), out.size))
        return out

    def awaitReads(self):
        """Wait for every asynchronous read submitted so far."""
        self._usable()
        self._check(self._L.jgs2_wait_reads(self._h))

    def readVelocities(self) -> np.ndarray:
        return self._read(self._L.jgs2_read_velocities, 4)

    def readPredictedPositions(self) -> np.ndarray:
        return self._read(self._L.jgs2_read_predicted_positions, 4)

    def readFinalIterationUpdates(self) -> np.ndarray:
        return self._read(self._L.jgs2_read_final_iteration_updates, 4)

    def readVertexRotations(self) -> np.ndarray:
        return self._read(self._L.jgs2_read_vertex_rotations, 12)

    def evaluateAssembledCandidateForTest(self, sourcePositions, candidatePositions,
                                          overrides: Optional[dict] = None) -> dict:
        """Run the assembled gate and convergence reduction once on a source /
        candidate pose pair; {'positions', 'control', 'history'}."""
        self._usable()
        src = np.ascontiguousarray(sourcePositions, dtype=np.float32).reshape(-1)
        cand = np.ascontiguousarray(candidatePositions, dtype=np.float32).reshape(-1)
        n = 4 * self.vertexCount
        if src.size != n or cand.size != n:
            raise JGS2RangeError(1, f"Assembled candidate poses must each contain {n} floats.")
        o, m = settings_struct(overrides)
        pos = np.empty(n, dtype=np.float32)
        control = np.empty(16, dtype=np.float32)
        history = np.empty(32, dtype=np.float32)
        self._check(self._L.jgs2_evaluate_assembled_candidate(
            self._h, _ffi.fptr(src), _ffi.fptr(cand), byref(o), m, _ffi.fptr(pos), _ffi.fptr(control),
            _ffi.fptr(history)))
        return {"positions": pos, "control": control, "history": history}

    def readGlobalizationDiagnostics(self) -> dict:
        """{'local': (V,16), 'control': (16,), 'history': (count,32), 'historyCount': n}: the raw
        records.  jgs2_b200.diagnostics.decode_globalization(result) gives the reference's
        decoded form (named fields, zero sentinels, validity flags)."""
        self._usable()
        local = np.empty(16 * self.vertexCount, dtype=np.float32)
        control = np.empty(16, dtype=np.float32)
        history = np.empty(32 * 64, dtype=np.float32)
        count = c_uint32(0)
        self._check(self._L.jgs2_read_globalization(self._h, _ffi.fptr(local), local.size, _ffi.fptr(control),
                                                    _ffi.fptr(history), history.size, byref(count)))
        n = int(count.value)
        return {"local": local.reshape(-1, 16), "control": control,
                "history": history.reshape(64, 32)[:n], "historyCount": n}


class JGS2Batch:
    """Many independent scenes stepped together (include/jgs2.h, batched form).

    Each scene keeps the solver's semantics (own settings, own assembled gate,
    convergence history and stop latch); `stepFrames` advances all of them with
    one launch sequence.  Per-scene reads mirror JGS2GpuSolver's."""

    def __init__(self, handle, lib, vertex_counts):
        self._h = handle
        self._L = lib
        self.vertexCounts = list(vertex_counts)
        self._destroyed = False

    @classmethod
    def create(cls, scene_inputs, settings=None, device: int = 0) -> "JGS2Batch":
        """settings: None, one dict for every scene, or a list of dicts."""
        L = _ffi.step_lib()
        n = len(scene_inputs)
        if n == 0:
            raise JGS2RangeError(1, "A batch needs at least one scene.")
        recs = [inp.as_ctypes() for inp in scene_inputs]
        ptrs = (ctypes.POINTER(_ffi.Input) * n)(*[ctypes.pointer(r) for r in recs])
        per = settings if isinstance(settings, (list, tuple)) else [settings] * n
        structs = (_ffi.Settings * n)()
        masks = (c_uint32 * n)()
        for i, o in enumerate(per):
            s, m = settings_struct(o)
            structs[i] = s
            masks[i] = m
        h = c_void_p()
        st = L.jgs2_batch_create(ptrs, n, structs, masks, int(device), byref(h))
        if st != 0:
            _raise(st, L.jgs2_global_last_error().decode())
        return cls(h, L, [inp.vertex_count for inp in scene_inputs])

    def destroy(self):
        if not self._destroyed and self._h:
            self._L.jgs2_batch_destroy(self._h)
        self._destroyed = True
        self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            msg = self._L.jgs2_batch_last_error(self._h).decode() if self._h else "destroyed"
            _raise(st, msg)

    def _usable(self):
        if self._destroyed:
            raise JGS2RangeError(6, "JGS2 batch has been destroyed.")

    @property
    def sceneCount(self) -> int:
        return len(self.vertexCounts)

    def kernelLaunchCount(self) -> int:
        return int(self._L.jgs2_batch_kernel_launch_count(self._h)) if self._h else 0

    # Launch shapes (include/jgs2.h): vertices per block of the local-solve
    # kernel; every shape gives bit-identical results.
    def autotune(self, rounds: int = 3):
        """Time the next rounds x 3 frames stepped, one shape per frame in
        turn, then keep the fastest shape."""
        self._usable()
        self._check(getattr(self._L, "jgs2_batch_" + "autotune")(self._h, int(rounds)))

    def launchShape(self) -> dict:
        self._usable()
        out = _ffi.LaunchShape()
        self._check(getattr(self._L, "jgs2_batch_" + "get_launch_shape")(self._h, byref(out)))
        return dict(shape=int(out.shape), solveVerticesPerBlock=int(out.solve_vertices_per_block),
                    tuning=int(out.tuning), samples=int(out.samples), frameMs=list(out.frame_ms))

    def setLaunchShape(self, shape: int):
        self._usable()
        self._check(getattr(self._L, "jgs2_batch_" + "set_launch_shape")(self._h, int(shape)))

    def stream(self) -> int:
        """The batch's cudaStream_t as an integer handle."""
        self._usable()
        return int(self._L.jgs2_batch_stream(self._h) or 0)

    def stepFrames(self, frameCount: int = 1, exactIterations: int = 0, overrides=None):
        """exactIterations 0: production step; overrides: None, a dict for
        every scene, or a list of dicts."""
        self._usable()
        n = self.sceneCount
        per = overrides if isinstance(overrides, (list, tuple)) else [overrides] * n
        structs = (_ffi.Settings * n)()
        masks = (c_uint32 * n)()
        for i, o in enumerate(per):
            s, m = settings_struct(o)
            structs[i] = s
            masks[i] = m
        self._check(self._L.jgs2_batch_step_frames(self._h, int(frameCount), int(exactIterations), structs, masks))

    def awaitIdle(self):
        self._usable()
        self._check(self._L.jgs2_batch_sync(self._h))

    def info(self, scene: int) -> dict:
        self._usable()
        out = _ffi.Info()
        self._check(self._L.jgs2_batch_get_info(self._h, int(scene), byref(out)))
        return {name: getattr(out, name) for name, _t in _ffi.Info._fields_}

    def _read(self, fn, scene, per_vertex):
        self._usable()
        out = np.empty(per_vertex * self.vertexCounts[scene], dtype=np.float32)
        self._check(fn(self._h, int(scene), _ffi.fptr(out), out.size))
        return out

    def readPositions(self, scene: int) -> np.ndarray:
        return self._read(self._L.jgs2_batch_read_positions, scene, 4)

    def readVelocities(self, scene: int) -> np.ndarray:
        return self._read(self._L.jgs2_batch_read_velocities, scene, 4)

    def readAllPositions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        self._usable()
        total = 4 * sum(self.vertexCounts)
        if out is None:
            out = np.empty(total, dtype=np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size < total:
            raise JGS2RangeError(1, "out must be a contiguous float32 array with 4 floats per vertex.")
        self._check(self._L.jgs2_batch_read_all_positions(self._h, _ffi.fptr(out), out.size))
        return out

    def readGlobalizationDiagnostics(self, scene: int) -> dict:
        self._usable()
        V = self.vertexCounts[scene]
        local = np.empty(16 * V, dtype=np.float32)
        control = np.empty(16, dtype=np.float32)
        history = np.empty(32 * 64, dtype=np.float32)
        count = c_uint32(0)
        self._check(self._L.jgs2_batch_read_globalization(self._h, int(scene), _ffi.fptr(local), local.size,
                                                          _ffi.fptr(control), _ffi.fptr(history), history.size,
                                                          byref(count)))
        n = int(count.value)
        return {"local": local.reshape(-1, 16), "control": control,
                "history": history.reshape(64, 32)[:n], "historyCount": n}

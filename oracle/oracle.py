"""Python handle on the CPU oracle — TEST INFRASTRUCTURE, not product code.

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's
cpu_baseline leg use this module.  It wraps oracle/libjgs2_oracle.so (a CPU
restatement of the reference's WGSL step, see jgs2_oracle.cpp) and restates
the reference's settings defaults and resolution
(DEFAULT_JGS2_STEP_SETTINGS and resolveJGS2StepSettings,
src/simulation/gpu/jgs2-solver.ts:164-187, 531-550) so the checker does not
depend on the product library for them.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_float, c_int, c_uint32, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjgs2_oracle.so")

DEFAULT_SETTINGS = dict(
    schedule=0, iterations=9, timestep=1 / 60, gravity=(0.0, -9.81, 0.0),
    floor_height=0.0, floor_stiffness=20000.0, velocity_damping=0.999,
    regularization=1e-6, rotation_epsilon=1e-7, max_step=0.1,
    residual_tolerance=1e-3, normalized_update_tolerance=1e-3,
    contact_tangential_damping=8.0, contact_margin=0.01,
    ipc_activation_distance=0.05, ipc_minimum_distance=0.001,
    ipc_barrier_stiffness=0.0, ipc_friction_coefficient=0.0,
    ipc_friction_velocity_epsilon=0.01, ipc_step_safety=0.9,
    horizontal_body_correction=1, parity_mode=0,
)


def resolve_settings(defaults=None, **overrides) -> dict:
    """Merge overrides into defaults and apply the parity override."""
    merged = dict(DEFAULT_SETTINGS if defaults is None else defaults)
    merged.update(overrides)
    if merged["parity_mode"]:
        merged.update(velocity_damping=1.0, contact_tangential_damping=0.0,
                      horizontal_body_correction=0)
    return merged


def normalize_odd_iterations(iterations: int) -> int:
    """normalizeOddIterationCount (src/simulation/gpu/layout.ts:742-748)."""
    it = max(1, int(iterations))
    return it + 1 if it % 2 == 0 else it


def ensure_built() -> str:
    if not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        import sys
        pkg = os.path.join(os.path.dirname(HERE), "webgpu-physics_b200")
        if pkg not in sys.path:
            sys.path.insert(0, pkg)
        ensure_built()
        L = ctypes.CDLL(LIB_PATH)
        L.jgs2_oracle_create.restype = c_void_p
        L.jgs2_oracle_create.argtypes = [c_void_p, c_int]
        L.jgs2_oracle_destroy.argtypes = [c_void_p]
        L.jgs2_oracle_set_threads.argtypes = [c_int]
        L.jgs2_oracle_max_threads.restype = c_int
        L.jgs2_oracle_color_count.argtypes = [c_void_p]
        L.jgs2_oracle_color_count.restype = c_uint32
        L.jgs2_oracle_colors.argtypes = [c_void_p, POINTER(c_uint32)]
        L.jgs2_oracle_step.argtypes = [c_void_p, c_void_p, c_uint32, c_uint32, c_int]
        L.jgs2_oracle_read.argtypes = [c_void_p, c_int, POINTER(c_float)]
        L.jgs2_oracle_set_objectives.argtypes = [c_void_p, POINTER(c_float), POINTER(c_float),
                                                 POINTER(c_float)]
        L.jgs2_oracle_evaluate_candidate.argtypes = [c_void_p, c_void_p, POINTER(c_float), POINTER(c_float)]
        L.jgs2_oracle_fix_contact.argtypes = [c_void_p, c_void_p]
        _lib = L
    return _lib


def _settings_struct(settings: dict):
    from jgs2_b200 import _ffi  # plain ctypes layout of jgs2_settings
    rec = _ffi.Settings()
    for name, _t in _ffi.SETTINGS_FIELDS:
        value = settings[name]
        if name == "gravity":
            rec.gravity[:] = [float(x) for x in value]
        else:
            setattr(rec, name, value)
    return rec


class OracleSolver:
    """CPU oracle over one scene input (jgs2_b200.scenes.SceneInput)."""

    READS = {"positions": (0, 4), "velocities": (1, 4), "predicted": (2, 4),
             "final_updates": (3, 4), "vertex_rotations": (4, 12), "local": (5, 16),
             "control": (6, None), "history": (7, None), "convergence": (8, 20),
             "vertex_energy": (9, 4)}

    def __init__(self, scene_input, settings: dict | None = None, precision: int = 32):
        self._L = lib()
        self._rec = scene_input.as_ctypes()
        self._h = self._L.jgs2_oracle_create(ctypes.byref(self._rec), precision)
        if not self._h:
            raise RuntimeError("oracle create failed")
        self.vertex_count = scene_input.vertex_count
        self.defaults = resolve_settings(None, **(settings or {}))
        # The IPC parameters the reference fixes at create.
        self._L.jgs2_oracle_fix_contact(self._h, ctypes.byref(_settings_struct(self.defaults)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.jgs2_oracle_destroy(h)
            self._h = None

    @property
    def color_count(self) -> int:
        return int(self._L.jgs2_oracle_color_count(self._h))

    def colors(self) -> np.ndarray:
        out = np.empty(self.vertex_count, dtype=np.uint32)
        self._L.jgs2_oracle_colors(self._h, out.ctypes.data_as(POINTER(c_uint32)))
        return out

    def _run(self, frames, iterations, stop, overrides):
        s = resolve_settings(self.defaults, **overrides)
        rec = _settings_struct(s)
        rc = self._L.jgs2_oracle_step(self._h, ctypes.byref(rec), frames, iterations, 1 if stop else 0)
        if rc != 0:
            raise RuntimeError("oracle step failed")

    def step(self, **overrides):
        s = resolve_settings(self.defaults, **overrides)
        self._run(1, normalize_odd_iterations(s["iterations"]), True, overrides)

    def step_frames(self, frames, **overrides):
        s = resolve_settings(self.defaults, **overrides)
        self._run(frames, normalize_odd_iterations(s["iterations"]), True, overrides)

    def step_exact_iterations(self, iterations, **overrides):
        self._run(1, iterations, False, overrides)

    def step_frames_exact_iterations(self, frames, iterations, **overrides):
        self._run(frames, iterations, False, overrides)

    def evaluate_assembled_candidate(self, source, candidate, **overrides) -> dict:
        """Gate + convergence of one source/candidate pose pair (4 floats per
        vertex); {'positions', 'control', 'history'} like the product call."""
        s = resolve_settings(self.defaults, **overrides)
        rec = _settings_struct(s)
        src = np.ascontiguousarray(source, dtype=np.float32).reshape(-1)
        cand = np.ascontiguousarray(candidate, dtype=np.float32).reshape(-1)
        assert src.size == cand.size == 4 * self.vertex_count
        rc = self._L.jgs2_oracle_evaluate_candidate(self._h, ctypes.byref(rec), src.ctypes.data_as(POINTER(c_float)),
                                                    cand.ctypes.data_as(POINTER(c_float)))
        if rc != 0:
            raise RuntimeError("oracle candidate evaluation failed")
        return {"positions": self.read("positions"), "control": self.read("control"),
                "history": self.read("history")[:32]}

    def read(self, what: str) -> np.ndarray:
        which, per_vertex = self.READS[what]
        n = {"control": 16, "history": 64 * 32}.get(what, (per_vertex or 0) * self.vertex_count)
        out = np.zeros(n, dtype=np.float32)
        self._L.jgs2_oracle_read(self._h, which, out.ctypes.data_as(POINTER(c_float)))
        return out

    def set_objectives(self, forces=None, targets=None, stiffnesses=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32)
                for a in (forces, targets, stiffnesses)]
        ptrs = [ctypes.cast(None, POINTER(c_float)) if a is None else a.ctypes.data_as(POINTER(c_float))
                for a in arrs]
        self._L.jgs2_oracle_set_objectives(self._h, *ptrs)


def set_threads(n: int):
    lib().jgs2_oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().jgs2_oracle_max_threads())

"""Scene construction and the packed step input (the reference's
src/scenes/index.ts + src/simulation/cpu/precompute.ts), driving the native
scene/precompute library through include/jgs2_scene.h.

`SceneInput` is the JGS2GpuInput (src/simulation/gpu/layout.ts:41-90) as numpy
arrays; `SceneInput.as_ctypes()` yields the jgs2_input record the step library
takes.  The named workloads below are the seeded synthetic scenes the
benchmarks and parity tests run on.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os
from ctypes import c_double, c_uint32
from typing import Optional

import numpy as np

from . import _ffi

MATERIAL_COROTATED_LINEAR = 0
MATERIAL_STABLE_NEO_HOOKEAN = 1
PRECOMPUTE_EXACT = 0
PRECOMPUTE_PATCH = 1
# Where the greedy cubature selection runs (same records either way).
SELECTION_CPU, SELECTION_GPU, SELECTION_AUTO = 0, 1, 2
# Revision of the training arithmetic, part of every cubature fingerprint:
# 2 = FP64 evaluated in source order (no multiply-add contraction), the
# rounding the GPU selection shares.
TRAINER_REVISION = 2
CONTACT_NONE, CONTACT_STATIC, CONTACT_SURFACE = 0, 1, 2
FACE_X_MIN, FACE_X_MAX, FACE_Y_MIN, FACE_Y_MAX, FACE_Z_MIN, FACE_Z_MAX = (
    1, 2, 4, 8, 16, 32)
EMPTY_TET = 0xFFFFFFFF


def select_nonnegative_columns(columns, target, max_columns, refinement_passes=4, residual_tolerance=0.01) -> dict:
    """selectGreedyNonnegativeColumns (src/simulation/cpu/cubature.ts:508-690)
    through the cubature trainer's selection core (jgs2_select_nonnegative_columns):
    {'selected': column indices in selection order, 'weights', 'normalizedResidual'}.
    The defaults are the reference's (4 refinement passes, tolerance 0.01)."""
    from ctypes import POINTER, byref

    from .solver import JGS2RangeError

    L = _ffi.scene_lib()
    D = POINTER(c_double)
    L.jgs2_select_nonnegative_columns.argtypes = [D, c_uint32, c_uint32, D, c_uint32, c_uint32, c_double,
                                                  POINTER(c_uint32), D, POINTER(c_uint32), D]
    t = np.ascontiguousarray(target, dtype=np.float64).reshape(-1)
    cols = np.ascontiguousarray(np.asarray(columns, dtype=np.float64).reshape(-1, t.size) if len(columns) else
                                np.zeros((0, t.size)))
    sel = np.zeros(max(1, max_columns), dtype=np.uint32)
    w = np.zeros(max(1, max_columns), dtype=np.float64)
    count, residual = c_uint32(0), c_double(0)
    st = L.jgs2_select_nonnegative_columns(cols.ctypes.data_as(D), cols.shape[0], t.size, t.ctypes.data_as(D),
                                           int(max_columns), int(refinement_passes), float(residual_tolerance),
                                           sel.ctypes.data_as(POINTER(c_uint32)), w.ctypes.data_as(D),
                                           byref(count), byref(residual))
    if st != 0:
        raise JGS2RangeError(st, "Invalid column selection input (sizes, values or settings).")
    n = int(count.value)
    return {"selected": [int(x) for x in sel[:n]], "weights": [float(x) for x in w[:n]],
            "normalizedResidual": float(residual.value)}


def mulberry32(seed: int):
    """createCorpusRandom (src/scenes/phase1.ts:106-115): uniform [0, 1)."""
    state = seed & 0xFFFFFFFF

    def imul(a, b):
        return (a * b) & 0xFFFFFFFF

    def rand():
        nonlocal state
        state = (state + 0x6D2B79F5) & 0xFFFFFFFF
        value = state
        value = imul(value ^ (value >> 15), value | 1)
        value ^= (value + imul(value ^ (value >> 7), value | 61)) & 0xFFFFFFFF
        return ((value ^ (value >> 14)) & 0xFFFFFFFF) / 4294967296.0

    return rand


@dataclasses.dataclass
class SceneInput:
    """JGS2GpuInput as contiguous numpy arrays."""

    vertex_count: int
    tet_count: int
    cubature_k: int
    positions: np.ndarray
    vertex_rest: np.ndarray
    vertex_info: np.ndarray
    tet_indices: np.ndarray
    tet_inverse_dm: np.ndarray
    tet_meta: np.ndarray
    adjacency: np.ndarray
    cubature_tet_ids: np.ndarray
    cubature_weights: np.ndarray
    cubature_basis: np.ndarray
    velocities: Optional[np.ndarray] = None
    vertex_colors: Optional[np.ndarray] = None
    tet_rest_stiffness: Optional[np.ndarray] = None
    external_forces: Optional[np.ndarray] = None
    target_positions: Optional[np.ndarray] = None
    target_stiffnesses: Optional[np.ndarray] = None
    rest_positions: Optional[np.ndarray] = None  # float64 FEM rest shape
    # Triangle cloth (JGS2GpuClothInput, src/simulation/gpu/cloth-layout.ts:88-104).
    cloth_triangles: Optional[np.ndarray] = None       # uint32, 3 per triangle
    cloth_inverse_rest: Optional[np.ndarray] = None    # float32, 4 per triangle
    cloth_rest_areas: Optional[np.ndarray] = None      # float32, 1 per triangle
    hinge_indices: Optional[np.ndarray] = None         # uint32, 4 per hinge
    hinge_rest_angles: Optional[np.ndarray] = None     # float32
    hinge_rest_edge_lengths: Optional[np.ndarray] = None  # float32
    cloth_material: Optional[np.ndarray] = None        # float32 (E, nu, thickness, bending)
    # Static IPC contact candidates: 4 indices each, vertex-triangle first,
    # and their counts (vertex-triangle, edge-edge).
    contact_indices: Optional[np.ndarray] = None       # uint32
    contact_counts: Optional[np.ndarray] = None        # uint32 (vt, ee)
    # Contact surface for the device broad phase instead (3 indices per
    # triangle) and its per-iteration candidate capacity (0: the default).
    contact_surface: Optional[np.ndarray] = None       # uint32
    contact_capacity: int = 0
    stats: Optional[dict] = None

    @property
    def contact_candidate_count(self) -> int:
        return 0 if self.contact_counts is None else int(self.contact_counts.sum())

    @property
    def cloth_triangle_count(self) -> int:
        return 0 if self.cloth_triangles is None else self.cloth_triangles.size // 3

    @property
    def hinge_count(self) -> int:
        return 0 if self.hinge_indices is None else self.hinge_indices.size // 4

    def cloth_ctypes(self):
        """The jgs2_cloth_input record, or None without cloth."""
        if self.cloth_triangles is None:
            return None
        c = _ffi.ClothInput()
        c.vertex_count = self.vertex_count
        c.triangle_count = self.cloth_triangle_count
        c.hinge_count = self.hinge_count
        c.triangle_indices = _ffi.uptr(self.cloth_triangles)
        c.triangle_inverse_rest_bases = _ffi.fptr(self.cloth_inverse_rest)
        c.triangle_rest_areas = _ffi.fptr(self.cloth_rest_areas)
        c.hinge_indices = _ffi.uptr(self.hinge_indices)
        c.hinge_rest_angles = _ffi.fptr(self.hinge_rest_angles)
        c.hinge_rest_edge_lengths = _ffi.fptr(self.hinge_rest_edge_lengths)
        (c.young_modulus, c.poisson_ratio, c.thickness,
         c.bending_stiffness) = (float(x) for x in self.cloth_material)
        return c

    def check_arrays(self):
        """The C-ABI takes plain pointers and sizes every array by the counts
        (vertices, tets, records, candidates, triangles, hinges), so a
        mis-sized, wrongly typed or strided array would be read out of
        bounds or misread.  Refuse such arrays here, before any pointer is
        taken, as the reference's layout validation does ("... must contain
        N values", src/simulation/gpu/layout.ts).  Absent (None) arrays are
        left to the library's own validation."""
        from .solver import JGS2RangeError

        V, T, K = self.vertex_count, self.tet_count, self.cubature_k
        f32, u32 = np.float32, np.uint32
        spec = [("positions", f32, 4 * V), ("velocities", f32, 4 * V), ("vertex_rest", f32, 4 * V),
                ("vertex_colors", f32, 4 * V), ("vertex_info", u32, 4 * V), ("external_forces", f32, 3 * V),
                ("target_positions", f32, 3 * V), ("target_stiffnesses", f32, V), ("tet_indices", u32, 4 * T),
                ("tet_inverse_dm", f32, 12 * T), ("tet_meta", f32, 4 * T), ("tet_rest_stiffness", f32, 144 * T),
                ("adjacency", u32, None), ("cubature_tet_ids", u32, V * K), ("cubature_weights", f32, V * K),
                ("cubature_basis", f32, 36 * V * K)]
        if self.contact_counts is not None and self.contact_candidate_count > 0:
            spec.append(("contact_indices", u32, 4 * self.contact_candidate_count))
        if self.contact_surface is not None:
            spec.append(("contact_surface", u32, 3 * (self.contact_surface.size // 3)))
        if self.cloth_triangles is not None:
            C, H = self.cloth_triangles.size // 3, (0 if self.hinge_indices is None else self.hinge_indices.size // 4)
            spec += [("cloth_triangles", u32, 3 * C), ("cloth_inverse_rest", f32, 4 * C),
                     ("cloth_rest_areas", f32, C), ("hinge_indices", u32, 4 * H), ("hinge_rest_angles", f32, H),
                     ("hinge_rest_edge_lengths", f32, H), ("cloth_material", f32, 4)]
        for name, dtype, size in spec:
            a = getattr(self, name)
            if a is None:
                continue
            label = name.split("_")[0] + "".join(w.capitalize() for w in name.split("_")[1:])
            if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags.c_contiguous:
                raise JGS2RangeError(1, f"{label} must be a contiguous {np.dtype(dtype).name} array.")
            if size is not None and a.size != size:
                raise JGS2RangeError(1, f"{label} must contain {size} values; got {a.size}.")

    def as_ctypes(self) -> _ffi.Input:
        self.check_arrays()
        rec = _ffi.Input()
        rec.vertex_count = self.vertex_count
        rec.tet_count = self.tet_count
        rec.cubature_k = self.cubature_k
        rec.positions = _ffi.fptr(self.positions)
        rec.velocities = _ffi.fptr(self.velocities)
        rec.vertex_rest = _ffi.fptr(self.vertex_rest)
        rec.vertex_colors = _ffi.fptr(self.vertex_colors)
        rec.vertex_info = _ffi.uptr(self.vertex_info)
        rec.external_forces = _ffi.fptr(self.external_forces)
        rec.target_positions = _ffi.fptr(self.target_positions)
        rec.target_stiffnesses = _ffi.fptr(self.target_stiffnesses)
        rec.tet_indices = _ffi.uptr(self.tet_indices)
        rec.tet_inverse_dm = _ffi.fptr(self.tet_inverse_dm)
        rec.tet_meta = _ffi.fptr(self.tet_meta)
        rec.tet_rest_stiffness = _ffi.fptr(self.tet_rest_stiffness)
        rec.adjacency = _ffi.uptr(self.adjacency)
        rec.adjacency_length = int(self.adjacency.size)
        rec.cubature_tet_ids = _ffi.uptr(self.cubature_tet_ids)
        rec.cubature_weights = _ffi.fptr(self.cubature_weights)
        rec.cubature_basis = _ffi.fptr(self.cubature_basis)
        cloth = self.cloth_ctypes()
        if cloth is not None:
            rec.cloth = ctypes.pointer(cloth)
        if self.contact_counts is not None and self.contact_candidate_count > 0:
            rec.contact_indices = _ffi.uptr(self.contact_indices)
            rec.contact_vertex_triangle_count = int(self.contact_counts[0])
            rec.contact_edge_edge_count = int(self.contact_counts[1])
        surface = None
        if self.contact_surface is not None:
            surface = _ffi.ContactSurface()
            surface.triangle_count = self.contact_surface.size // 3
            surface.triangles = _ffi.uptr(self.contact_surface)
            surface.candidate_capacity = int(self.contact_capacity)
            rec.contact_surface = ctypes.pointer(surface)
        # Keep the arrays (and the cloth / surface records) alive as long as the record.
        rec._owner = (self, cloth, surface)  # type: ignore[attr-defined]
        return rec

    def copy(self) -> "SceneInput":
        return dataclasses.replace(
            self, **{f.name: (getattr(self, f.name).copy()
                              if isinstance(getattr(self, f.name), np.ndarray)
                              else getattr(self, f.name))
                     for f in dataclasses.fields(self)})

    def arrays(self) -> dict:
        """Every array of the input plus its counts (the artifact payload)."""
        out = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)
               if isinstance(getattr(self, f.name), np.ndarray)}
        out["__meta"] = np.array([self.vertex_count, self.tet_count, self.cubature_k], dtype=np.int64)
        return out

    @classmethod
    def from_arrays(cls, arrays: dict) -> "SceneInput":
        meta = arrays["__meta"]
        kwargs = {k: v for k, v in arrays.items() if k != "__meta"}
        return cls(vertex_count=int(meta[0]), tet_count=int(meta[1]), cubature_k=int(meta[2]), **kwargs)

    def save(self, path: str):
        arrays = {f.name: getattr(self, f.name) for f in dataclasses.fields(self)
                  if isinstance(getattr(self, f.name), np.ndarray)}
        meta = np.array([self.vertex_count, self.tet_count, self.cubature_k], dtype=np.int64)
        tmp = path + ".tmp.npz"
        np.savez(tmp, __meta=meta, **arrays)
        import os
        os.replace(tmp, path)

    @classmethod
    def load(cls, path: str) -> "SceneInput":
        with np.load(path) as z:
            meta = z["__meta"]
            kwargs = {k: z[k] for k in z.files if k != "__meta"}
        return cls(vertex_count=int(meta[0]), tet_count=int(meta[1]), cubature_k=int(meta[2]), **kwargs)

    def bbox_diagonal(self) -> float:
        p = self.positions.reshape(-1, 4)[:, :3].astype(np.float64)
        return float(np.linalg.norm(p.max(axis=0) - p.min(axis=0)))

    def active_vertex_count(self) -> int:
        return int(np.count_nonzero(self.vertex_info.reshape(-1, 4)[:, 2] == 0))

    def split_bodies(self) -> list:
        """One SceneInput per body.  Bodies are disjoint meshes whose vertices
        and tets are contiguous (as the scene builder lays them out), so each
        body's slice, re-indexed to start at zero, is a complete scene with
        the same rest data and cubature records it had in the whole."""
        if self.cloth_triangles is not None:
            raise ValueError("split_bodies takes tetrahedral scenes only")
        info = self.vertex_info.reshape(-1, 4)
        tets = self.tet_indices.reshape(-1, 4)
        body_of_vertex = info[:, 3]
        bodies = np.unique(body_of_vertex)
        body_of_tet = body_of_vertex[tets[:, 0]] if self.tet_count else np.zeros(0, np.uint32)
        K = self.cubature_k
        out = []
        for b in bodies:
            vs = np.flatnonzero(body_of_vertex == b)
            ts = np.flatnonzero(body_of_tet == b)
            v0, v1 = int(vs[0]), int(vs[-1]) + 1
            t0, t1 = (int(ts[0]), int(ts[-1]) + 1) if ts.size else (0, 0)
            if v1 - v0 != vs.size or t1 - t0 != ts.size:
                raise ValueError(f"body {b} is not contiguous")
            bi = info[v0:v1].copy()
            a0 = int(bi[:, 0].min()) if bi[:, 1].any() else 0
            a1 = int((bi[:, 0] + bi[:, 1]).max())
            bi[:, 0] -= a0
            bi[:, 3] = 0
            adj = self.adjacency[a0:a1].astype(np.int64) - t0
            if adj.size and (adj.min() < 0 or adj.max() >= t1 - t0):
                raise ValueError(f"body {b} has adjacency outside its tets")
            cub = self.cubature_tet_ids[v0 * K:v1 * K].astype(np.int64)
            empty = cub == 0xFFFFFFFF
            cub = np.where(empty, cub, cub - t0)
            if (~empty).any() and (cub[~empty].min() < 0 or cub[~empty].max() >= t1 - t0):
                raise ValueError(f"body {b} has cubature records outside its tets")

            def vs4(a, per):
                return None if a is None else a[v0 * per:v1 * per].copy()

            out.append(SceneInput(
                vertex_count=v1 - v0, tet_count=t1 - t0, cubature_k=K,
                positions=vs4(self.positions, 4), vertex_rest=vs4(self.vertex_rest, 4),
                vertex_info=bi.reshape(-1).astype(np.uint32),
                tet_indices=(tets[t0:t1].astype(np.int64) - v0).astype(np.uint32).reshape(-1),
                tet_inverse_dm=self.tet_inverse_dm[t0 * 12:t1 * 12].copy(),
                tet_meta=self.tet_meta[t0 * 4:t1 * 4].copy(),
                adjacency=adj.astype(np.uint32),
                cubature_tet_ids=cub.astype(np.uint32),
                cubature_weights=self.cubature_weights[v0 * K:v1 * K].copy(),
                cubature_basis=self.cubature_basis[v0 * K * 36:v1 * K * 36].copy(),
                velocities=vs4(self.velocities, 4), vertex_colors=vs4(self.vertex_colors, 4),
                tet_rest_stiffness=(None if self.tet_rest_stiffness is None
                                    else self.tet_rest_stiffness[t0 * 144:t1 * 144].copy()),
                external_forces=vs4(self.external_forces, 3), target_positions=vs4(self.target_positions, 3),
                target_stiffnesses=vs4(self.target_stiffnesses, 1),
                rest_positions=None if self.rest_positions is None else self.rest_positions[v0:v1].copy()))
        return out


class Scene:
    """Owner of a native jgs2_scene handle (include/jgs2_scene.h)."""

    def __init__(self):
        self._lib = _ffi.scene_lib()
        self._h = self._lib.jgs2_scene_new()
        if not self._h:
            raise MemoryError("jgs2_scene_new failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.jgs2_scene_destroy(h)
            self._h = None

    def _error(self) -> str:
        return self._lib.jgs2_scene_last_error(self._h).decode()

    def add_material(self, density, young, poisson, model=MATERIAL_STABLE_NEO_HOOKEAN) -> int:
        mid = self._lib.jgs2_scene_add_material(self._h, density, young, poisson, model)
        if mid < 0:
            raise ValueError(self._error())
        return mid

    def add_cuboid(self, cells, origin, size, material=0, body=0, pinned_faces=0) -> int:
        c = (c_uint32 * 3)(*cells)
        o = (c_double * 3)(*origin)
        s = (c_double * 3)(*size)
        base = self._lib.jgs2_scene_add_cuboid(self._h, c, o, s, material, body, pinned_faces)
        if base < 0:
            raise ValueError(self._error())
        return base

    def add_mesh(self, positions, tets, material=0, pinned=None, body=0, tet_materials=None) -> int:
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(tets, dtype=np.uint32).reshape(-1)
        pin = None if pinned is None else np.ascontiguousarray(pinned, dtype=np.uint8)
        mats = None if tet_materials is None else np.ascontiguousarray(tet_materials, dtype=np.uint32)
        base = self._lib.jgs2_scene_add_mesh(
            self._h, pos.size // 3, _ffi.dptr(pos), q.size // 4, _ffi.uptr(q),
            _ffi.uptr(mats), material,
            None if pin is None else pin.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), body)
        if base < 0:
            raise ValueError(self._error())
        return base

    def add_cloth(self, positions, triangles, pinned=None, body=0, density=480.0, young=9000.0,
                  poisson=0.3, thickness=0.012, bending=0.045) -> int:
        """Triangle cloth sheet as one body (defaults: the reference's pinned
        cloth drape material, src/scenes/index.ts:688-696)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        tri = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1)
        pin = None if pinned is None else np.ascontiguousarray(pinned, dtype=np.uint8)
        base = self._lib.jgs2_scene_add_cloth(
            self._h, pos.size // 3, _ffi.dptr(pos), tri.size // 3, _ffi.uptr(tri),
            None if pin is None else pin.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), body,
            density, young, poisson, thickness, bending)
        if base < 0:
            raise ValueError(self._error())
        return base

    def set_rest_positions(self, positions):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1)
        if pos.size != 3 * self.vertex_count:
            raise ValueError("positions must hold 3 values per vertex")
        status = self._lib.jgs2_scene_set_rest_positions(self._h, _ffi.dptr(pos))
        if status != 0:
            raise _ffi.JGS2Error(status, self._error())

    def set_contact(self, enabled=True, capacity=0):
        """True (or CONTACT_STATIC): static candidates; CONTACT_SURFACE: the
        surface for the device broad phase, listing at most `capacity`
        candidates an iteration (0: the default); False: no contact."""
        mode = CONTACT_STATIC if enabled is True else (CONTACT_NONE if enabled is False else int(enabled))
        self._lib.jgs2_scene_set_contact(self._h, mode)
        self._lib.jgs2_scene_set_contact_capacity(self._h, int(capacity))

    def set_pinned(self, pinned):
        pin = np.ascontiguousarray(pinned, dtype=np.uint8)
        if pin.size != self.vertex_count:
            raise ValueError("pinned must have one entry per vertex")
        status = self._lib.jgs2_scene_set_pinned(
            self._h, pin.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        if status != 0:
            raise _ffi.JGS2Error(status, self._error())

    @property
    def vertex_count(self) -> int:
        return self._lib.jgs2_scene_vertex_count(self._h)

    @property
    def tet_count(self) -> int:
        return self._lib.jgs2_scene_tet_count(self._h)

    def rest_positions(self) -> np.ndarray:
        out = np.empty(3 * self.vertex_count, dtype=np.float64)
        self._lib.jgs2_scene_rest_positions(self._h, _ffi.dptr(out))
        return out.reshape(-1, 3)

    def precompute(self, timestep=1 / 60, cubature_k=6, method=PRECOMPUTE_EXACT,
                   patch_radius=2, threads=0, **overrides) -> dict:
        opt = _ffi.PrecomputeOptions()
        self._lib.jgs2_default_precompute_options(ctypes.byref(opt))
        opt.timestep = timestep
        opt.cubature_k = cubature_k
        opt.method = method
        opt.patch_radius = patch_radius
        opt.threads = threads
        for key, value in overrides.items():
            setattr(opt, key, value)
        st = _ffi.PrecomputeStats()
        status = self._lib.jgs2_scene_precompute(self._h, ctypes.byref(opt), ctypes.byref(st))
        if status != 0:
            raise _ffi.JGS2Error(status, self._error())
        return {name: getattr(st, name) for name, _t in _ffi.PrecomputeStats._fields_}

    def set_initial_state(self, positions=None, velocities=None, pin_at_initial=False):
        p = None if positions is None else np.ascontiguousarray(positions, dtype=np.float32)
        v = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float32)
        self._keep_state = (p, v)
        self._lib.jgs2_scene_set_initial_state(self._h, _ffi.fptr(p), _ffi.fptr(v),
                                               1 if pin_at_initial else 0)

    def set_objectives(self, external_forces=None, target_positions=None,
                       target_stiffnesses=None):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32)
                for a in (external_forces, target_positions, target_stiffnesses)]
        status = self._lib.jgs2_scene_set_objectives(self._h, *[_ffi.fptr(a) for a in arrs])
        if status != 0:
            raise _ffi.JGS2Error(status, self._error())

    def pack(self) -> SceneInput:
        rec = _ffi.Input()
        status = self._lib.jgs2_scene_pack(self._h, ctypes.byref(rec))
        if status != 0:
            raise _ffi.JGS2Error(status, self._error())
        V, T, K = rec.vertex_count, rec.tet_count, rec.cubature_k

        def f(ptr, n):
            if not ptr:
                return None
            return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

        cloth = {}
        if rec.cloth:
            c = rec.cloth.contents
            C, H = c.triangle_count, c.hinge_count
            cloth = dict(
                cloth_triangles=f(c.triangle_indices, 3 * C),
                cloth_inverse_rest=f(c.triangle_inverse_rest_bases, 4 * C),
                cloth_rest_areas=f(c.triangle_rest_areas, C),
                hinge_indices=f(c.hinge_indices, 4 * H) if H else np.zeros(0, np.uint32),
                hinge_rest_angles=f(c.hinge_rest_angles, H) if H else np.zeros(0, np.float32),
                hinge_rest_edge_lengths=f(c.hinge_rest_edge_lengths, H) if H else np.zeros(0, np.float32),
                cloth_material=np.array([c.young_modulus, c.poisson_ratio, c.thickness, c.bending_stiffness],
                                        dtype=np.float32))
        contact = {}
        nc = rec.contact_vertex_triangle_count + rec.contact_edge_edge_count
        if nc:
            contact = dict(contact_indices=f(rec.contact_indices, 4 * nc),
                           contact_counts=np.array([rec.contact_vertex_triangle_count,
                                                    rec.contact_edge_edge_count], dtype=np.uint32))
        if rec.contact_surface:
            cs = rec.contact_surface.contents
            contact = dict(contact_surface=f(cs.triangles, 3 * cs.triangle_count),
                           contact_capacity=int(cs.candidate_capacity))
        return SceneInput(
            **cloth, **contact,
            vertex_count=V, tet_count=T, cubature_k=K,
            positions=f(rec.positions, 4 * V), vertex_rest=f(rec.vertex_rest, 4 * V),
            vertex_info=f(rec.vertex_info, 4 * V), tet_indices=f(rec.tet_indices, 4 * T),
            tet_inverse_dm=f(rec.tet_inverse_dm, 12 * T), tet_meta=f(rec.tet_meta, 4 * T),
            adjacency=f(rec.adjacency, rec.adjacency_length),
            cubature_tet_ids=f(rec.cubature_tet_ids, V * K),
            cubature_weights=f(rec.cubature_weights, V * K),
            cubature_basis=f(rec.cubature_basis, V * K * 36),
            velocities=f(rec.velocities, 4 * V), vertex_colors=f(rec.vertex_colors, 4 * V),
            tet_rest_stiffness=f(rec.tet_rest_stiffness, 144 * T),
            external_forces=f(rec.external_forces, 3 * V),
            target_positions=f(rec.target_positions, 3 * V),
            target_stiffnesses=f(rec.target_stiffnesses, V),
            rest_positions=self.rest_positions(),
        )


# ---- named workloads -----------------------------------------------------------

def cantilever(cells=(20, 4, 4), size=(1.0, 0.2, 0.2), young=1e5, poisson=0.4,
               density=1000.0, timestep=1 / 60, cubature_k=6,
               method=PRECOMPUTE_EXACT, patch_radius=2, threads=0) -> SceneInput:
    """Minimal cantilever: a bar of hexes x6 tets with its x=0 face pinned,
    stable Neo-Hookean (the 525-vertex / 1920-tet configuration)."""
    sc = Scene()
    m = sc.add_material(density, young, poisson, MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_cuboid(cells, (0.0, 0.0, 0.0), size, m, 0, FACE_X_MIN)
    stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=method,
                          patch_radius=patch_radius, threads=threads)
    inp = sc.pack()
    inp.stats = stats
    return inp


def single_tetrahedron(timestep=1 / 60, cubature_k=4) -> SceneInput:
    """The single stable Neo-Hookean tetrahedron of the material parity
    fixture (src/scenes/phase1.ts:44-64, 246-271): rest A=(0,0,0),
    B=(1,0,0), C=(0,1,0), D=(0,0,1), A pinned, density 1000, E=8e4, nu=0.3."""
    sc = Scene()
    m = sc.add_material(1000.0, 80000.0, 0.3, MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_mesh([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1], [0, 1, 2, 3], m, pinned=[1, 0, 0, 0])
    sc.precompute(timestep=timestep, cubature_k=cubature_k)
    return sc.pack()


def cloth_grid(cells, prefold=False):
    """Vertices and triangles of a (cells+1)^2 sheet in the xz plane spanning
    [-0.8, 0.8]^2 at y = 1.15, two triangles per cell wound (i00, i01, i10),
    (i10, i01, i11) (clothDefinition, src/scenes/index.ts:632-681).  With
    `prefold` the columns x >= 3 are folded back over the sheet at y = 1.229,
    as the reference's 4-cell demo is."""
    n = cells + 1
    pos = np.zeros((n * n, 3))
    for z in range(n):
        for x in range(n):
            folded = prefold and x >= 3
            wx = (0.8 - 0.4 * x) if folded else (-0.8 + 1.6 * x / cells)
            pos[x + z * n] = (wx, 1.229 if folded else 1.15, -0.8 + 1.6 * z / cells)
    tri = []
    for z in range(cells):
        for x in range(cells):
            i00, i10 = x + z * n, x + 1 + z * n
            i01, i11 = x + (z + 1) * n, x + 1 + (z + 1) * n
            tri += [i00, i01, i10, i10, i01, i11]
    return pos, np.array(tri, dtype=np.uint32)


def cloth_drape(cells=4, prefold=True, pinned_columns=(0, 2), young=9000.0, poisson=0.3, thickness=0.012,
                bending=0.045, density=480.0, timestep=1 / 120, cubature_k=4, contact=CONTACT_NONE) -> SceneInput:
    """Pinned cloth drape (clothDefinition, src/scenes/index.ts:632-720): a
    fully pinned stable Neo-Hookean box collider (E=1.1e5, nu=0.34) and a
    StVK sheet whose z = 0 row is pinned at the given columns.  Without IPC
    the sheet does not touch the collider; the collider keeps the scene on the
    stable Neo-Hookean path that cloth requires.  contact=CONTACT_STATIC lists
    the static IPC candidate superset (collider-cloth and cloth self-contact),
    as the reference's cloth demo does."""
    sc = Scene()
    m = sc.add_material(1000.0, 110000.0, 0.34, MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_cuboid((1, 1, 1), (-0.65, 0.0, -0.45), (0.9, 0.5, 0.9), m, 0, 63)
    pos, tri = cloth_grid(cells, prefold)
    n = cells + 1
    pin = np.zeros(n * n, dtype=np.uint8)
    for x in pinned_columns:
        pin[x] = 1
    sc.add_cloth(pos, tri, pin, 1, density, young, poisson, thickness, bending)
    if contact != CONTACT_NONE:
        sc.set_contact(contact)
    stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=PRECOMPUTE_PATCH)
    inp = sc.pack()
    inp.stats = stats
    return inp


def cloth_sheet(cells=127, young=1e4, bending=1e-3, **kwargs) -> SceneInput:
    """The serving mix's cloth request: a (cells+1)^2-vertex StVK sheet
    (16,384 vertices and 32,258 triangles at 127 cells) with its two z = 0
    corners pinned, over a pinned box collider."""
    return cloth_drape(cells=cells, prefold=False, pinned_columns=(0, cells), young=young, bending=bending,
                       **kwargs)


# Settings of the reference app's cloth scene (src/App.tsx:529-575: activation
# distance 0.01, step bound 0.01, friction 0.3) at dt = 1/120 and 5 iterations.
CLOTH_SETTINGS = dict(timestep=1 / 120, gravity=(0.0, -9.81, 0.0), floorHeight=-0.18, floorStiffness=0.0,
                      iterations=5, velocityDamping=0.997, contactTangentialDamping=0.0, contactMargin=0.01,
                      horizontalBodyCorrection=False, ipcActivationDistance=0.01, ipcMinimumDistance=0.003,
                      ipcBarrierStiffness=1e5, ipcFrictionCoefficient=0.3, ipcFrictionVelocityEpsilon=0.05,
                      ipcStepSafety=0.9, regularization=1e-6, rotationEpsilon=1e-7, maxStep=0.01)


def spherify(p):
    """Map points of the cube [-1, 1]^3 onto the unit ball (each axis scaled
    by sqrt(1 - a^2/2 - b^2/2 + a^2 b^2 / 3) of the other two): the cube's
    faces land on the sphere and a hex grid stays a valid mesh."""
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    x2, y2, z2 = x * x, y * y, z * z
    return np.stack([x * np.sqrt(1 - y2 / 2 - z2 / 2 + y2 * z2 / 3),
                     y * np.sqrt(1 - z2 / 2 - x2 / 2 + z2 * x2 / 3),
                     z * np.sqrt(1 - x2 / 2 - y2 / 2 + x2 * y2 / 3)], axis=1)


def cloth_sphere(cells=127, radius=0.3, centre=(0.0, 0.8, 0.0), sphere_cells=8, young=1e4, bending=1e-3,
                 contact=CONTACT_SURFACE, capacity=4 << 20, timestep=1 / 120) -> SceneInput:
    """The serving mix's cloth request: the (cells+1)^2-vertex StVK sheet of
    `cloth_sheet` (E = 1e4, bending 1e-3, its two z = -0.8 corners pinned,
    y = 1.15) draping over a fixed sphere of `radius` (a pinned hex grid of
    sphere_cells^3 x6 tets mapped onto the ball) with IPC over the sheet and
    the sphere's surface, the sheet's self-contact included.  A draped sheet
    lists about 2.7 million candidates an iteration (pairs within 3 cm of
    each other), hence the capacity of 4 Mi candidates."""
    sc = Scene()
    m = sc.add_material(1000.0, 110000.0, 0.34, MATERIAL_STABLE_NEO_HOOKEAN)
    start = sc.add_cuboid((sphere_cells,) * 3, (-1.0,) * 3, (2.0,) * 3, m, 0, 63)
    n_sphere = (sphere_cells + 1) ** 3
    p = sc.rest_positions()
    p[start:start + n_sphere] = spherify(p[start:start + n_sphere]) * radius + np.array(centre)
    sc.set_rest_positions(p)
    pos, tri = cloth_grid(cells)
    n = cells + 1
    pin = np.zeros(n * n, dtype=np.uint8)
    pin[0] = pin[cells] = 1
    sc.add_cloth(pos, tri, pin, 1, 480.0, young, 0.3, 0.012, bending)
    sc.set_contact(contact, capacity)
    stats = sc.precompute(timestep=timestep, cubature_k=4, method=PRECOMPUTE_PATCH)
    inp = sc.pack()
    inp.stats = stats
    return inp


def static_contact_candidates(vertex_count, triangles):
    """buildStaticIpcContactCandidates: (indices uint32[4n], vt count, ee count)."""
    lib = _ffi.scene_lib()
    tri = np.ascontiguousarray(triangles, dtype=np.uint32).reshape(-1)
    vt, ee = c_uint32(0), c_uint32(0)
    n = lib.jgs2_build_static_contact_candidates(vertex_count, _ffi.uptr(tri), tri.size // 3, None, 0,
                                                 ctypes.byref(vt), ctypes.byref(ee))
    if n < 0:
        raise ValueError("invalid surface triangles")
    out = np.zeros(4 * n, dtype=np.uint32)
    lib.jgs2_build_static_contact_candidates(vertex_count, _ffi.uptr(tri), tri.size // 3, _ffi.uptr(out), n,
                                             ctypes.byref(vt), ctypes.byref(ee))
    return out, vt.value, ee.value


def rotate_euler_xyz(p, rx, ry, rz):
    """rotateEulerXyz (src/simulation/cpu/mesh.ts:210-235): x, then y, then z."""
    cx, sx, cy, sy, cz, sz = math.cos(rx), math.sin(rx), math.cos(ry), math.sin(ry), math.cos(rz), math.sin(rz)
    x, y, z = p[:, 0], p[:, 1] * cx - p[:, 2] * sx, p[:, 1] * sx + p[:, 2] * cx
    x, z = cy * x + sy * z, -sy * x + cy * z
    x, y = cz * x - sz * y, sz * x + cz * y
    return np.stack([x, y, z], axis=1)


# Trough settings of the reference app for its IPC scenes (src/App.tsx:529-575).
TROUGH_SETTINGS = dict(timestep=1 / 60, gravity=(0.0, -9.81, 0.0), floorHeight=-0.18, floorStiffness=0.0,
                       iterations=3, velocityDamping=0.997, contactTangentialDamping=0.0, contactMargin=0.01,
                       horizontalBodyCorrection=False, ipcActivationDistance=0.08, ipcMinimumDistance=0.003,
                       ipcBarrierStiffness=1e5, ipcFrictionCoefficient=0.45, ipcFrictionVelocityEpsilon=0.05,
                       ipcStepSafety=0.9, regularization=1e-6, rotationEpsilon=1e-7, maxStep=0.075)


def trough(boxes=10, cubature_k=6, timestep=1 / 60, method=PRECOMPUTE_EXACT, contact=CONTACT_STATIC,
           capacity=0) -> SceneInput:
    """IPC box trough (troughDefinition, src/scenes/index.ts:551-630): a
    pinned two-cell solid warped into a V (y = 0.05 + 0.65|x| - 0.18(1 - layer))
    and `boxes` one-cell stable Neo-Hookean boxes (0.46 m) stacked four per
    layer above it, each slightly rotated; static IPC candidates over the
    whole boundary surface."""
    sc = Scene()
    m_trough = sc.add_material(1000.0, 120000.0, 0.34, MATERIAL_STABLE_NEO_HOOKEAN)
    m_box = [sc.add_material(850.0, 70000.0, 0.35, MATERIAL_STABLE_NEO_HOOKEAN) for _ in range(2)]
    sc.add_cuboid((2, 1, 1), (-2.2, 0.0, -1.5), (4.4, 1.0, 3.0), m_trough, 0, 63)
    starts = []
    for i in range(boxes):
        starts.append(sc.add_cuboid((1, 1, 1), (-0.23, -0.23, -0.23), (0.46, 0.46, 0.46), m_box[i % 2], i + 1, 0))
    p = sc.rest_positions()
    x, layer = p[:12, 0].copy(), p[:12, 1].copy()
    p[:12, 1] = 0.05 + 0.65 * np.abs(x) - 0.18 * (1 - layer)
    for i, s in enumerate(starts):
        slot, lay = i % 4, i // 4
        rot = (((i % 3) - 1) * 0.04, ((i % 5) - 2) * 0.035, (-1 if i % 2 == 0 else 1) * 0.055)
        q = rotate_euler_xyz(p[s:s + 8], *rot)
        q += np.array([-0.37 if slot % 2 == 0 else 0.37, 2.15 + 0.72 * lay, -0.38 if slot < 2 else 0.38])
        p[s:s + 8] = q
    sc.set_rest_positions(p)
    sc.set_contact(contact, capacity)
    stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=method)
    inp = sc.pack()
    inp.stats = stats
    return inp


# Settings of the box trough: the trough's contact parameters with the
# activation distance 1e-3 m, friction 0.3 and 15 iterations; the minimum
# distance (1e-4 m, below the activation distance) and the per-iteration step
# bound (0.02 m, room for 9 m/s at 15 iterations per 1/60 s frame) are this
# workload's choices.
BOX_TROUGH_SETTINGS = dict(TROUGH_SETTINGS, iterations=15, ipcActivationDistance=1e-3, ipcMinimumDistance=1e-4,
                           ipcFrictionCoefficient=0.3, maxStep=0.02)


def box_trough(boxes=20, cells=8, box_size=0.46, heights=(1.0, 3.0), seed=3003, young=2e5, poisson=0.4,
               density=7800.0, plate_cells=(16, 4), plate_thickness=0.04, cubature_k=6, timestep=1 / 60,
               method=PRECOMPUTE_PATCH, contact=CONTACT_SURFACE, capacity=0, threads=0,
               exact_complement=True, patch_radius=1) -> SceneInput:
    """IPC box trough: `boxes` stable Neo-Hookean boxes of cells^3 hexes x6
    tets (edge `box_size`, the reference trough's box), dropped from seeded
    heights U[heights] and yaws U[0, 2 pi) into a pinned V-trough of two
    4 x 1 m plates at +-45 degrees (plate_cells along the trough and down the
    slope, one cell thick, inner edges 1 cm apart at the apex).  Placement
    (Mulberry32): x U[-0.3, 0.3], z within the trough, redrawn until every
    pair of boxes is 2 cm apart horizontally (footprint radius edge / sqrt 2)
    or vertically, and each box clears the plates.  Contact over the whole
    boundary surface.

    Cubature: by default the patch method's exact complement (every
    candidate tet within `patch_radius` rings, weight one; K is the largest
    candidate count).  The density (steel) keeps the step's elastic to
    inertial ratio E h^2 / (rho cell^2) near 2: fine free bodies far above
    that (1000 kg/m^3 gives 40 at 8^3 cells), or trained K = `cubature_k`
    records (exact_complement False), deform in the Jacobi sweep until the
    assembled gate reverts every pose and the pile stops."""
    sc = Scene()
    m_plate = sc.add_material(1000.0, 1.2e5, 0.34, MATERIAL_STABLE_NEO_HOOKEAN)
    m_box = sc.add_material(density, young, poisson, MATERIAL_STABLE_NEO_HOOKEAN)
    t = plate_thickness
    plates = [sc.add_cuboid((plate_cells[1], 1, plate_cells[0]), (0.0, 0.0, -2.0), (1.0, t, 4.0), m_plate, 0, 63)
              for _ in range(2)]
    starts = [sc.add_cuboid((cells, cells, cells), (-box_size / 2,) * 3, (box_size,) * 3, m_box, i + 1, 0)
              for i in range(boxes)]
    p = sc.rest_positions()
    n_plate = plates[1] - plates[0]
    c = s_ = math.sqrt(0.5)
    gap = 0.005
    for side, base in ((1.0, plates[0]), (-1.0, plates[1])):
        q = p[base:base + n_plate].copy()
        # Top face (local y = t) on the line from (side * gap, 0) at 45 degrees;
        # the plate's thickness lies outside the trough.
        ux, uy, nx, ny = side * c, s_, -side * s_, c
        x, y = q[:, 0], q[:, 1] - t
        p[base:base + n_plate, 0] = side * gap + x * ux + y * nx
        p[base:base + n_plate, 1] = x * uy + y * ny
    rand = mulberry32(seed)
    foot = box_size / math.sqrt(2.0)  # horizontal reach of a yawed box
    centres = []
    n_box = cells + 1
    for i, start in enumerate(starts):
        for _attempt in range(10000):
            yaw = 2 * math.pi * rand()
            height = heights[0] + (heights[1] - heights[0]) * rand()
            x = -0.3 + 0.6 * rand()
            z = -2.0 + foot + (4.0 - 2 * foot) * rand()
            ctr = np.array([x, height, z])
            clear = height - box_size / 2 > abs(x) + foot + 0.02
            apart = all(math.hypot(x - o[0], z - o[2]) > 2 * foot + 0.02 or abs(height - o[1]) > box_size + 0.02
                        for o in centres)
            if clear and apart:
                break
        else:
            raise ValueError("box_trough could not place the boxes apart; lower the count or widen the heights")
        centres.append(ctr)
        q = rotate_euler_xyz(p[start:start + n_box ** 3], 0.0, yaw, 0.0)
        p[start:start + n_box ** 3] = q + ctr
    sc.set_rest_positions(p)
    sc.set_contact(contact, capacity)
    if exact_complement:
        args = dict(timestep=timestep, method=method, threads=threads, patch_radius=patch_radius, exact_complement=1)
        # Probe with a bound on the patch's candidate tets (192 at one ring
        # of a hex grid, 400 at two), then pack exactly the widest count.
        probe = 256 * patch_radius
        stats = sc.precompute(cubature_k=probe, **args)
        while stats["max_records_per_vertex"] >= probe:
            probe *= 2
            stats = sc.precompute(cubature_k=probe, **args)
        stats = sc.precompute(cubature_k=max(1, stats["max_records_per_vertex"]), **args)
    else:
        stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=method, threads=threads,
                              patch_radius=patch_radius)
    inp = sc.pack()
    stats["centres"] = [c_.tolist() for c_ in centres]
    inp.stats = stats
    return inp


def batched_scenes(count=256, **kwargs) -> list:
    """The batched uneven bodies of `batched_bodies`, one independent scene
    per body (their cubature training is shared across identical patches)."""
    return batched_bodies(count=count, **kwargs).split_bodies()


# The cantilever's scripted soft target, restating the reference's public
# demo target (minimalScriptedTargetAtFrame, src/scenes/index.ts:252-328) on
# the frame window of the 300-frame cantilever workload: one free-tip vertex
# (the x = max, y = min, z = min corner, as vertex 1 is on the reference's
# one-cell beam), stiffness 30 000, a smoothstep pull on keyframes every 3
# frames from frame 60 to frame 120, held until frame 180 and then released
# (stiffness 0).  The pull offset is the reference's (0.45, 0.65, 0.25) m on
# its 2 m beam, scaled by the bar's length.
CANTILEVER_TARGET_PULL_START = 60
CANTILEVER_TARGET_PULL_END = 120
CANTILEVER_TARGET_RELEASE = 180
CANTILEVER_TARGET_KEYFRAME_INTERVAL = 3
CANTILEVER_TARGET_STIFFNESS = 30000.0
CANTILEVER_TARGET_OFFSET = (0.45, 0.65, 0.25)  # per 2 m of beam


def cantilever_tip_vertex(inp: SceneInput) -> int:
    """The free tip the scripted target pulls: the x = max, y = min, z = min
    corner of the bar."""
    rest = inp.rest_positions
    key = np.lexsort((rest[:, 2], rest[:, 1], -rest[:, 0]))
    return int(key[0])


def cantilever_target(inp: SceneInput, frame: int):
    """Scripted target of `frame`: (vertex, target position (3,), stiffness).
    Stiffness is 0 before the pull starts and after the release."""
    if frame < 0:
        raise ValueError("cantilever target frame must be nonnegative")
    vertex = cantilever_tip_vertex(inp)
    rest = inp.rest_positions[vertex].astype(np.float64)
    length = float(np.ptp(inp.rest_positions[:, 0]))
    start, end = CANTILEVER_TARGET_PULL_START, CANTILEVER_TARGET_PULL_END
    step = CANTILEVER_TARGET_KEYFRAME_INTERVAL
    pull = min(frame, end)
    key = min(end, start + ((pull - start) // step) * step) if frame >= start else start
    u = (key - start) / (end - start)
    progress = u * u * (3 - 2 * u)
    target = rest + np.array(CANTILEVER_TARGET_OFFSET) * (length / 2.0) * progress
    active = start <= frame < CANTILEVER_TARGET_RELEASE
    return vertex, target.astype(np.float32), (CANTILEVER_TARGET_STIFFNESS if active else 0.0)


def unit_cube_components(cells=100, young=1e6, poisson=0.45, density=1000.0, timestep=1 / 60, cubature_k=6,
                         seed=1048583, patch_radius=2, method=PRECOMPUTE_PATCH, exact_complement=0,
                         schedule="jacobi") -> dict:
    """Fingerprint components of a unit_cube input (artifact.COMPONENTS)."""
    return {"topology": {"builder": "unit_cube", "cells": [cells] * 3, "size": [1.0, 1.0, 1.0],
                         "pinned": "y_min", "stretch_seed": seed},
            "materials": {"density": density, "young": young, "poisson": poisson, "model": "stable-neo-hookean"},
            "timestep": timestep,
            "basis": {"method": method, "patch_radius": patch_radius},
            "cubature": {"k": cubature_k, "exact_complement": exact_complement, "trainer": TRAINER_REVISION},
            "solverSchedule": schedule}


def cached_input(cache_dir: str, prefix: str, components: dict, build):
    """The input `build()` makes, kept as a fingerprinted artifact under
    `cache_dir` and reused only when every component fingerprint matches and
    the payload is intact; returns (input, reused)."""
    from . import artifact

    prints = artifact.fingerprints(components)
    path = os.path.join(cache_dir, artifact.cache_name(prefix, prints))
    try:
        return artifact.load(path, prints, SceneInput), True
    except artifact.ArtifactMismatch:
        pass
    inp = build()
    try:
        artifact.save(path, inp, prints)
    except OSError:
        pass
    return inp, False


def unit_cube(cells=100, young=1e6, poisson=0.45, density=1000.0, timestep=1 / 60,
              cubature_k=6, seed=1048583, patch_radius=2, threads=0,
              method=PRECOMPUTE_PATCH) -> SceneInput:
    """Single large body: unit cube of cells^3 hexes x6 tets, bottom face
    pinned, initial pose = rest stretched per axis by U[0.9, 1.1] (Mulberry32
    seeded) about the bottom-face centre, the pinned face clamped in its
    stretched position."""
    sc = Scene()
    m = sc.add_material(density, young, poisson, MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_cuboid((cells, cells, cells), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), m, 0, FACE_Y_MIN)
    stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=method,
                          patch_radius=patch_radius, threads=threads)
    rand = mulberry32(seed)
    stretch = np.array([0.9 + 0.2 * rand() for _ in range(3)])
    rest = sc.rest_positions()
    centre = np.array([0.5, 0.0, 0.5])
    pos = centre + (rest - centre) * stretch
    p4 = np.ones((rest.shape[0], 4), dtype=np.float32)
    p4[:, :3] = pos
    sc.set_initial_state(p4.reshape(-1), None, pin_at_initial=True)
    inp = sc.pack()
    stats["stretch"] = stretch.tolist()
    inp.stats = stats
    return inp


def batched_bodies(count=256, seed=65537, min_cells=4, max_cells=32, soft=5e4, stiff=5e6,
                   poisson=0.4, density=1000.0, timestep=1 / 60, cubature_k=6,
                   patch_radius=2, threads=0, spacing=0.25) -> SceneInput:
    """Batched uneven bodies: `count` hex-grid boxes with per-axis cell counts
    drawn uniformly from [min_cells, max_cells] (Mulberry32 seeded), cell size
    1/32 m, alternating soft/stiff materials, laid out on a square grid above
    a penalty floor at y = 0."""
    rand = mulberry32(seed)
    sc = Scene()
    m_soft = sc.add_material(density, soft, poisson, MATERIAL_STABLE_NEO_HOOKEAN)
    m_stiff = sc.add_material(density, stiff, poisson, MATERIAL_STABLE_NEO_HOOKEAN)
    side = int(math.ceil(math.sqrt(count)))
    h = 1.0 / 32.0
    pitch = max_cells * h + spacing
    for b in range(count):
        cells = [min_cells + min(max_cells - min_cells,
                                 int(rand() * (max_cells - min_cells + 1))) for _ in range(3)]
        gx, gz = b % side, b // side
        origin = (gx * pitch, 0.25, gz * pitch)
        size = tuple(c * h for c in cells)
        sc.add_cuboid(cells, origin, size, m_soft if b % 2 == 0 else m_stiff, b, 0)
    stats = sc.precompute(timestep=timestep, cubature_k=cubature_k, method=PRECOMPUTE_PATCH,
                          patch_radius=patch_radius, threads=threads)
    inp = sc.pack()
    inp.stats = stats
    return inp

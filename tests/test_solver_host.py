"""Host logic of the solver on the reference's own solver unit cases
(src/simulation/gpu/jgs2-solver.test.ts:183-276): settings resolution, the
graph-coloured dependencies of non-incident cubature records, and the initial
convergence scene scale.  None of these needs a GPU.
"""
import ctypes

import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

UNUSED = 0xFFFFFFFF


def test_default_settings_keep_the_demo_stabilizers():
    # jgs2-solver.test.ts:184-195.
    r = solver.resolve_settings({})
    assert r["parity_mode"] == 0
    assert r["schedule"] == 0  # Jacobi
    assert r["velocity_damping"] < 1.0
    assert r["contact_tangential_damping"] > 0.0
    assert r["horizontal_body_correction"] == 1


def test_parity_mode_overrides_conflicting_stabilizers():
    # jgs2-solver.test.ts:197-212: parity mode wins over every stabilizer.
    r = solver.resolve_settings({"parityMode": True, "velocityDamping": 0.25, "contactTangentialDamping": 99,
                                 "horizontalBodyCorrection": True})
    assert r["parity_mode"] == 1
    assert r["velocity_damping"] == 1.0
    assert r["contact_tangential_damping"] == 0.0
    assert r["horizontal_body_correction"] == 0


def _one_tet_with_remote_record():
    """Five vertices, one tet (0 1 2 3) and one cubature slot per vertex; only
    vertex 4, which no tet touches, has a record: tet 0 with weight 1."""
    pos = np.array([0, 0, 0, 1, 1, 0, 0, 1, 0, 1, 0, 1, 0, 0, 1, 1, 2, 2, 2, 1], dtype=np.float32)
    return scenes.SceneInput(
        vertex_count=5, tet_count=1, cubature_k=1,
        positions=pos.copy(), vertex_rest=pos.copy(),
        vertex_info=np.array([0, 1, 0, 0, 1, 1, 0, 0, 2, 1, 0, 0, 3, 1, 0, 0, 4, 0, 0, 0], dtype=np.uint32),
        tet_indices=np.array([0, 1, 2, 3], dtype=np.uint32),
        tet_inverse_dm=np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], dtype=np.float32),
        tet_meta=np.array([1 / 6, 1, 1, 1.0], dtype=np.float32),
        adjacency=np.zeros(4, dtype=np.uint32),
        cubature_tet_ids=np.array([UNUSED, UNUSED, UNUSED, UNUSED, 0], dtype=np.uint32),
        cubature_weights=np.array([0, 0, 0, 0, 1], dtype=np.float32),
        cubature_basis=np.zeros(36 * 5, dtype=np.float32),
        vertex_colors=np.zeros(20, dtype=np.float32),
    )


def test_remote_cubature_record_conflicts_with_every_vertex_it_reads():
    # jgs2-solver.test.ts:215-237: the source vertex of a non-incident record
    # conflicts with the four vertices of the record's tet.
    colors, count = solver.build_vertex_coloring(_one_tet_with_remote_record())
    assert count == 5
    for v in range(4):
        assert colors[4] != colors[v]
    assert sorted(int(c) for c in colors) == [0, 1, 2, 3, 4]


def _scene_scale(positions, vertex_info):
    L = O.lib()
    fn = L.jgs2_oracle_initial_scene_scale
    fn.restype = ctypes.c_double
    fn.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32]
    p = np.ascontiguousarray(positions, dtype=np.float32)
    i = np.ascontiguousarray(vertex_info, dtype=np.uint32)
    return fn(p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), i.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
              p.size // 4)


def test_scene_scale_excludes_a_distant_fixed_anchor():
    # jgs2-solver.test.ts:240-256: the pinned anchor far away does not widen
    # the dynamic box; the diagonal of (0,0,0)-(3,4,0) is 5.
    scale = _scene_scale([0, 0, 0, 1, 3, 4, 0, 1, 10_000, -20_000, 30_000, 1],
                         [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0])
    assert scale == 5.0


def test_scene_scale_falls_back_for_a_degenerate_dynamic_box():
    # jgs2-solver.test.ts:258-275: one free vertex has no extent.
    scale = _scene_scale([2, 3, 4, 1, 50_000, 60_000, 70_000, 1], [0, 0, 0, 0, 0, 0, 1, 0])
    assert scale == 1e-12 and np.isfinite(scale) and scale > 0
    # Every vertex pinned: the same fallback.
    assert _scene_scale([0, 0, 0, 1, 1, 1, 1, 1], [0, 0, 1, 0, 0, 0, 1, 0]) == 1e-12


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_normalises_updates_by_its_input_scene_scale(precision):
    # The oracle's convergence reduction, given no scale of its own, divides
    # the largest update by the scale of its input: a single tetrahedron's
    # free-vertex box diagonal, rounded to f32 as the step stores it.
    inp = scenes.single_tetrahedron()
    scale = _scene_scale(inp.positions, inp.vertex_info)
    p = inp.positions.reshape(-1, 4)[inp.vertex_info.reshape(-1, 4)[:, 2] == 0, :3].astype(np.float64)
    assert scale == pytest.approx(float(np.linalg.norm(p.max(0) - p.min(0))), rel=1e-15)
    L = O.lib()
    F = ctypes.POINTER(ctypes.c_float)
    L.jgs2_oracle_reduce_convergence.argtypes = [ctypes.c_void_p, ctypes.c_void_p, F, F, F, ctypes.c_double, F]
    o = O.OracleSolver(inp, {}, precision=precision)
    comp = np.zeros((inp.vertex_count, 5, 4), dtype=np.float32)
    upd = np.zeros(inp.vertex_count, dtype=np.float32)
    upd[0] = 1e-3
    control = np.zeros(16, dtype=np.float32)
    control[:8] = [1, 1, 1, 15, 1, 0, 0, 0]
    out = np.zeros(32, dtype=np.float32)
    rec = O._settings_struct(O.resolve_settings(None))
    L.jgs2_oracle_reduce_convergence(o._h, ctypes.byref(rec), comp.ctypes.data_as(F), upd.ctypes.data_as(F),
                                     control.ctypes.data_as(F), -1.0, out.ctypes.data_as(F))
    want = np.float32(1e-3) / np.float32(scale)
    assert out[21] == pytest.approx(float(want), rel=1e-6)  # normalised update lane

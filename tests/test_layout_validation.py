"""Input validation (jgs2_validate_input) on the reference's own layout
fixtures (src/simulation/gpu/layout.test.ts:19-420), with its messages.

The two-tetrahedron fixture (:19-75) has five vertices, tets (0 1 2 3) and
(1 2 3 4), co-rotated material, and no cubature records. Its CSR adjacency
lists each vertex's incident tetrahedra, sorted.
"""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver

COROTATED, STABLE = 0.0, 1.0


def _two_tets(material=COROTATED):
    eye = [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0]
    pos = np.array([0, 0, 0, 1, 1, 0, 0, 1, 0, 1, 0, 1, 0, 0, 1, 1, 1, 1, 1, 1], dtype=np.float32)
    return scenes.SceneInput(
        vertex_count=5, tet_count=2, cubature_k=0,
        positions=pos.copy(), vertex_rest=pos.copy(),
        vertex_info=np.array([0, 1, 0, 0, 1, 2, 0, 0, 3, 2, 0, 0, 5, 2, 0, 0, 7, 1, 0, 0], dtype=np.uint32),
        tet_indices=np.array([0, 1, 2, 3, 1, 2, 3, 4], dtype=np.uint32),
        tet_inverse_dm=np.array(eye + eye, dtype=np.float32),
        tet_meta=np.array([1 / 6, 1, 1, material, 1 / 6, 1, 1, material], dtype=np.float32),
        adjacency=np.array([0, 0, 1, 0, 1, 0, 1, 1], dtype=np.uint32),
        cubature_tet_ids=np.zeros(0, dtype=np.uint32), cubature_weights=np.zeros(0, dtype=np.float32),
        cubature_basis=np.zeros(0, dtype=np.float32),
        vertex_colors=np.zeros(20, dtype=np.float32),
        tet_rest_stiffness=np.zeros(2 * 144, dtype=np.float32) if material == COROTATED else None,
    )


def _rejects(inp, pattern):
    with pytest.raises(solver.JGS2RangeError, match=pattern):
        solver.validate_input(inp)


def test_accepts_sorted_unique_incident_slices():
    solver.validate_input(_two_tets())
    solver.validate_input(_two_tets(STABLE))


def test_rejects_a_duplicate_tetrahedron_in_a_slice():
    inp = _two_tets()
    inp.adjacency[2] = 0
    _rejects(inp, "vertex 1 must equal incident tetrahedron 1; got 0")


def test_rejects_a_tetrahedron_not_incident_to_the_vertex():
    inp = _two_tets()
    inp.adjacency[0] = 1
    _rejects(inp, "vertex 0 must equal incident tetrahedron 0; got 1")


def test_rejects_a_slice_that_omits_an_incident_tetrahedron():
    inp = _two_tets()
    inp.vertex_info = np.array([0, 1, 0, 0, 1, 1, 0, 0, 2, 2, 0, 0, 4, 2, 0, 0, 6, 1, 0, 0], dtype=np.uint32)
    inp.adjacency = np.array([0, 0, 0, 1, 0, 1, 1], dtype=np.uint32)
    _rejects(inp, "vertex 1 must list exactly 2 unique incident tetrahedra; got 1")


def test_rejects_adjacency_entries_outside_every_slice():
    inp = _two_tets()
    inp.adjacency = np.append(inp.adjacency, np.uint32(0))
    _rejects(inp, "adjacency contains 1 unused entry\\.")
    inp.adjacency = np.append(inp.adjacency, np.uint32(0))
    _rejects(inp, "adjacency contains 2 unused entries\\.")


def test_rejects_invalid_objective_values():
    inp = _two_tets()
    inp.target_positions = np.zeros(15, dtype=np.float32)
    inp.target_stiffnesses = np.zeros(5, dtype=np.float32)
    inp.target_stiffnesses[1] = -1
    _rejects(inp, "must be nonnegative")

    inp = _two_tets()
    inp.external_forces = np.zeros(15, dtype=np.float32)
    inp.external_forces[0] = np.inf
    _rejects(inp, "must be finite")


def test_rejects_active_objectives_on_a_pinned_vertex():
    inp = _two_tets()
    inp.vertex_info[2] = 1
    inp.external_forces = np.zeros(15, dtype=np.float32)
    inp.external_forces[0] = 1
    _rejects(inp, "Pinned vertex 0")

    inp = _two_tets()
    inp.vertex_info[2] = 1
    inp.target_positions = np.zeros(15, dtype=np.float32)
    inp.target_stiffnesses = np.zeros(5, dtype=np.float32)
    inp.target_stiffnesses[0] = 2
    _rejects(inp, "Pinned vertex 0")


def test_rejects_a_mixed_material_solve():
    # inferJGS2MaterialMode (layout.ts:509-522) runs at create, before any
    # device work, so the refusal needs no GPU.
    inp = _two_tets()
    inp.tet_meta[7] = STABLE
    solver.validate_input(inp)
    with pytest.raises(solver.JGS2RangeError, match="(?i)cannot mix"):
        solver.JGS2GpuSolver.create(inp, {"iterations": 1})


def test_host_mirror_refuses_arrays_the_counts_do_not_fit():
    # The C-ABI sizes each array by the counts; the host mirror refuses a
    # mismatch before any pointer reaches the library (the reference's
    # "count does not match" and "must contain N values" checks,
    # ipc-contact-layout.test.ts:169-177, layout.test.ts:183-201).
    inp = _two_tets()
    inp.external_forces = np.zeros(14, dtype=np.float32)
    _rejects(inp, "externalForces must contain 15 values; got 14")
    inp = _two_tets()
    inp.positions = inp.positions.astype(np.float64)
    _rejects(inp, "positions must be a contiguous float32 array")
    inp = _two_tets()
    inp.vertex_info = np.repeat(inp.vertex_info, 2)[::2]  # a strided view
    _rejects(inp, "vertexInfo must be a contiguous uint32 array")
    trough = scenes.trough(1)
    trough.contact_counts = trough.contact_counts.copy()
    trough.contact_counts[0] += 1
    _rejects(trough, r"contactIndices must contain \d+ values")

"""CPU tests: the C-ABI surface, host logic (settings, validation, colouring),
the precompute restatement and the oracle's own consistency.  None of these
needs a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from jgs2_b200 import _ffi, scenes, solver
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(jgs2_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("jgs2.h", "libjgs2.so"), ("jgs2_server.h", "libjgs2.so"),
                                        ("jgs2_scene.h", "libjgs2_scene.so")])
def test_library_exports_every_declared_symbol(header, lib):
    cdll = ctypes.CDLL(os.path.join(_ffi.LIB_DIR, lib))
    missing = [name for name in _declared(header) if not hasattr(cdll, name)]
    assert not missing, f"{lib} lacks {missing}"


def test_default_settings_match_reference_defaults():
    # DEFAULT_JGS2_STEP_SETTINGS (src/simulation/gpu/jgs2-solver.ts:164-187).
    d = solver.default_settings()
    ref = O.DEFAULT_SETTINGS
    for key, value in ref.items():
        got = d[key]
        if key == "gravity":
            np.testing.assert_allclose(got, value, rtol=1e-6)
        else:
            assert got == pytest.approx(value, rel=1e-6), key


def test_parity_mode_override():
    r = solver.resolve_settings({"parityMode": True, "velocityDamping": 0.5, "contactTangentialDamping": 4})
    assert r["velocity_damping"] == 1.0
    assert r["contact_tangential_damping"] == 0.0
    assert r["horizontal_body_correction"] == 0


@pytest.mark.parametrize("overrides,fragment", [
    ({"timestep": 0.0}, "timestep must be positive"),
    ({"residualTolerance": 2e-3}, "residualTolerance must be positive"),
    ({"ipcStepSafety": 1.0}, "ipcStepSafety must be strictly between"),
    ({"velocityDamping": 1.5}, "velocityDamping must be between"),
    ({"schedule": 7}, "Unknown JGS2 schedule"),
    ({"floorStiffness": -1.0}, "floorStiffness must be nonnegative"),
    ({"ipcMinimumDistance": 0.2}, "ipcMinimumDistance must be nonnegative and below"),
])
def test_settings_validation_errors(overrides, fragment):
    with pytest.raises(solver.JGS2RangeError, match=fragment):
        solver.resolve_settings(overrides)


@pytest.fixture(scope="module")
def small_bar():
    return scenes.cantilever(cells=(3, 2, 1), size=(0.3, 0.2, 0.1))


def test_packed_input_validates(small_bar):
    solver.validate_input(small_bar)


@pytest.mark.parametrize("mutate,fragment", [
    (lambda i: i.tet_indices.__setitem__(0, i.vertex_count + 5), "references vertex"),
    (lambda i: i.adjacency.__setitem__(0, i.adjacency[1]), "must equal incident tetrahedron"),
    (lambda i: i.cubature_weights.__setitem__(0, -1.0), "must be nonnegative"),
    (lambda i: i.tet_meta.__setitem__(0, 0.0), "requires positive volume"),
    (lambda i: i.tet_meta.__setitem__(3, 0.0), "Co-rotated tetMeta|tetRestStiffness is required"),
    (lambda i: i.positions.__setitem__(0, np.inf), "positions\\[0\\] must be finite"),
    (lambda i: i.vertex_info.__setitem__(0, 1), "canonical adjacency offset"),
])
def test_input_validation_errors(small_bar, mutate, fragment):
    bad = small_bar.copy()
    mutate(bad)
    with pytest.raises(solver.JGS2RangeError, match=fragment):
        solver.validate_input(bad)


def test_pinned_vertex_rejects_force(small_bar):
    bad = small_bar.copy()
    pinned = np.nonzero(bad.vertex_info.reshape(-1, 4)[:, 2])[0][0]
    bad.external_forces = np.zeros(3 * bad.vertex_count, dtype=np.float32)
    bad.external_forces[3 * pinned] = 1.0
    with pytest.raises(solver.JGS2RangeError, match="cannot have a nonzero external force"):
        solver.validate_input(bad)


def _greedy_coloring(vertex_count, groups):
    """buildGreedyVertexColoring (src/simulation/cpu/vertex-coloring.ts:20-110)
    over conflict groups, with plain Python loops (small cases only): every
    vertex in order takes the smallest colour no neighbour holds."""
    adj = [set() for _ in range(vertex_count)]
    for g in groups:
        u = list(dict.fromkeys(int(x) for x in g))
        for a in range(len(u)):
            for b in range(a + 1, len(u)):
                adj[u[a]].add(u[b])
                adj[u[b]].add(u[a])
    colors = [None] * vertex_count
    count = 0
    for v in range(vertex_count):
        used = {colors[n] for n in adj[v] if colors[n] is not None}
        c = 0
        while c < count and c in used:
            c += 1
        colors[v] = c
        count = max(count, c + 1)
    return np.array(colors, dtype=np.uint32), count


def _python_greedy_coloring(inp):
    """The colouring over buildJGS2InputVertexColoring's groups: every tet,
    and every cubature record's source vertex with its tet's vertices."""
    groups = [list(inp.tet_indices[4 * t:4 * t + 4]) for t in range(inp.tet_count)]
    K = inp.cubature_k
    for v in range(inp.vertex_count):
        for s in range(K):
            r = v * K + s
            t = int(inp.cubature_tet_ids[r])
            if t == 0xFFFFFFFF or not inp.cubature_weights[r] > 0:
                continue
            groups.append([v] + list(inp.tet_indices[4 * t:4 * t + 4]))
    colors, count = _greedy_coloring(inp.vertex_count, groups)
    return colors, count, groups


def test_greedy_coloring_matches_the_reference_known_answer():
    # vertex-coloring.test.ts:6-29: tetrahedron, cloth and IPC groups.
    groups = [[0, 1, 2, 3], [0, 4, 5], [1, 4, 6, 7], [2, 5, 6, 8]]
    colors, count = _greedy_coloring(9, groups)
    assert list(colors) == [0, 1, 2, 3, 2, 1, 0, 3, 3] and count == 4
    counts = np.bincount(colors, minlength=count)
    assert list(counts) == [2, 2, 2, 3]
    assert list(np.concatenate([[0], np.cumsum(counts)])) == [0, 2, 4, 6, 9]
    by_color = [v for c in range(count) for v in range(9) if colors[v] == c]
    assert by_color == [0, 6, 1, 5, 2, 4, 3, 7, 8]
    again, _ = _greedy_coloring(9, list(reversed(groups)))
    assert list(again) == list(colors)


def test_coloring_bit_exact_against_python_and_oracle(small_bar):
    colors, count = solver.build_vertex_coloring(small_bar)
    ref, ref_count, groups = _python_greedy_coloring(small_bar)
    assert count == ref_count
    np.testing.assert_array_equal(colors, ref)
    o = O.OracleSolver(small_bar)
    np.testing.assert_array_equal(o.colors(), colors)
    for g in groups:
        u = list(dict.fromkeys(int(x) for x in g))
        assert len({int(colors[x]) for x in u}) == len(u), "two vertices of one conflict group share a colour"


def test_mulberry32_sequence_is_stable():
    r = scenes.mulberry32(1048583)
    values = [r() for _ in range(4)]
    assert all(0.0 <= v < 1.0 for v in values)
    r2 = scenes.mulberry32(1048583)
    assert [r2() for _ in range(4)] == values


def test_precompute_twelve_tet_fixture_meets_one_percent():
    # buildPhase1NonlinearCubatureDefinition (src/scenes/phase1.ts:287-319) and
    # the reference test "meets the paper's one-percent nonlinear training
    # residual with six samples" (nonlinear-cubature-training.test.ts:380).
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 5000.0, 0.3)
    sc.add_cuboid((2, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), m, 0, 0)
    rest = sc.rest_positions()
    sc.set_pinned((np.isclose(rest[:, 0], 0) & np.isclose(rest[:, 1], 0)).astype(np.uint8))
    stats = sc.precompute(timestep=1 / 60, cubature_k=6)
    assert stats["source_vertices"] == 10
    assert stats["max_residual"] <= 0.01


def test_basis_is_identity_at_the_source_vertex(small_bar):
    # S_i Ubar_i = I (precompute.test.ts:334-438): the block of a record at the
    # source vertex's own slot is the identity.
    K = small_bar.cubature_k
    checked = 0
    for v in range(small_bar.vertex_count):
        for s in range(K):
            r = v * K + s
            t = int(small_bar.cubature_tet_ids[r])
            if t == 0xFFFFFFFF:
                continue
            q = list(small_bar.tet_indices[4 * t:4 * t + 4])
            if v in q:
                block = small_bar.cubature_basis[36 * r + 9 * q.index(v):36 * r + 9 * q.index(v) + 9]
                np.testing.assert_allclose(block.reshape(3, 3), np.eye(3), atol=2e-6)
                checked += 1
    assert checked > 0


def test_patch_precompute_shares_classes():
    inp = scenes.unit_cube(cells=12)
    st = inp.stats
    assert st["training_classes"] < st["source_vertices"] / 2
    assert st["max_records_per_vertex"] == 6
    solver.validate_input(inp)


def test_selection_device_option():
    # The selection place is validated; a GPU selection asked for where no
    # CUDA device is visible fails with a message, and AUTO falls back to the
    # CPU threads there.
    import torch

    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e6, 0.45)
    sc.add_cuboid((3, 2, 2), (0.0, 0.0, 0.0), (0.3, 0.2, 0.2), m, 0, scenes.FACE_X_MIN)
    with pytest.raises(_ffi.JGS2Error, match="selection_device"):
        sc.precompute(timestep=1 / 60, selection_device=3)
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(_ffi.JGS2Error, match="no CUDA device"):
        sc.precompute(timestep=1 / 60, selection_device=scenes.SELECTION_GPU)
    st = sc.precompute(timestep=1 / 60, selection_device=scenes.SELECTION_AUTO)
    assert st["selection_on_gpu"] == 0 and st["source_vertices"] > 0


def test_lumped_masses_sum_to_body_mass(small_bar):
    total = float(small_bar.vertex_rest.reshape(-1, 4)[:, 3].sum())
    assert total == pytest.approx(1000.0 * 0.3 * 0.2 * 0.1, rel=1e-5)


def _local(inp, settings, vertex, d, precision=64):
    L = O.lib()
    L.jgs2_oracle_local_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    o = O.OracleSolver(inp, settings, precision=precision)
    rec = O._settings_struct(O.resolve_settings(None, **settings))
    out = np.zeros(14)
    dd = np.asarray(d, dtype=np.float64)
    L.jgs2_oracle_local_system(o._h, ctypes.byref(rec), vertex, dd.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def test_oracle_restricted_energy_matches_gradient_and_hessian(small_bar):
    settings = dict(timestep=1 / 60, gravity=(0, -9.8, 0), floor_stiffness=0.0, parity_mode=1)
    free = int(np.nonzero(small_bar.vertex_info.reshape(-1, 4)[:, 2] == 0)[0][-1])
    base = _local(small_bar, settings, free, [0, 0, 0])
    g, H = base[:3], base[3:12].reshape(3, 3).T
    for k in range(3):
        eps = 1e-5
        d = np.zeros(3)
        d[k] = eps
        de = _local(small_bar, settings, free, d)[12]
        assert de / eps == pytest.approx(g[k], rel=5e-3, abs=5e-3 * np.abs(g).max())
        quad = (de - eps * g[k]) / (0.5 * eps * eps)
        assert quad == pytest.approx(H[k, k], rel=5e-3)


def test_oracle_exact_complement_converges_without_revert():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((6, 1, 1), (0.0, 0.0, 0.0), (0.6, 0.1, 0.1), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    inp = sc.pack()
    o = O.OracleSolver(inp, dict(timestep=1 / 60, gravity=(0, -9.8, 0), floor_stiffness=0.0, parity_mode=1))
    for _ in range(10):
        o.step_exact_iterations(10)
        h = o.read("history").reshape(64, 32)[:10]
        assert (h[:, 4] == 1).all(), "an iteration was reverted"
        assert h[-1, 19] < 0.05, "relative residual did not drop"


def test_oracle_f32_tracks_f64_on_contractive_scene():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((4, 1, 1), (0.0, 0.0, 0.0), (0.4, 0.1, 0.1), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    inp = sc.pack()
    s = dict(timestep=1 / 60, gravity=(0, -9.8, 0), floor_stiffness=0.0, parity_mode=1)
    a, b = O.OracleSolver(inp, s, 32), O.OracleSolver(inp, s, 64)
    for _ in range(20):
        a.step_exact_iterations(10)
        b.step_exact_iterations(10)
    err = np.abs(a.read("positions") - b.read("positions")).max() / inp.bbox_diagonal()
    assert err < 1e-4

"""Triangle cloth: the St. Venant-Kirchhoff membrane and quadratic dihedral
bending path (the reference's cloth terms, src/simulation/gpu/jgs2-shader.ts:
1225-1844 and their call sites in jgs2Solve, the restricted determinant and
energy, the assembled gate and the convergence gradient).

CPU tests pin the oracle's element math to the reference's own cloth tests
(src/simulation/cpu/cloth.test.ts: zero energy and gradient at rest,
finite-difference gradients within 2e-8), check the scene builder's rest
data, hinges and masses, input validation and the conflict colouring.  GPU
tests compare the CUDA step with the f32 oracle on the same inputs: positions
and velocities within 1e-4 of the bounding-box diagonal.
"""
import ctypes

import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

D = ctypes.POINTER(ctypes.c_double)
TOL = 1e-4

# cloth.test.ts:11-29
MEMBRANE = dict(young=8000.0, poisson=0.3, thickness=0.02)
REST_TRIANGLE = np.array([0, 0, 0, 1, 0, 0, 0.2, 0.8, 0.0])
REST_HINGE = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 1, -1, 0.0])
DEFORMED_TRIANGLE = np.array([-0.03, 0.02, 0.04, 1.08, -0.04, 0.12, 0.16, 0.91, -0.08])
BENT_HINGE = np.array([-0.02, 0.01, 0.03, 1.04, -0.03, -0.02, 0.08, 0.94, 0.22, 0.91, -1.07, -0.14])


def _lib():
    L = O.lib()
    L.jgs2_oracle_cloth_membrane.argtypes = [D, D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, D]
    L.jgs2_oracle_cloth_bending.argtypes = [D, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, D]
    return L


def _rest_triangle_basis():
    # precomputeStVKTriangleRest for REST_TRIANGLE: Dm = [[1, 0.2], [0, 0.8]].
    return np.array([1.0, -0.25, 0.0, 1.25]), 0.4


def membrane(x, inverse, area, precision=64, young=8000.0, poisson=0.3, thickness=0.02):
    out = np.zeros(10)
    x = np.ascontiguousarray(x, dtype=np.float64)
    inv = np.ascontiguousarray(inverse, dtype=np.float64)
    _lib().jgs2_oracle_cloth_membrane(x.ctypes.data_as(D), inv.ctypes.data_as(D), area, young, poisson, thickness,
                                      precision, out.ctypes.data_as(D))
    return out[0], out[1:]


def bending(x, rest_angle, rest_length, stiffness, precision=64):
    out = np.zeros(14)
    x = np.ascontiguousarray(x, dtype=np.float64)
    _lib().jgs2_oracle_cloth_bending(x.ctypes.data_as(D), rest_angle, rest_length, stiffness, precision,
                                     out.ctypes.data_as(D))
    return out[0], out[1:13], bool(out[13])


def central_difference(f, x, h=1e-6):
    g = np.zeros_like(x)
    for k in range(x.size):
        p, m = x.copy(), x.copy()
        p[k] += h
        m[k] -= h
        g[k] = (f(p) - f(m)) / (2 * h)
    return g


def relative_error(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ---- oracle element math against the reference's cloth tests -----------------

def test_membrane_and_bending_vanish_at_rest():
    inv, area = _rest_triangle_basis()
    e, g = membrane(REST_TRIANGLE, inv, area)
    assert e < 1e-24
    assert np.linalg.norm(g) < 1e-12
    be, bg, valid = bending(REST_HINGE, 0.0, 1.0, 2.5)
    assert valid and be == 0.0
    assert np.all(bg == 0.0)


def test_membrane_gradient_matches_finite_differences():
    inv, area = _rest_triangle_basis()
    _, g = membrane(DEFORMED_TRIANGLE, inv, area)
    fd = central_difference(lambda x: membrane(x, inv, area)[0], DEFORMED_TRIANGLE)
    assert relative_error(g, fd) < 2e-8


def test_bending_gradient_matches_finite_differences():
    e, g, valid = bending(BENT_HINGE, 0.0, 1.0, 3.25)
    assert valid and e > 0
    fd = central_difference(lambda x: bending(x, 0.0, 1.0, 3.25)[0], BENT_HINGE)
    assert relative_error(g, fd) < 2e-8


def test_f32_element_math_tracks_f64():
    inv, area = _rest_triangle_basis()
    e64, g64 = membrane(DEFORMED_TRIANGLE, inv, area, 64)
    e32, g32 = membrane(DEFORMED_TRIANGLE, inv, area, 32)
    assert e32 == pytest.approx(e64, rel=1e-5)
    assert relative_error(g32, g64) < 1e-5
    b64, bg64, _ = bending(BENT_HINGE, 0.0, 1.0, 3.25, 64)
    b32, bg32, _ = bending(BENT_HINGE, 0.0, 1.0, 3.25, 32)
    assert b32 == pytest.approx(b64, rel=1e-4)
    assert relative_error(bg32, bg64) < 1e-4


def test_degenerate_hinge_is_invalid():
    # A collinear first triangle (cloth.test.ts:94-104) has no dihedral.
    flat = np.array([0, 0, 0, 1, 0, 0, 0.5, 0, 0, 1, -1, 0.0])
    e, g, valid = bending(flat, 0.0, 1.0, 1.0)
    assert not valid
    assert e == pytest.approx(3.0e38, rel=1e-6)


# ---- scene builder: rest data, hinges, masses ---------------------------------

def _two_triangle_scene(positions=REST_HINGE, triangles=(0, 1, 2, 1, 0, 3), **material):
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.3, scenes.MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_mesh([5, 0, 0, 6, 0, 0, 5, 1, 0, 5, 0, 1], [0, 1, 2, 3], m, pinned=[1, 1, 1, 1])
    sc.add_cloth(positions, np.array(triangles, dtype=np.uint32), None, 1, **material)
    sc.precompute(timestep=1 / 60, cubature_k=1, method=scenes.PRECOMPUTE_PATCH)
    return sc.pack()


def test_scene_rest_basis_area_and_hinge():
    inp = _two_triangle_scene()
    np.testing.assert_allclose(inp.cloth_inverse_rest[:4], [1.0, 0.0, 0.0, 1.0], atol=1e-7)
    np.testing.assert_allclose(inp.cloth_rest_areas, [0.5, 0.5])
    # One interior edge (0, 1): hinge (0, 1, 2, 3) with a zero rest angle
    # (precomputeQuadraticDihedralRest of coplanar, consistently oriented faces).
    np.testing.assert_array_equal(inp.hinge_indices, np.array([4, 5, 6, 7], dtype=np.uint32))
    assert inp.hinge_rest_angles[0] == 0.0
    assert inp.hinge_rest_edge_lengths[0] == 1.0
    solver.validate_input(inp)


def test_scene_rest_basis_of_the_reference_triangle():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.3, scenes.MATERIAL_STABLE_NEO_HOOKEAN)
    sc.add_mesh([5, 0, 0, 6, 0, 0, 5, 1, 0, 5, 0, 1], [0, 1, 2, 3], m, pinned=[1, 1, 1, 1])
    sc.add_cloth(REST_TRIANGLE, np.array([0, 1, 2], dtype=np.uint32), None, 1)
    sc.precompute(timestep=1 / 60, cubature_k=1, method=scenes.PRECOMPUTE_PATCH)
    inp = sc.pack()
    inv, area = _rest_triangle_basis()
    np.testing.assert_allclose(inp.cloth_inverse_rest, inv, rtol=1e-6)
    assert inp.cloth_rest_areas[0] == pytest.approx(area)
    assert inp.hinge_count == 0


def test_cloth_masses_are_areal():
    inp = scenes.cloth_drape(cells=4, prefold=False)
    cloth_vertices = np.unique(inp.cloth_triangles)
    mass = inp.vertex_rest.reshape(-1, 4)[cloth_vertices, 3].astype(np.float64)
    # 1.6 m x 1.6 m sheet, density 480, thickness 0.012.
    assert mass.sum() == pytest.approx(480 * 0.012 * 1.6 * 1.6, rel=1e-5)


def test_inconsistent_orientation_and_non_manifold_edges_are_rejected():
    with pytest.raises(_Error, match="consistent orientation"):
        _two_triangle_scene(triangles=(0, 1, 2, 0, 1, 3))
    quad = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 1, -1, 0, 0.5, 0.5, 1.0])
    with pytest.raises(_Error, match="non-manifold"):
        _two_triangle_scene(positions=quad, triangles=(0, 1, 2, 1, 0, 3, 0, 1, 4))


_Error = (ValueError, RuntimeError)


def test_drape_matches_the_reference_topology():
    # clothDefinition (src/scenes/index.ts:632-720): 25 cloth vertices, 32
    # triangles, 2 pinned cloth vertices and 8 pinned collider vertices.
    inp = scenes.cloth_drape()
    assert inp.cloth_triangle_count == 32
    info = inp.vertex_info.reshape(-1, 4)
    assert int(info[:8, 2].sum()) == 8
    assert int(info[8:, 2].sum()) == 2
    assert int((info[8:, 2] == 0).sum()) == 23  # cloth-demo.spec.ts:126-128
    assert inp.hinge_count == 40
    big = scenes.cloth_sheet()
    assert big.cloth_triangle_count == 32258 and big.hinge_count == 48133



def test_drape_static_candidates_include_cloth_self_contact():
    # cloth-demo.spec.ts:129-132: the topology-filtered IPC candidates include
    # nonlocal cloth self-contact, beside the collider-cloth pairs.
    inp = scenes.cloth_drape(contact=scenes.CONTACT_STATIC)
    solver.validate_input(inp)
    cand = inp.contact_indices.reshape(-1, 4) & np.uint32(0x7FFFFFFF)
    cloth_only = (cand >= 8).all(axis=1)
    assert int(cloth_only.sum()) > 0
    assert int(((cand >= 8).any(axis=1) & ~cloth_only).sum()) > 0

# ---- validation and colouring --------------------------------------------------

def test_cloth_input_validation():
    inp = scenes.cloth_drape()
    bad = inp.copy()
    bad.cloth_triangles[1] = bad.cloth_triangles[0]
    with pytest.raises(solver.JGS2RangeError, match="distinct"):
        solver.validate_input(bad)
    bad = inp.copy()
    bad.cloth_rest_areas[3] = 0.0
    with pytest.raises(solver.JGS2RangeError, match="triangleRestAreas"):
        solver.validate_input(bad)
    bad = inp.copy()
    bad.cloth_material[1] = 0.5
    with pytest.raises(solver.JGS2RangeError, match="Poisson"):
        solver.validate_input(bad)
    bad = inp.copy()
    bad.hinge_rest_edge_lengths[0] = -1.0
    with pytest.raises(solver.JGS2RangeError, match="hingeRestEdgeLengths"):
        solver.validate_input(bad)


def test_cloth_validation_on_the_reference_cases():
    # cloth-layout.test.ts:207-250: index, rest-data and material violations.
    inp = scenes.cloth_drape()
    cases = [
        (lambda b: b.hinge_indices.__setitem__(3, b.hinge_indices[2]), "(?i)distinct"),
        (lambda b: b.cloth_triangles.__setitem__(2, b.vertex_count + 5), "(?i)outside vertexCount"),
        (lambda b: b.cloth_inverse_rest.__setitem__(slice(0, 4), np.array([1, 2, 2, 4], dtype=np.float32)),
         "(?i)invertible"),
        (lambda b: b.cloth_material.__setitem__(3, -1.0), "(?i)nonnegative"),
        (lambda b: b.cloth_material.__setitem__(1, 0.5), "(?i)Poisson"),
        (lambda b: b.cloth_rest_areas.__setitem__(1, 0.0), "(?i)positive"),
    ]
    for mutate, pattern in cases:
        bad = inp.copy()
        mutate(bad)
        with pytest.raises(solver.JGS2RangeError, match=pattern):
            solver.validate_input(bad)


def test_cloth_requires_the_stable_path():
    # jgs2-solver.ts:998-1002: a co-rotated scene cannot carry cloth.
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.3, scenes.MATERIAL_COROTATED_LINEAR)
    sc.add_mesh([5, 0, 0, 6, 0, 0, 5, 1, 0, 5, 0, 1], [0, 1, 2, 3], m, pinned=[1, 1, 1, 1])
    sc.add_cloth(REST_HINGE, np.array([0, 1, 2, 1, 0, 3], dtype=np.uint32), None, 1)
    sc.precompute(timestep=1 / 60, cubature_k=1, method=scenes.PRECOMPUTE_PATCH)
    inp = sc.pack()
    with pytest.raises(solver.JGS2RangeError, match="Triangle cloth requires"):
        solver.JGS2GpuSolver.create(inp, {"parityMode": True})


def test_colouring_separates_cloth_elements():
    inp = scenes.cloth_drape()
    colors, count = solver.build_vertex_coloring(inp)
    o = O.OracleSolver(inp, dict(timestep=1 / 120))
    np.testing.assert_array_equal(colors, o.colors())
    assert count == o.color_count
    for tri in inp.cloth_triangles.reshape(-1, 3):
        assert len(set(colors[tri])) == 3
    for h in inp.hinge_indices.reshape(-1, 4):
        assert len(set(colors[h])) == 4


# ---- oracle step: local system and behaviour ----------------------------------

SETTINGS = dict(timestep=1 / 120, gravity=(0.0, -9.81, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=5)


def _deformed_drape(bending_stiffness=0.045):
    inp = scenes.cloth_drape(bending=bending_stiffness)
    rng = np.random.default_rng(7)
    p = inp.positions.reshape(-1, 4)
    cloth = np.unique(inp.cloth_triangles)
    free = cloth[inp.vertex_info.reshape(-1, 4)[cloth, 2] == 0]
    p[free, :3] += rng.uniform(-0.03, 0.03, size=(free.size, 3)).astype(np.float32)
    return inp


def _local(inp, vertex, d, precision=64):
    L = O.lib()
    L.jgs2_oracle_local_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, D, D]
    o = O.OracleSolver(inp, SETTINGS, precision=precision)
    rec = O._settings_struct(O.resolve_settings(None, **SETTINGS))
    out = np.zeros(14)
    dd = np.asarray(d, dtype=np.float64)
    L.jgs2_oracle_local_system(o._h, ctypes.byref(rec), vertex, dd.ctypes.data_as(D), out.ctypes.data_as(D))
    return out


@pytest.mark.parametrize("bending_stiffness", [0.045, 0.0])
def test_oracle_cloth_local_system_matches_restricted_energy(bending_stiffness):
    inp = _deformed_drape(bending_stiffness)
    v = 8 + 12  # an interior cloth vertex
    base = _local(inp, v, [0, 0, 0])
    g, H = base[:3], base[3:12].reshape(3, 3).T
    for k in range(3):
        eps = 1e-6
        d = np.zeros(3)
        d[k] = eps
        de = _local(inp, v, d)[12]
        assert de / eps == pytest.approx(g[k], rel=2e-3, abs=2e-3 * np.abs(g).max())
        if bending_stiffness == 0.0:
            # Without bending the local Hessian is exact (membrane diagonal block).
            eps = 1e-4
            d[k] = eps
            dp, dm = _local(inp, v, d)[12], _local(inp, v, -d)[12]
            assert (dp + dm) / (eps * eps) == pytest.approx(H[k, k], rel=2e-3)


def test_oracle_drape_falls_without_inversion():
    # cloth-demo.spec.ts:150-160: the free centre falls and the pinned sheet
    # deforms; every frame keeps a positive minimum area stretch.
    inp = scenes.cloth_drape()
    o = O.OracleSolver(inp, SETTINGS, precision=64)
    p0 = o.read("positions").reshape(-1, 4)[:, :3].copy()
    centre = 8 + 2 + 2 * 5
    for _ in range(48):
        o.step_exact_iterations(5)
        h = o.read("history").reshape(64, 32)[:5]
        assert (h[:, 4] == 1).all(), "a cloth iteration was reverted"
        assert (h[:, 1] > 1e-4).all()
    p = o.read("positions").reshape(-1, 4)[:, :3]
    assert p0[centre, 1] - p[centre, 1] > 0.01
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    np.testing.assert_array_equal(p[pinned], p0[pinned])
    assert np.abs(p - p0).max() > 0.02



IPC_DRAPE = dict(timestep=1 / 120, gravity=(0.0, -9.8, 0.0), floor_stiffness=0.0, parity_mode=0,
                 velocity_damping=0.997, horizontal_body_correction=0, contact_tangential_damping=0.0, iterations=5,
                 ipc_activation_distance=0.01, ipc_minimum_distance=0.003, ipc_barrier_stiffness=1e5,
                 ipc_friction_coefficient=0.3, ipc_friction_velocity_epsilon=0.05, max_step=0.01)


@pytest.mark.parametrize("precision", [64, 32])
def test_oracle_ipc_drape_falls_without_crossing(precision):
    # cloth-demo.spec.ts:120-170 with the app's cloth IPC settings
    # (App.tsx:529-575): over 6 x 8 frames the sheet falls onto the pinned
    # collider and deforms; no pair comes closer than the minimum distance
    # (5e-4 tolerance), the sheet reaches the activation band, no element
    # inverts, and the pinned vertices stay put.
    inp = scenes.cloth_drape(contact=scenes.CONTACT_STATIC)
    L = O.lib()
    L.jgs2_oracle_min_contact_distance.restype = ctypes.c_double
    L.jgs2_oracle_min_contact_distance.argtypes = [ctypes.c_void_p]
    o = O.OracleSolver(inp, IPC_DRAPE, precision=precision)
    p0 = o.read("positions").reshape(-1, 4)[:, :3].copy()
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    d = None
    for _ in range(6):
        o.step_frames_exact_iterations(8, 5)
        d = L.jgs2_oracle_min_contact_distance(o._h)
        assert d >= IPC_DRAPE["ipc_minimum_distance"] - 5e-4
        h = o.read("history").reshape(64, 32)[:5]
        assert (h[:, 1] > 1e-4).all(), "an element inverted"
    p = o.read("positions").reshape(-1, 4)[:, :3]
    assert d <= IPC_DRAPE["ipc_activation_distance"] + 5e-4
    centre = 8 + 2 + 2 * 5
    assert p0[centre, 1] - p[centre, 1] > 0.01
    assert np.abs(p - p0).max() > 0.02
    assert np.abs(p[pinned] - p0[pinned]).max() <= 2e-5

# ---- GPU parity ------------------------------------------------------------------

def _camel(s):
    inv = {v: k for k, v in solver.CAMEL.items()}
    return {inv.get(k, k): (bool(v) if k in ("parity_mode", "horizontal_body_correction") else v)
            for k, v in s.items()}


def _compare(inp, gpu_pos, gpu_vel, cpu, h):
    diag = inp.bbox_diagonal()
    g = gpu_pos.reshape(-1, 4)[:, :3]
    c = cpu.read("positions").reshape(-1, 4)[:, :3]
    assert float(np.abs(g - c).max()) / diag <= TOL
    gv = gpu_vel.reshape(-1, 4)[:, :3]
    cv = cpu.read("velocities").reshape(-1, 4)[:, :3]
    assert float(np.abs(gv - cv).max()) * h / diag <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [0, 1])
def test_cloth_drape_gpu_matches_oracle(schedule):
    inp = scenes.cloth_drape()
    s = dict(SETTINGS, schedule=schedule)
    gpu = solver.JGS2GpuSolver.create(inp, _camel(s))
    assert gpu.clothTriangleCount == 32
    assert gpu.globalizationElementCount == inp.tet_count + 32
    cpu = O.OracleSolver(inp, s, precision=32)
    for _ in range(24):
        gpu.stepExactIterations(5)
        cpu.step_exact_iterations(5)
    _compare(inp, gpu.readPositions(), gpu.readVelocities(), cpu, 1 / 120)
    gd = gpu.readGlobalizationDiagnostics()
    ch = cpu.read("history").reshape(64, 32)[:5]
    gh = gd["history"].reshape(-1, 32)[:5]
    assert gh.shape == (5, 32)
    np.testing.assert_array_equal(gh[:, 4], ch[:, 4])  # accept flags
    np.testing.assert_allclose(gh[:, 1], ch[:, 1], rtol=1e-4)  # candidate minimum stretch
    gpu.destroy()


@pytest.mark.gpu
def test_deformed_bent_cloth_gpu_matches_oracle():
    inp = _deformed_drape()
    gpu = solver.JGS2GpuSolver.create(inp, _camel(SETTINGS))
    cpu = O.OracleSolver(inp, SETTINGS, precision=32)
    for _ in range(10):
        gpu.stepExactIterations(5)
        cpu.step_exact_iterations(5)
    _compare(inp, gpu.readPositions(), gpu.readVelocities(), cpu, 1 / 120)
    gpu.destroy()


@pytest.mark.gpu
def test_cloth_sheet_gpu_matches_oracle():
    inp = scenes.cloth_sheet(cells=24)
    s = dict(SETTINGS, iterations=10)
    gpu = solver.JGS2GpuSolver.create(inp, _camel(s))
    cpu = O.OracleSolver(inp, s, precision=32)
    for _ in range(8):
        gpu.stepExactIterations(10)
        cpu.step_exact_iterations(10)
    _compare(inp, gpu.readPositions(), gpu.readVelocities(), cpu, 1 / 120)
    gpu.destroy()


@pytest.mark.gpu
def test_cloth_batch_matches_alone():
    parts = [scenes.cloth_drape(), scenes.cantilever(cells=(6, 2, 2)), scenes.cloth_sheet(cells=8)]
    opts = _camel(SETTINGS)
    batch = solver.JGS2Batch.create(parts, opts)
    alone = [solver.JGS2GpuSolver.create(p, opts) for p in parts]
    batch.stepFrames(4, exactIterations=5)
    for a in alone:
        a.stepFramesExactIterations(4, 5)
    for i, a in enumerate(alone):
        if parts[i].cloth_triangles is not None:
            # The same kernels alone and in the batch: bitwise.
            np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(), err_msg=f"scene {i}")
        else:
            # Alone, a tet-only scene runs the kernel variant without cloth
            # terms, whose floating-point contractions may differ.
            err = np.abs(batch.readPositions(i) - a.readPositions()).max() / parts[i].bbox_diagonal()
            assert err <= TOL, f"scene {i}: {err}"
        a.destroy()
    batch.destroy()

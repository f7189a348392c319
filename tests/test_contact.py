"""IPC contact: static vertex-triangle / edge-edge candidates, the log
barrier with its PSD normal block, lagged friction, the restricted line
search terms, the Lipschitz safe step and the exact validation of the scaled
pose (src/simulation/gpu/jgs2-shader.ts:233-874, 1997-2038, 2137-2196,
2694-2917; src/simulation/gpu/ipc-contact-wgsl.ts).

CPU tests pin the oracle's contact math and the candidate enumeration to the
reference's own contact tests (src/simulation/cpu/ipc-contact.test.ts; the
scalar cases of src/simulation/gpu/ipc-contact-wgsl.test.ts:144-245: barrier
signs, the Lipschitz safe-step cap, lagged friction, the PSD normal block) and to
the documented candidate count of the 10-box trough (docs/ROADMAP.md:319-320:
92 vertices, 72 tets, 31 801 static VT/EE candidates), and check the
reference's trough feasibility bounds (tests/e2e/ipc-trough-demo.spec.ts:
124-170) on the oracle.  GPU tests compare the CUDA step with the f32 oracle
(positions and velocities within 1e-4 of the bounding-box diagonal) and check
the same trough bounds on the device.
"""
import ctypes
import math

import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

D = ctypes.POINTER(ctypes.c_double)
TOL = 1e-4
DMIN = 0.003


def _lib():
    L = O.lib()
    L.jgs2_oracle_ipc_barrier.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, D]
    L.jgs2_oracle_ipc_friction.argtypes = [ctypes.c_double, ctypes.c_double, D]
    L.jgs2_oracle_ipc_contact.argtypes = [ctypes.c_uint32, D, D]
    L.jgs2_oracle_min_contact_distance.argtypes = [ctypes.c_void_p]
    L.jgs2_oracle_min_contact_distance.restype = ctypes.c_double
    return L


def barrier(d, dhat, precision=64):
    out = np.zeros(3)
    _lib().jgs2_oracle_ipc_barrier(d, dhat, precision, out.ctypes.data_as(D))
    return out


def friction(s, eps):
    out = np.zeros(2)
    _lib().jgs2_oracle_ipc_friction(s, eps, out.ctypes.data_as(D))
    return out


def contact(kind, x):
    out = np.zeros(9)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    _lib().jgs2_oracle_ipc_contact(kind, xx.ctypes.data_as(D), out.ctypes.data_as(D))
    return out


def snake(settings):
    s = {solver.CAMEL.get(k, k): v for k, v in settings.items()}
    return {k: (1 if v is True else 0 if v is False else v) for k, v in s.items()}


# ---- contact math against ipc-contact.test.ts ----------------------------------

def test_barrier_matches_closed_form_and_finite_differences():
    dhat, d, h = 1.2, 0.37, 1e-5
    b0, b1, b2 = barrier(d, dhat)
    assert b0 == pytest.approx(-((d - dhat) ** 2) * math.log(d / dhat), abs=1e-14)
    assert b1 == pytest.approx((barrier(d + h, dhat)[0] - barrier(d - h, dhat)[0]) / (2 * h), abs=1e-8)
    fd2 = (barrier(d + h, dhat)[0] - 2 * b0 + barrier(d - h, dhat)[0]) / (h * h)
    assert b2 == pytest.approx(fd2, abs=1e-4)
    assert list(barrier(dhat, dhat)) == [0.0, 0.0, 0.0]
    assert barrier(2.0, dhat)[0] == 0.0
    # Outside the barrier's domain the kernels return zero; callers reject d <= 0.
    assert list(barrier(0.0, dhat)) == [0.0, 0.0, 0.0]


def test_friction_smoothing_branches():
    eps = 0.2
    assert friction(0.0, eps)[0] == 0.0
    assert friction(0.1, eps)[0] == pytest.approx(0.75, abs=1e-14)
    # f1 is the derivative of the dissipation potential (mu = lambda = 1).
    h = 1e-6
    fd = (friction(0.1 + h, eps)[1] - friction(0.1 - h, eps)[1]) / (2 * h)
    assert friction(0.1, eps)[0] == pytest.approx(fd, abs=1e-9)
    assert friction(eps, eps)[0] == 1.0
    assert friction(2 * eps, eps)[0] == 1.0
    # The potential is C1 at the smoothing threshold.
    assert friction(eps, eps)[1] == pytest.approx(eps - eps / 3.0)


def ipc_scalar(which, args, precision=64):
    L = _lib()
    L.jgs2_oracle_ipc_scalar.argtypes = [ctypes.c_int, D, ctypes.c_int, D]
    L.jgs2_oracle_ipc_scalar.restype = ctypes.c_double
    a = np.ascontiguousarray(args, dtype=np.float64)
    out = np.zeros(9)
    value = L.jgs2_oracle_ipc_scalar(which, a.ctypes.data_as(D), precision, out.ctypes.data_as(D))
    return value, out.reshape(3, 3)


def test_barrier_signs_and_derivatives_inside_the_band():
    # ipc-contact-wgsl.test.ts:144-177 (d-hat 2.3): inside the band the value
    # is positive, the first derivative negative, the second positive, and
    # both derivatives match central differences to 5 decimals.
    dhat, eps = 2.3, 1e-6
    for d in (0.17, 0.61, 1.4, 2.1):
        b0, b1, b2 = barrier(d, dhat)
        fd1 = (barrier(d + eps, dhat)[0] - barrier(d - eps, dhat)[0]) / (2 * eps)
        fd2 = (barrier(d + eps, dhat)[1] - barrier(d - eps, dhat)[1]) / (2 * eps)
        assert abs(b1 - fd1) < 5e-6 and abs(b2 - fd2) < 5e-6
        assert b0 > 0 and b1 < 0 and b2 > 0
    assert barrier(dhat, dhat)[0] == 0.0
    assert barrier(3.0, dhat)[1] == 0.0
    assert barrier(0.0, dhat)[2] == 0.0


@pytest.mark.parametrize("precision", [64, 32])
def test_safe_step_cap_respects_the_lipschitz_bound(precision):
    # ipc-contact-wgsl.test.ts:197-215.
    for d, dmin, bound, safety in ((0.04, 0.001, 0.2, 0.9), (0.2, 0.01, 0.05, 0.9), (0.02, 0.005, 3, 1)):
        alpha, _ = ipc_scalar(0, [d, dmin, bound, safety], precision)
        assert 0.0 <= alpha <= 1.0
        slack = 1e-12 if precision == 64 else 1e-7
        assert alpha * bound <= min(bound, min(1.0, max(0.0, safety)) * (d - dmin)) + slack
    assert ipc_scalar(0, [0.04, 0.001, 0.0, 0.9], precision)[0] == 1.0
    assert ipc_scalar(0, [0.001, 0.001, 1.0, 0.9], precision)[0] == 0.0
    assert ipc_scalar(0, [math.nan, 0.0, 1.0, 0.9], precision)[0] == 0.0
    assert ipc_scalar(0, [0.04, -0.001, 1.0, 0.9], precision)[0] == 0.0
    assert ipc_scalar(0, [0.04, 0.001, -1.0, 0.9], precision)[0] == 0.0


def test_lagged_friction_is_c1_and_nonnegative_through_zero_slip():
    # ipc-contact-wgsl.test.ts:217-245 (threshold 0.03, coefficient 0.4,
    # lagged normal force 120): f1 is the derivative of f0, f0(0) = eps/3,
    # and the dissipation is c N (f0(s) - f0(0)), zero at zero slip.
    eps, c, n = 0.03, 0.4, 120.0
    assert friction(0.0, eps)[0] == 0.0 and friction(eps, eps)[0] == 1.0
    for s in (0.001, 0.008, 0.02, 0.029, 0.04):
        h = 1e-7
        fd = (friction(s + h, eps)[1] - friction(s - h, eps)[1]) / (2 * h)
        assert abs(friction(s, eps)[0] - fd) < 5e-7
        dissipation, _ = ipc_scalar(1, [s, eps, c, n])
        assert dissipation >= 0.0
        assert dissipation == pytest.approx(c * n * friction(s, eps)[1], abs=1e-12)
    assert ipc_scalar(1, [0.0, eps, c, n])[0] == 0.0
    # Negative coefficients and normal forces are clamped to zero.
    assert ipc_scalar(1, [0.02, eps, -0.4, n])[0] == 0.0
    assert ipc_scalar(1, [0.02, eps, c, -120.0])[0] == 0.0


@pytest.mark.parametrize("precision", [64, 32])
def test_normal_hessian_block_is_psd(precision):
    # ipc-contact-wgsl.test.ts:180-195: the block is max(scale, 0) n n^T, so a
    # negative barrier curvature contributes nothing.
    normal = np.array([0.6, 0.0, 0.8])
    for scale in (-3.0, 0.0, 17.5):
        _, h = ipc_scalar(2, list(normal) + [scale], precision)
        want = max(scale, 0.0) * np.outer(normal, normal)
        np.testing.assert_allclose(h, want, atol=1e-12 if precision == 64 else 1e-5)
        # f32: the rank-one block's zero eigenvalues carry its rounding.
        floor = 1e-12 if precision == 64 else 1e-7 * max(scale, 1.0)
        assert np.linalg.eigvalsh(0.5 * (h + h.T)).min() >= -floor


def test_point_triangle_distances_and_degeneracies():
    p = [0.25, 1, 0.25]
    assert contact(0, p + [0, 0, 0, 1, 0, 0, 0, 0, 1])[0] == pytest.approx(1.0)
    assert contact(0, p + [0, 0, 0, 2, 0, 0, 1, 0, 0])[0] == pytest.approx(math.sqrt(1.0625), abs=1e-14)
    assert contact(0, p + [0, 0, 0] * 3)[0] == pytest.approx(math.sqrt(1.125), abs=1e-14)
    k = contact(0, p + [0, 0, 0, 1, 0, 0, 0, 0, 1])
    assert k[8] == 1.0
    np.testing.assert_allclose(k[1:4], [0, 1, 0], atol=1e-14)
    # sum_i w_i x_i = point_a - point_b
    x = np.array(p + [0, 0, 0, 1, 0, 0, 0, 0, 1]).reshape(4, 3)
    np.testing.assert_allclose(k[4:8] @ x, [0, 1, 0], atol=1e-14)


def test_edge_edge_crossing_parallel_and_collapsed():
    assert contact(1, [-1, 0, 0, 1, 0, 0, 0, -1, 0.5, 0, 1, 0.5])[0] == pytest.approx(0.5)
    assert contact(1, [0, 0, 0, 1, 0, 0, 0, 0.3, 0, 1, 0.3, 0])[0] == pytest.approx(0.3)
    assert contact(1, [0, 0, 0, 0, 0, 0, 0, 2, 0, 0, 2, 0])[0] == pytest.approx(2.0)
    k = contact(1, [-1, 0, 0, 1, 0, 0, 0, -1, 0.5, 0, 1, 0.5])
    x = np.array([-1, 0, 0, 1, 0, 0, 0, -1, 0.5, 0, 1, 0.5], dtype=float).reshape(4, 3)
    np.testing.assert_allclose(k[4:8] @ x, [0, 0, -0.5], atol=1e-14)


# ---- candidate enumeration -------------------------------------------------------

def _tuples(indices):
    return [tuple(int(v) for v in indices[i:i + 4]) for i in range(0, len(indices), 4)]


def test_candidates_filter_one_rings_and_are_order_independent():
    # ipc-contact.test.ts:104-150
    fwd, vt, ee = scenes.static_contact_candidates(6, [0, 1, 2, 3, 4, 5])
    assert (vt, ee) == (6, 9)
    t = _tuples(fwd)
    assert t[:6] == [(0, 3, 4, 5), (1, 3, 4, 5), (2, 3, 4, 5), (3, 0, 1, 2), (4, 0, 1, 2), (5, 0, 1, 2)]
    assert t[6] == (0, 1, 3, 4) and t[-1] == (1, 2, 4, 5)
    rev, vt2, ee2 = scenes.static_contact_candidates(6, [5, 3, 4, 2, 1, 0, 4, 5, 3])
    np.testing.assert_array_equal(rev, fwd)
    patch, vt3, ee3 = scenes.static_contact_candidates(4, [0, 1, 2, 2, 1, 3])
    assert (vt3, ee3) == (0, 0) and patch.size == 0


def test_trough_matches_the_reference_candidate_count():
    inp = scenes.trough(10)
    assert (inp.vertex_count, inp.tet_count) == (92, 72)
    assert inp.contact_candidate_count == 31801
    solver.validate_input(inp)


def test_trough_box_count_configures_bodies():
    # ipc-trough-demo.spec.ts:49-72: boxes=3 gives four bodies (the trough
    # and three boxes); the ten-box trough is the roadmap's 92 vertices and
    # 72 tets (docs/ROADMAP.md:319-320).
    for boxes in (1, 3, 10):
        inp = scenes.trough(boxes)
        assert len(np.unique(inp.vertex_info.reshape(-1, 4)[:, 3])) == boxes + 1
    ten = scenes.trough(10)
    assert (ten.vertex_count, ten.tet_count) == (92, 72)


def _contact_demo():
    """contactDefinition (src/scenes/index.ts:455-540): a pinned slab, two
    deformable blocks (the upper one sliding at +0.8 m/s in x) and a
    same-body anchor / faller pair, with the static IPC superset."""
    sc = scenes.Scene()
    slab = sc.add_material(1000.0, 120000.0, 0.34)
    lower = sc.add_material(900.0, 65000.0, 0.36)
    upper = sc.add_material(850.0, 75000.0, 0.35)
    pair = sc.add_material(825.0, 62000.0, 0.35)
    sc.add_cuboid((1, 1, 1), (-1.4, -0.18, -0.7), (2.8, 0.18, 1.4), slab, 0, 63)
    sc.add_cuboid((1, 1, 1), (-0.45, 0.08, -0.38), (0.9, 0.56, 0.76), lower, 1, 0)
    sc.add_cuboid((1, 1, 1), (-0.42, 0.74, -0.34), (0.84, 0.52, 0.68), upper, 2, 0)
    sc.add_mesh([-1.22, 0.02, -0.58, -1.22, 0.24, -0.58, -1.22, 0.24, -0.16, -0.76, 0.24, -0.58], [0, 1, 2, 3], pair,
                pinned=[1, 1, 1, 1], body=3)
    sc.add_mesh([-1.2, 0.28, -0.56, -1.2, 0.28, -0.18, -0.78, 0.28, -0.56, -1.2, 0.5, -0.56], [0, 1, 2, 3], pair,
                pinned=[0, 0, 0, 0], body=3)
    sc.set_contact(scenes.CONTACT_STATIC)
    sc.precompute(timestep=1 / 60, cubature_k=6)
    base = sc.pack()
    body = base.vertex_info.reshape(-1, 4)[:, 3]
    pos = base.positions.reshape(-1, 4).copy()
    vel = np.zeros_like(pos)
    vel[body == 2, 0] = 0.8
    sc.set_initial_state(pos.reshape(-1), vel.reshape(-1), pin_at_initial=False)
    return sc.pack()


@pytest.mark.parametrize("precision", [64, 32])
def test_oracle_contact_demo_friction_opposes_sliding(precision):
    # ipc-contact-demo.spec.ts:85-145 with the app's IPC settings
    # (App.tsx:529-575), 36 frames: without friction the upper block keeps
    # more than 0.05 m of its +x slide, and friction reduces that travel by
    # more than 1 mm. Both runs stay finite and no pair crosses the minimum
    # distance.
    inp = _contact_demo()
    body = inp.vertex_info.reshape(-1, 4)[:, 3]
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3]
    upper = body == 2
    L = _lib()
    L.jgs2_oracle_min_contact_distance.restype = ctypes.c_double
    L.jgs2_oracle_min_contact_distance.argtypes = [ctypes.c_void_p]
    travel = {}
    for mu in (0.45, 0.0):
        settings = dict(timestep=1 / 60, gravity=(0.0, -9.81, 0.0), floor_stiffness=0.0, floor_height=-0.18,
                        parity_mode=0, velocity_damping=0.997, iterations=7, ipc_activation_distance=0.08,
                        ipc_minimum_distance=0.003, ipc_barrier_stiffness=1e5, ipc_friction_coefficient=mu,
                        ipc_friction_velocity_epsilon=0.05, max_step=0.075)
        o = O.OracleSolver(inp, settings, precision=precision)
        p0 = o.read("positions").reshape(-1, 4)[:, :3].copy()
        for frames in (2, 2, 4, 12, 12, 4):
            o.step_frames(frames)
            assert L.jgs2_oracle_min_contact_distance(o._h) >= 0.003 - 5e-4
        p = o.read("positions").reshape(-1, 4)[:, :3]
        assert np.isfinite(p).all()
        com = lambda x: float((mass[upper] * x[upper, 0]).sum() / mass[upper].sum())  # noqa: E731
        travel[mu] = com(p) - com(p0)
    assert travel[0.0] > 0.05
    assert travel[0.0] - travel[0.45] > 0.001


def test_contact_validation_and_create_checks():
    inp = scenes.trough(1)
    bad = inp.copy()
    bad.contact_indices[1] = bad.contact_indices[0]
    with pytest.raises(solver.JGS2RangeError, match="distinct"):
        solver.validate_input(bad)
    # The box lowered onto the trough wall, within the minimum distance: the
    # source pose is infeasible (jgs2-solver.ts:1040-1070); the check runs
    # before any device work.
    sunk = inp.copy()
    p = sunk.positions.reshape(-1, 4)
    p[12:, 1] -= 1.486
    o = O.OracleSolver(sunk, {}, precision=64)
    assert 0.0 < _lib().jgs2_oracle_min_contact_distance(o._h) < DMIN
    with pytest.raises(solver.JGS2RangeError, match="initially feasible"):
        solver.JGS2GpuSolver.create(sunk, scenes.TROUGH_SETTINGS)


# ---- oracle trough behaviour (ipc-trough-demo.spec.ts:124-170) -------------------

def _oracle_trough(boxes, frames, precision=64):
    inp = scenes.trough(boxes)
    o = O.OracleSolver(inp, snake(scenes.TROUGH_SETTINGS), precision=precision)
    return inp, o


def _body_stats(inp, pos):
    body = inp.vertex_info.reshape(-1, 4)[:, 3]
    out = []
    for b in range(1, body.max() + 1):
        p = pos[body == b]
        out.append((p.mean(axis=0), p[:, 1].min()))
    return out


def test_oracle_trough_pile_stays_feasible():
    inp, o = _oracle_trough(4, 96)
    L = _lib()
    p0 = o.read("positions").reshape(-1, 4)[:, :3].copy()
    start = _body_stats(inp, p0)
    minimum = L.jgs2_oracle_min_contact_distance(o._h)
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    for frame in range(1, 97):
        o.step()
        if frame % 12 == 0:
            d = L.jgs2_oracle_min_contact_distance(o._h)
            assert d > DMIN - 5e-4, f"frame {frame} IPC distance {d}"
            minimum = min(minimum, d)
            pos = o.read("positions").reshape(-1, 4)[:, :3]
            assert np.isfinite(pos).all()
            assert np.abs(pos[pinned] - p0[pinned]).max() < 2e-5
    pos = o.read("positions").reshape(-1, 4)[:, :3]
    boxes = inp.vertex_info.reshape(-1, 4)[:, 3] != 0
    assert (np.abs(pos[boxes, 0]) < 2.2).all() and (np.abs(pos[boxes, 2]) < 1.5).all()
    for (c0, _), (c1, miny) in zip(start, _body_stats(inp, pos)):
        assert c1[1] < c0[1] - 0.1 and c1[1] < 2.0
        assert miny > 0.05
    assert minimum < 0.08, "no IPC pair entered the activation band"


# ---- GPU -----------------------------------------------------------------------------

def _in_contact_state(boxes=2, frames=44):
    """The trough after `frames` f64 oracle frames (boxes resting on the V),
    as a new input whose initial pose and velocities are that state."""
    inp, o = _oracle_trough(boxes, frames)
    for _ in range(frames):
        o.step()
    state = inp.copy()
    state.positions = o.read("positions").astype(np.float32).reshape(-1, 4).copy()
    state.positions[:, 3] = 1.0
    state.positions = state.positions.reshape(-1)
    vel = o.read("velocities").astype(np.float32).reshape(-1, 4).copy()
    vel[:, 3] = 0.0
    state.velocities = vel.reshape(-1)
    return state


def _compare(inp, gpu, cpu, h):
    diag = inp.bbox_diagonal()
    g = gpu.readPositions().reshape(-1, 4)[:, :3]
    c = cpu.read("positions").reshape(-1, 4)[:, :3]
    err = float(np.abs(g - c).max()) / diag
    assert err <= TOL, err
    gv = gpu.readVelocities().reshape(-1, 4)[:, :3]
    cv = cpu.read("velocities").reshape(-1, 4)[:, :3]
    assert float(np.abs(gv - cv).max()) * h / diag <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [0, 1])
def test_trough_in_contact_gpu_matches_oracle(schedule):
    inp = _in_contact_state()
    s = dict(scenes.TROUGH_SETTINGS, schedule=schedule)
    gpu = solver.JGS2GpuSolver.create(inp, s)
    assert gpu.info()["contact_candidate_count"] == inp.contact_candidate_count
    cpu = O.OracleSolver(inp, snake(s), precision=32)
    for _ in range(6):
        gpu.stepExactIterations(3)
        cpu.step_exact_iterations(3)
    _compare(inp, gpu, cpu, 1 / 60)
    assert _lib().jgs2_oracle_min_contact_distance(cpu._h) < 0.08, "the compared frames had no active contact"
    gpu.destroy()


@pytest.mark.gpu
def test_trough_falling_gpu_matches_oracle():
    inp = scenes.trough(2)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    cpu = O.OracleSolver(inp, snake(scenes.TROUGH_SETTINGS), precision=32)
    for _ in range(20):
        gpu.step()
        cpu.step()
    _compare(inp, gpu, cpu, 1 / 60)
    gpu.destroy()


@pytest.mark.gpu
def test_trough_pile_stays_feasible_on_gpu():
    # ipc-trough-demo.spec.ts:124-170 with the reference's 10 boxes.
    inp = scenes.trough(10)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    checker = O.OracleSolver(inp, snake(scenes.TROUGH_SETTINGS), precision=64)
    L = _lib()
    p0 = gpu.readPositions().reshape(-1, 4)[:, :3].copy()
    start = _body_stats(inp, p0)
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    minimum = 1e30
    for frame in range(12, 97, 12):
        gpu.stepFrames(12)
        pos4 = gpu.readPositions()
        pos = pos4.reshape(-1, 4)[:, :3]
        assert np.isfinite(pos).all()
        assert np.abs(pos[pinned] - p0[pinned]).max() < 2e-5
        # Exact f64 distances of the device pose, measured by the oracle.
        checker_in = inp.copy()
        checker_in.positions = pos4.copy()
        measure = O.OracleSolver(checker_in, {}, precision=64)
        d = L.jgs2_oracle_min_contact_distance(measure._h)
        del measure
        assert d > DMIN - 5e-4, f"frame {frame} IPC distance {d}"
        minimum = min(minimum, d)
    pos = gpu.readPositions().reshape(-1, 4)[:, :3]
    boxes = inp.vertex_info.reshape(-1, 4)[:, 3] != 0
    assert (np.abs(pos[boxes, 0]) < 2.2).all() and (np.abs(pos[boxes, 2]) < 1.5).all()
    for (c0, _), (c1, miny) in zip(start, _body_stats(inp, pos)):
        assert c1[1] < c0[1] - 0.1 and c1[1] < 2.0
        assert miny > 0.05
    assert minimum < 0.08
    diag = gpu.readGlobalizationDiagnostics()
    assert np.isfinite(diag["control"]).all()
    del checker
    gpu.destroy()


@pytest.mark.gpu
def test_minimum_distance_is_fixed_after_create():
    inp = scenes.trough(1)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    with pytest.raises(solver.JGS2RangeError, match="ipcMinimumDistance is fixed"):
        gpu.step({"ipcMinimumDistance": 0.004})
    gpu.step({"ipcMinimumDistance": DMIN})
    gpu.destroy()


@pytest.mark.gpu
def test_contact_batch_matches_alone():
    # Contact scenes run the same kernels alone and in the batch: bitwise.  A
    # tet-only scene runs the kernel variant without cloth and contact terms
    # alone, whose floating-point contractions may differ: parity tolerance.
    free_box = scenes.batched_scenes(count=1, min_cells=2, max_cells=3)[0]
    parts = [scenes.trough(2), free_box, scenes.trough(1)]
    opts = [dict(scenes.TROUGH_SETTINGS), dict(timestep=1 / 60, floorStiffness=0.0, parityMode=True),
            dict(scenes.TROUGH_SETTINGS)]
    batch = solver.JGS2Batch.create(parts, opts)
    alone = [solver.JGS2GpuSolver.create(p, o) for p, o in zip(parts, opts)]
    for frames, check_free in ((4, True), (26, False)):
        batch.stepFrames(frames, exactIterations=3)
        for a in alone:
            a.stepFramesExactIterations(frames, 3)
        for i, a in enumerate(alone):
            if parts[i].contact_candidate_count:
                np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(), err_msg=f"scene {i}")
            elif check_free:
                err = np.abs(batch.readPositions(i) - a.readPositions()).max() / parts[i].bbox_diagonal()
                assert err <= TOL, f"scene {i}: {err}"
    for a in alone:
        a.destroy()
    batch.destroy()

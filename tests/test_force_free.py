"""Force-free conservation, the reference's P0-EC-10/11
(tests/e2e/jgs2.spec.ts:470-575).

The fixture is the reference's canonical force-free cuboid
(src/scenes/canonical-phase0.ts:20-166):
- an unconstrained 2x2x2-hex cube, origin -0.5, edge 1 m;
- density 1000, E 8e4, nu 0.3 (src/simulation/cpu/phase0-canonical.ts:42-48);
- exact all-element cubature, one weight-one record per tetrahedron;
- h = 1/120, 12 iterations, no gravity or floor, parity mode.

It starts at its rest shape rotated by the Euler angles (0.17, -0.23, 0.31),
applied about x, then y, then z (src/simulation/cpu/mesh.ts:210-235). Its
initial velocity is the rigid field v_cm + w x (x - x_cm), with
v_cm = (0.37, -0.11, 0.23), w = (0.41, 0.29, -0.19) and x_cm the lumped-mass
centre (canonical-phase0.ts:38-41, 232-268).

After 4 s (480 frames) two quantities are checked: the total linear momentum
and the total angular momentum about the origin
(src/simulation/diagnostics.ts:166-207). Each must differ from its initial
value by less than 0.005. The linear error is normalised by max(|P0|, M d)
and the angular one by max(|L0|, M d^2), with M the total mass and d the
initial bounding-box diagonal (jgs2.spec.ts:540-575).

The reference's frozen corpus of 32 seeded rigid velocities (P0-CORPUS-01,
jgs2.spec.ts:589-686) runs in its quick form: every case for one frame, and
cases 0 and 27 for 120 frames. Each case must stay finite and uninverted,
and hold the same momentum bound. The corpus generator is pinned to the
reference's frozen cases 0 and 31.
"""
import functools
import math

import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

MOMENTUM_TOL = 0.005
POSITION_TOL = 1e-4  # of the bounding-box diagonal
FRAMES = 480  # 4 s at h = 1/120
SETTINGS = dict(timestep=1 / 120, gravity=(0.0, 0.0, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=12)


def _euler_xyz(e):
    cx, sx = math.cos(e[0]), math.sin(e[0])
    cy, sy = math.cos(e[1]), math.sin(e[1])
    cz, sz = math.cos(e[2]), math.sin(e[2])
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ ry @ rx


@functools.lru_cache(maxsize=1)
def _fixture():
    """The fixture's scene (precomputed once), its lumped vertex masses and
    its rotated initial pose."""
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 8.0e4, 0.3)
    sc.add_cuboid((2, 2, 2), (-0.5, -0.5, -0.5), (1.0, 1.0, 1.0), m, 0, 0)
    sc.precompute(timestep=SETTINGS["timestep"], cubature_k=sc.tet_count, exact_complement=1)
    mass = sc.pack().vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    rest = sc.rest_positions()
    pos = np.ones((rest.shape[0], 4), dtype=np.float32)
    pos[:, :3] = rest @ _euler_xyz((0.17, -0.23, 0.31)).T
    return sc, mass, pos


def _force_free_cuboid(v_cm=(0.37, -0.11, 0.23), omega=(0.41, 0.29, -0.19)):
    """The fixture's packed input with the rigid velocity field
    v_cm + omega x (x - x_cm), and its lumped vertex masses."""
    sc, mass, pos = _fixture()
    centre = (mass[:, None] * pos[:, :3]).sum(0) / mass.sum()
    vel = np.zeros_like(pos)
    vel[:, :3] = np.asarray(v_cm) + np.cross(np.asarray(omega), pos[:, :3] - centre)
    sc.set_initial_state(pos.reshape(-1), vel.reshape(-1), pin_at_initial=False)
    return sc.pack(), mass


def _momenta(positions, velocities, mass):
    x = positions.reshape(-1, 4)[:, :3].astype(np.float64)
    p = mass[:, None] * velocities.reshape(-1, 4)[:, :3].astype(np.float64)
    return p.sum(0), np.cross(x, p).sum(0)


def _momentum_errors(inp, mass, positions, velocities):
    p0, l0 = _momenta(inp.positions, inp.velocities, mass)
    p1, l1 = _momenta(positions, velocities, mass)
    m, d = mass.sum(), inp.bbox_diagonal()
    linear = float(np.linalg.norm(p1 - p0) / max(np.linalg.norm(p0), m * d))
    angular = float(np.linalg.norm(l1 - l0) / max(np.linalg.norm(l0), m * d * d))
    return linear, angular


def test_fixture_moves_rigidly_at_start():
    inp, mass = _force_free_cuboid()
    assert inp.vertex_count == 27 and inp.tet_count == 48
    assert abs(mass.sum() - 1000.0) < 1e-3
    p0, l0 = _momenta(inp.positions, inp.velocities, mass)
    np.testing.assert_allclose(p0, 1000.0 * np.array([0.37, -0.11, 0.23]), rtol=1e-5)
    assert np.linalg.norm(l0) > 0.0


def test_oracle_conserves_momentum_force_free():
    inp, mass = _force_free_cuboid()
    cpu = O.OracleSolver(inp, SETTINGS, precision=32)
    cpu.step_frames(FRAMES)
    linear, angular = _momentum_errors(inp, mass, cpu.read("positions"), cpu.read("velocities"))
    print(f"oracle f32, {FRAMES} frames: linear {linear:.3e}, angular {angular:.3e}")
    assert linear < MOMENTUM_TOL and angular < MOMENTUM_TOL


@pytest.mark.gpu
def test_gpu_conserves_momentum_force_free():
    inp, mass = _force_free_cuboid()
    camel = dict(timestep=SETTINGS["timestep"], gravity=SETTINGS["gravity"], floorStiffness=0.0, parityMode=True,
                 iterations=SETTINGS["iterations"])
    gpu = solver.JGS2GpuSolver.create(inp, camel)
    cpu = O.OracleSolver(inp, SETTINGS, precision=32)
    try:
        # The first second against the f32 oracle (the reference's sentinel
        # depth), then the whole 4 s on the GPU alone.
        gpu.stepFrames(120)
        cpu.step_frames(120)
        diag = inp.bbox_diagonal()
        g = gpu.readPositions().reshape(-1, 4)[:, :3]
        c = cpu.read("positions").reshape(-1, 4)[:, :3]
        err = float(np.abs(g - c).max()) / diag
        assert err <= POSITION_TOL, f"position error after 120 frames {err:.3e} of bbox diagonal"
        for _ in range((FRAMES - 120) // 120):
            gpu.stepFrames(120)
        linear, angular = _momentum_errors(inp, mass, gpu.readPositions(), gpu.readVelocities())
    finally:
        gpu.destroy()
    print(f"GPU, {FRAMES} frames: linear {linear:.3e}, angular {angular:.3e}; 120-frame position error {err:.2e}")
    assert linear < MOMENTUM_TOL and angular < MOMENTUM_TOL


# ---- the frozen force-free corpus (P0-CORPUS-01, jgs2.spec.ts:589-686) ----
CORPUS_SEED = 104729  # canonical-phase0.ts:26
SENTINELS = (0, 27)  # the quick run's 120-frame cases (jgs2.spec.ts:44)


def _corpus():
    """generatePhase0ForceFreeInitialStateCorpus (canonical-phase0.ts:60-101):
    32 cases, each a linear then an angular velocity; a velocity is a unit
    direction (components uniform in [-1, 1), rejected when shorter than
    1e-8, then normalised) times a speed uniform in [0.1, 1)."""
    rand = scenes.mulberry32(CORPUS_SEED)

    def unit():
        while True:
            c = [rand() * 2 - 1 for _ in range(3)]
            n = math.hypot(*c)
            if 1e-8 < n <= math.sqrt(3):
                return [x / n for x in c]

    def velocity():
        d = unit()
        speed = 0.1 + 0.9 * rand()
        return [x * speed for x in d]

    cases = []
    for _ in range(32):
        linear = velocity()
        angular = velocity()
        cases.append((linear, angular))
    return cases


def _min_tet_determinant(inp, positions):
    x = positions.reshape(-1, 4)[:, :3].astype(np.float64)
    t = inp.tet_indices.reshape(-1, 4)
    e = np.stack([x[t[:, 1]] - x[t[:, 0]], x[t[:, 2]] - x[t[:, 0]], x[t[:, 3]] - x[t[:, 0]]], axis=-1)
    return float(np.linalg.det(e).min())


def test_corpus_generator_matches_frozen_vectors():
    # The reference's frozen cases 00 and 31 (src/scenes/scenes.test.ts:251-275).
    cases = _corpus()
    np.testing.assert_allclose(cases[0][0], [-0.45846957506529673, 0.33551068797554123, -0.3184711985400522],
                               rtol=1e-14)
    np.testing.assert_allclose(cases[0][1], [-0.9724775707987993, 0.21396913055014707, 0.05338255748009366],
                               rtol=1e-14)
    np.testing.assert_allclose(cases[31][0], [-0.1613361445196155, -0.5490207886538739, -0.4162380237814731],
                               rtol=1e-14)
    np.testing.assert_allclose(cases[31][1], [-0.2369681366893712, -0.3062079393113022, -0.32347516329834597],
                               rtol=1e-14)
    for linear, angular in cases:
        assert 0.1 <= math.hypot(*linear) <= 1.0 and 0.1 <= math.hypot(*angular) <= 1.0


def _corpus_frames(i):
    return 120 if i in SENTINELS else 1


def _check_case(i, inp, mass, positions, velocities):
    assert np.isfinite(positions).all() and np.isfinite(velocities).all(), f"case {i} not finite"
    det = _min_tet_determinant(inp, positions)
    assert det > 0.0, f"case {i} inverted (min det {det:.3e})"
    linear, angular = _momentum_errors(inp, mass, positions, velocities)
    assert linear <= MOMENTUM_TOL and angular <= MOMENTUM_TOL, f"case {i}: linear {linear:.3e}, angular {angular:.3e}"
    return linear, angular


def test_oracle_corpus_conserves_momentum():
    worst = [0.0, 0.0]
    for i, (linear, angular) in enumerate(_corpus()):
        inp, mass = _force_free_cuboid(linear, angular)
        cpu = O.OracleSolver(inp, SETTINGS, precision=32)
        cpu.step_frames(_corpus_frames(i))
        errs = _check_case(i, inp, mass, cpu.read("positions"), cpu.read("velocities"))
        worst = [max(worst[0], errs[0]), max(worst[1], errs[1])]
    print(f"oracle corpus: worst linear {worst[0]:.3e}, worst angular {worst[1]:.3e}")


@pytest.mark.gpu
def test_gpu_corpus_conserves_momentum():
    camel = dict(timestep=SETTINGS["timestep"], gravity=SETTINGS["gravity"], floorStiffness=0.0, parityMode=True,
                 iterations=SETTINGS["iterations"])
    worst = [0.0, 0.0, 0.0]
    for i, (linear, angular) in enumerate(_corpus()):
        inp, mass = _force_free_cuboid(linear, angular)
        gpu = solver.JGS2GpuSolver.create(inp, camel)
        try:
            gpu.stepFrames(_corpus_frames(i))
            g, gv = gpu.readPositions(), gpu.readVelocities()
        finally:
            gpu.destroy()
        errs = _check_case(i, inp, mass, g, gv)
        cpu = O.OracleSolver(inp, SETTINGS, precision=32)
        cpu.step_frames(_corpus_frames(i))
        err = float(np.abs(g.reshape(-1, 4)[:, :3] - cpu.read("positions").reshape(-1, 4)[:, :3]).max())
        err /= inp.bbox_diagonal()
        assert err <= POSITION_TOL, f"case {i}: position error {err:.3e} of bbox diagonal"
        worst = [max(worst[0], errs[0]), max(worst[1], errs[1]), max(worst[2], err)]
    print(f"GPU corpus: worst linear {worst[0]:.3e}, worst angular {worst[1]:.3e}, "
          f"worst position error vs f32 oracle {worst[2]:.2e}")


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_keeps_a_translated_rigid_pose_that_is_its_own_target(precision):
    # nonlinear-oracle.test.ts:128-155: the rest shape rotated and moved
    # rigidly, at rest, with no gravity, is its own inertial target and has
    # no elastic force, so a frame leaves it where it is.
    sc, mass, pos = _fixture()
    moved = pos.copy()
    moved[:, :3] += np.array([3.0, -1.5, 0.75], dtype=np.float32)
    sc.set_initial_state(moved.reshape(-1), np.zeros_like(moved).reshape(-1), pin_at_initial=False)
    inp = sc.pack()
    cpu = O.OracleSolver(inp, SETTINGS, precision=precision)
    cpu.step_frames(2)
    err = float(np.abs(cpu.read("positions").reshape(-1, 4)[:, :3] - moved[:, :3]).max()) / inp.bbox_diagonal()
    vel = float(np.abs(cpu.read("velocities")).max())
    print(f"oracle f{precision}: rigid pose moved by {err:.2e} of the diagonal, speed {vel:.2e}")
    assert err < (1e-6 if precision == 32 else 1e-12)
    assert vel < (1e-4 if precision == 32 else 1e-10)

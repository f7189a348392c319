"""External forces are the paper predictor's constant force
(src/simulation/cpu/nonlinear-objective.test.ts:120-177): a force
f = m a on every free vertex, without gravity, steps like gravity a without
forces. The inertial target of the second run moves by h^2 a. The first run
adds -f to the gradient of every vertex and, through the complement
records, of its neighbours; the two gradients are the same, and the two
energies differ by a constant that the line search's differences cancel.
A released target (zero stiffness) is exactly an absent objective."""
import numpy as np
import pytest

from jgs2_b200 import scenes
from oracle import oracle as O

ACCEL = (0.3, -2.0, 0.5)


def _bar(k=None):
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((6, 2, 2), (0.0, 0.0, 0.0), (0.3, 0.1, 0.1), m, 0, scenes.FACE_X_MIN)
    if k is None:
        sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    else:
        sc.precompute(timestep=1 / 60, cubature_k=k)
    return sc.pack()


@pytest.mark.parametrize("k", [None, 6], ids=["exact-complement", "trained-k6"])
@pytest.mark.parametrize("precision,tol", [(64, 1e-9), (32, 2e-5)])
def test_constant_force_equals_predictor_gravity(k, precision, tol):
    inp = _bar(k)
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3]
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    forced = inp.copy()
    f = np.zeros((inp.vertex_count, 3), dtype=np.float32)
    f[~pinned] = mass[~pinned, None] * np.array(ACCEL, dtype=np.float32)
    forced.external_forces = f.reshape(-1)
    base = dict(timestep=1 / 60, floor_stiffness=0.0, parity_mode=1, iterations=8)
    a = O.OracleSolver(forced, dict(base, gravity=(0.0, 0.0, 0.0)), precision=precision)
    b = O.OracleSolver(inp, dict(base, gravity=ACCEL), precision=precision)
    for _ in range(3):
        a.step_exact_iterations(8)
        b.step_exact_iterations(8)
    pa = a.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    pb = b.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    moved = float(np.abs(pb - inp.positions.reshape(-1, 4)[:, :3]).max())
    err = float(np.abs(pa - pb).max()) / inp.bbox_diagonal()
    print(f"f{precision} {k}: forced vs predictor gravity {err:.2e} of the diagonal (moved {moved:.3e})")
    assert moved > 1e-4
    assert err < tol
    ha, hb = a.read("history").reshape(64, 32), b.read("history").reshape(64, 32)
    # Same accept / revert decisions in every iteration.
    np.testing.assert_array_equal(ha[:8, 4:6], hb[:8, 4:6])


@pytest.mark.parametrize("precision", [64, 32])
def test_released_target_is_exactly_an_absent_objective(precision):
    # nonlinear-restricted-energy.test.ts:421-456: target positions with zero
    # stiffness change nothing, bit for bit.
    inp = _bar(6)
    released = inp.copy()
    released.target_positions = (inp.positions.reshape(-1, 4)[:, :3] + 0.05).astype(np.float32).reshape(-1)
    released.target_stiffnesses = np.zeros(inp.vertex_count, dtype=np.float32)
    settings = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=8)
    a = O.OracleSolver(released, settings, precision=precision)
    b = O.OracleSolver(inp, settings, precision=precision)
    for _ in range(3):
        a.step_exact_iterations(8)
        b.step_exact_iterations(8)
    for what in ("positions", "velocities", "history"):
        np.testing.assert_array_equal(a.read(what), b.read(what))


def _minimal_target(frame):
    """minimalScriptedTargetAtFrame (src/scenes/index.ts:252-328): waiting
    before frame 48, keyframed smoothstep pull to frame 90, holding, and a
    zero-stiffness release from frame 108; (position, stiffness)."""
    rest, offset = np.array([1.0, 1.35, -0.4]), np.array([0.45, 0.65, 0.25])
    if frame < 48:
        return rest, 0.0
    key = min(90, 48 + ((min(frame, 90) - 48) // 3) * 3)
    u = (key - 48) / (90 - 48)
    return rest + offset * (u * u * (3 - 2 * u)), (0.0 if frame >= 108 else 30000.0)


def test_minimal_demo_pulls_holds_and_releases():
    # nonlinear-solid-demo.spec.ts:45-160 on the oracle: the minimal
    # cantilever with the steady 250 N demo force on its tip (index.ts:
    # 1069-1075), the scripted target and the app's production settings.
    from test_gpu_configs import MINIMAL_SETTINGS, _minimal_scene

    inp = _minimal_scene()
    V = inp.vertex_count
    forces = np.zeros(3 * V, dtype=np.float32)
    forces[3:6] = (250.0, 0.0, 0.0)
    targets = inp.positions.reshape(-1, 4)[:, :3].astype(np.float32).copy()
    stiff = np.zeros(V, dtype=np.float32)
    inp.external_forces, inp.target_positions, inp.target_stiffnesses = forces, targets.reshape(-1), stiff
    o = O.OracleSolver(inp, MINIMAL_SETTINGS, precision=64)
    tip = lambda: o.read("positions").reshape(-1, 4)[1, :3].astype(np.float64)  # noqa: E731
    start, marks = tip(), {}
    for frame in range(126):
        targets[1], stiff[1] = _minimal_target(frame)
        o.set_objectives(forces, targets.reshape(-1), stiff)
        o.step()
        if frame + 1 in (47, 107, 108, 126):
            marks[frame + 1] = (tip(), int(o.read("control")[7]), o.read("velocities").copy())
    assert start[1] - marks[47][0][1] > 0.01  # sags before the pull
    assert np.linalg.norm(_minimal_target(107)[0] - _minimal_target(0)[0]) > 0.5
    assert np.linalg.norm(marks[107][0] - start) > 0.05
    assert marks[107][1] < 7  # the settled hold trips the convergence latch
    assert np.linalg.norm(marks[108][0] - marks[107][0]) < 0.35  # no teleport on release
    assert np.abs(marks[108][2]).max() > 1e-5
    assert all(np.isfinite(m[0]).all() for m in marks.values())


@pytest.mark.parametrize("precision", [64, 32])
def test_oracle_schedules_agree_on_the_minimal_scene(precision):
    # colored-schedule.spec.ts:56-137 on the oracle: 12 production frames of
    # Jacobi and of graph-coloured GGS2 from the same start differ by less
    # than 5e-4 RMS and 1e-3 max of the scene scale. The reference's
    # roadmap reports an RMS of 1.97e-5 (docs/ROADMAP.md:236-240).
    from test_gpu_configs import MINIMAL_SETTINGS, _minimal_scene

    from test_oracle_diagnostics import _reference

    inp = _minimal_scene()
    V = inp.vertex_count
    ends, energies = {}, {}
    for schedule in (0, 1):
        o = O.OracleSolver(inp, dict(MINIMAL_SETTINGS, schedule=schedule), precision=precision)
        if schedule == 1:
            assert o.color_count > 1
        o.step_frames(12)
        ends[schedule] = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
        pred = o.read("predicted").reshape(-1, 4)[:, :3].astype(np.float64)
        e = _reference(inp, ends[schedule], pred, MINIMAL_SETTINGS["timestep"], np.zeros((V, 3)), np.zeros((V, 4)),
                       MINIMAL_SETTINGS["floor_height"], MINIMAL_SETTINGS["floor_stiffness"])[0]
        energies[schedule] = (e["elasticity"], sum(e.values()))
    scale = inp.bbox_diagonal()
    diff = ends[0] - ends[1]
    rms = float(np.sqrt((diff ** 2).sum(axis=1).mean())) / scale
    print(f"oracle f{precision}: Jacobi vs GGS2 RMS {rms:.4e} of the scene scale")
    assert rms < 5e-4
    assert float(np.linalg.norm(diff, axis=1).max()) / scale < 1e-3
    # The published 1.97e-5 (f32 hardware): the FP64 run reproduces its three
    # digits (1.9715e-5), the f32 mirror lands within 10 % (1.858e-5).
    if precision == 64:
        assert abs(rms - 1.97e-5) < 0.005e-5
        # The exact material and implicit energies of the two end poses
        # (the float64 restatement of readOracleDiagnostics) differ by
        # 1.76e-4 and 1.73e-4 relative; the roadmap reports 1.96e-4 and 1.87e-4.
        material = abs(energies[0][0] - energies[1][0]) / abs(energies[0][0])
        implicit = abs(energies[0][1] - energies[1][1]) / abs(energies[0][1])
        assert abs(material / 1.96e-4 - 1) < 0.2 and abs(implicit / 1.87e-4 - 1) < 0.2
    else:
        assert abs(rms / 1.97e-5 - 1) < 0.1

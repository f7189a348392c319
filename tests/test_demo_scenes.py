"""The reference's deterministic demo scenes (tests/e2e/jgs2.spec.ts:
688-790, cases :178-207), stepped on the oracle with the app's production
settings (src/App.tsx:520-575):
- minimal: the public cantilever with its steady 250 N tip force, 45 frames;
- drop: a rotated block falling onto the floor, 90 frames;
- stiffness: a soft and a stiff cantilever side by side, 60 frames;
- stress: six rotated soft and stiff blocks falling in separate lanes, 60
  frames.

Each run must move the landmark down by the case's fraction of the initial
bounding-box diagonal, but by less than two diagonals. The bounds must move,
every tet must keep at least 1 % of the initial minimum determinant, and the
drop and stress blocks must not pass more than 0.12 m through the floor.

The long-run settle bounds (jgs2.spec.ts:793-915, 20 s) run for the drop
and for every body of the stress scene."""
import numpy as np
import pytest

from jgs2_b200 import scenes
from oracle import oracle as O

from test_gpu_configs import MINIMAL_SETTINGS, _minimal_scene


def _drop_scene():
    """dropDefinition (src/scenes/index.ts:412-453): one 1.5 x 1 x 0.9 m hex
    rotated 0.12 rad about y and lifted to y = 2.45, 900 kg/m^3, E 70 000,
    nu 0.36, h = 1/60, six cubature samples."""
    sc = scenes.Scene()
    m = sc.add_material(900.0, 70000.0, 0.36)
    sc.add_cuboid((1, 1, 1), (-0.75, -0.5, -0.45), (1.5, 1.0, 0.9), m, 0, 0)
    rest = scenes.rotate_euler_xyz(sc.rest_positions(), 0.0, 0.12, 0.0) + np.array([0.0, 2.45, 0.0])
    sc.set_rest_positions(rest)
    sc.precompute(timestep=1 / 60, cubature_k=6)
    return sc.pack()


def _stiffness_scene():
    """stiffnessDefinition (src/scenes/index.ts:366-411): a soft (850 kg/m^3,
    E 35 000, nu 0.35) and a stiff (950 kg/m^3, E 280 000, nu 0.32) one-hex
    cantilever of 2 x 0.7 x 0.7 m side by side, x = min faces pinned,
    h = 1/30, six cubature samples.  The reference's soft and stiff
    materials name no model, so they are co-rotated linear and train the
    linear cubature (src/simulation/cpu/precompute.ts:250-261)."""
    sc = scenes.Scene()
    soft = sc.add_material(850.0, 35000.0, 0.35, scenes.MATERIAL_COROTATED_LINEAR)
    stiff = sc.add_material(950.0, 280000.0, 0.32, scenes.MATERIAL_COROTATED_LINEAR)
    sc.add_cuboid((1, 1, 1), (-1.0, 1.35, -1.05), (2.0, 0.7, 0.7), soft, 0, scenes.FACE_X_MIN)
    sc.add_cuboid((1, 1, 1), (-1.0, 1.35, 0.35), (2.0, 0.7, 0.7), stiff, 1, scenes.FACE_X_MIN)
    sc.precompute(timestep=1 / 30, cubature_k=6)
    return sc.pack()


def _stress_scene():
    """stressDefinition (src/scenes/index.ts:719-771): six 2 x 1 x 1-hex
    blocks of 1.2 x 0.64 x 0.64 m, alternating soft and stiff, each rotated
    by (0.04 b, 0.08 (b - 2), 0.1 (b mod 2)) and moved to its lane,
    h = 1/120, six cubature samples; co-rotated linear like the stiffness
    scene."""
    sc = scenes.Scene()
    mats = (sc.add_material(850.0, 35000.0, 0.35, scenes.MATERIAL_COROTATED_LINEAR),
            sc.add_material(950.0, 280000.0, 0.32, scenes.MATERIAL_COROTATED_LINEAR))
    starts = [sc.add_cuboid((2, 1, 1), (-0.6, -0.32, -0.32), (1.2, 0.64, 0.64), mats[b % 2], b, 0) for b in range(6)]
    rest = sc.rest_positions().copy()
    ends = starts[1:] + [rest.shape[0]]
    for b, (lo, hi) in enumerate(zip(starts, ends)):
        moved = scenes.rotate_euler_xyz(rest[lo:hi], 0.04 * b, 0.08 * (b - 2), 0.1 * (b % 2))
        rest[lo:hi] = moved + np.array([(b % 3 - 1) * 1.45, 1.25 + 0.08 * (b % 2), (b // 3 - 0.5) * 1.25])
    sc.set_rest_positions(rest)
    sc.precompute(timestep=1 / 120, cubature_k=6)
    return sc.pack()


def _minimal_with_force():
    inp = _minimal_scene()
    forces = np.zeros(3 * inp.vertex_count, dtype=np.float32)
    forces[3:6] = (250.0, 0.0, 0.0)  # MINIMAL_EXTERNAL_FORCE on vertex 1 (index.ts:1069-1075)
    inp.external_forces = forces
    return inp


CASES = {
    "minimal": (_minimal_with_force, dict(MINIMAL_SETTINGS), 45, 1, 0.003, 0.001),
    "drop": (_drop_scene, dict(MINIMAL_SETTINGS, timestep=1 / 60, iterations=11), 90, 0, 0.05, 0.025),
    "stiffness": (_stiffness_scene, dict(MINIMAL_SETTINGS, iterations=9), 60, 1, 0.006, 0.003),
    "stress": (_stress_scene, dict(MINIMAL_SETTINGS, timestep=1 / 120, iterations=17), 60, 0, 0.003, 0.001),
}


def _min_det(inp, x):
    t = inp.tet_indices.reshape(-1, 4)
    e = np.stack([x[t[:, k]] - x[t[:, 0]] for k in (1, 2, 3)], axis=-1)
    return float(np.linalg.det(e).min())


@pytest.mark.parametrize("name", list(CASES))
def test_demo_scene_moves_deforms_and_stays_feasible(name):
    build, settings, frames, landmark, min_drop, min_bounds = CASES[name]
    inp = build()
    o = O.OracleSolver(inp, settings, precision=64)
    x0 = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    o.step_frames(frames)
    x1 = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    diag = float(np.linalg.norm(x0.max(0) - x0.min(0)))
    drop = (x0[landmark, 1] - x1[landmark, 1]) / diag
    moved = float(np.linalg.norm(x1[landmark] - x0[landmark])) / diag
    bounds = float(max(np.abs(x1.min(0) - x0.min(0)).max(), np.abs(x1.max(0) - x0.max(0)).max())) / diag
    print(f"{name}: landmark drop {drop:.4f}, bounds motion {bounds:.4f} of the diagonal")
    assert drop > min_drop
    assert moved < 2
    assert bounds > min_bounds
    assert _min_det(inp, x1) / _min_det(inp, x0) > 0.01
    if name in ("drop", "stress"):
        assert x1[:, 1].min() >= settings["floor_height"] - 0.12
    if name == "stiffness":
        # jgs2.spec.ts:1398-1435: the stiff tip (landmark + V/2) responds, the
        # soft tip deflects at least 1.5x as far, and the two differ by more
        # than 3 % of the diagonal.
        stiff_tip = landmark + inp.vertex_count // 2
        soft = x0[landmark, 1] - x1[landmark, 1]
        stiff = x0[stiff_tip, 1] - x1[stiff_tip, 1]
        print(f"stiffness: soft tip {soft:.4f} m, stiff tip {stiff:.4f} m")
        assert stiff > 0 and soft > 1.5 * stiff and (soft - stiff) / diag > 0.03


def _body_states(o, inp):
    """Per body: mass centre, mass-weighted velocity and lowest y."""
    x = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    v = o.read("velocities").reshape(-1, 4)[:, :3].astype(np.float64)
    m = inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    body = inp.vertex_info.reshape(-1, 4)[:, 3]
    out = {}
    for b in np.unique(body):
        sel = body == b
        w = m[sel][:, None]
        out[int(b)] = ((w * x[sel]).sum(0) / w.sum(), (w * v[sel]).sum(0) / w.sum(), float(x[sel, 1].min()))
    return out


LONG_RUNS = {
    "drop": (_drop_scene, dict(MINIMAL_SETTINGS, timestep=1 / 60, iterations=11)),
    "stress": (_stress_scene, dict(MINIMAL_SETTINGS, timestep=1 / 120, iterations=17)),
}


@pytest.mark.parametrize("name", list(LONG_RUNS))
def test_long_run_bodies_settle(name):
    # jgs2.spec.ts:793-915, per body: at 1 s it has reached the floor; at 4 s
    # it is still in contact and vertically settled; over 20 s it stays in
    # its lane, drifts less than 5 cm after settling, and its tangential
    # speed decays below 1 cm/s.
    build, settings = LONG_RUNS[name]
    inp = build()
    o = O.OracleSolver(inp, settings, precision=64)
    h, floor = settings["timestep"], settings["floor_height"]
    x0 = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    start, marks, done = _body_states(o, inp), {}, 0
    for sec in (1, 4, 20):
        n = int(round(sec / h)) - done
        o.step_frames(n)
        done += n
        marks[sec] = _body_states(o, inp)
    hspeed = lambda v: float(np.hypot(v[0], v[2]))  # noqa: E731
    drift = lambda a, b: float(np.hypot(*(a - b)[[0, 2]]))  # noqa: E731
    for b in start:
        (c1, v1, y1), (c4, v4, y4), (c20, v20, y20) = marks[1][b], marks[4][b], marks[20][b]
        print(f"{name} body {b}: drift {drift(c20, start[b][0]):.4f} / {drift(c20, c4):.4f} m, "
              f"tangential speed {hspeed(v1):.4f} -> {hspeed(v4):.4f} -> {hspeed(v20):.4f} m/s")
        assert y1 <= floor + 0.05 and y4 <= floor + 0.05 and y20 >= floor - 0.12
        assert drift(c20, start[b][0]) <= 0.5 and drift(c20, c4) <= 0.05
        assert hspeed(v4) <= hspeed(v1) + 0.01 and hspeed(v20) <= hspeed(v4) + 0.005
        assert hspeed(v20) <= 0.5 * hspeed(v1) + 0.005 and hspeed(v20) <= 0.01
        assert abs(v4[1]) < 0.1 and abs(v20[1]) < 0.05
    x20 = o.read("positions").reshape(-1, 4)[:, :3].astype(np.float64)
    assert _min_det(inp, x20) / _min_det(inp, x0) > 0.01

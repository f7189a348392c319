"""Vertex frames as polar averages of deformation gradients, the reference's
P1-FRAME-01 (tests/e2e/stable-neo-hookean-gpu-oracle.spec.ts:544-758).

The fixture:
- a 2x2x2-hex cuboid at centimetre scale: origin (-0.8, -0.5, -0.65) cm,
  size (1.6, 1.1, 1.3) cm;
- stable Neo-Hookean, density 1000, E 8e4, nu 0.3
  (src/scenes/phase1.ts:44-51);
- deformed by the non-affine map (x + 0.25 y z, y - 0.15 x^2, z + 0.18 x y)
  in units of the scale, rounded to f32.

After one exact iteration the step's frames are those of its source pose.
Each must match the polar factor of the vertex's volume-weighted average
deformation gradient over its incident tetrahedra, sum(vol F) / sum(vol)
(src/simulation/cpu/deformation-gradient.ts:22-177), within the reference's
relative error 1e-4. The expected frames are computed independently here in
float64, with the polar factor from an SVD.
"""
import math

import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

SCALE = 1e-2
FRAME_TOL = 1e-4
SETTINGS = dict(timestep=1 / 60, gravity=(0.0, 0.0, 0.0), iterations=1, floor_height=-100.0, floor_stiffness=0.0,
                max_step=0.01 * SCALE, parity_mode=1)


def _fixture():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 8.0e4, 0.3)
    sc.add_cuboid((2, 2, 2), (-0.8 * SCALE, -0.5 * SCALE, -0.65 * SCALE), (1.6 * SCALE, 1.1 * SCALE, 1.3 * SCALE),
                  m, 0, 0)
    sc.precompute(timestep=SETTINGS["timestep"], cubature_k=sc.tet_count, exact_complement=1)
    rest = sc.rest_positions().astype(np.float64)
    n = rest / SCALE
    pose = np.stack([SCALE * (n[:, 0] + 0.25 * n[:, 1] * n[:, 2]),
                     SCALE * (n[:, 1] - 0.15 * n[:, 0] * n[:, 0]),
                     SCALE * (n[:, 2] + 0.18 * n[:, 0] * n[:, 1])], axis=1).astype(np.float32)
    p4 = np.ones((pose.shape[0], 4), dtype=np.float32)
    p4[:, :3] = pose
    sc.set_initial_state(p4.reshape(-1), None, pin_at_initial=False)
    inp = sc.pack()
    return inp, rest, pose.astype(np.float64)


def _expected_frames(inp, rest, pose):
    tets = inp.tet_indices.reshape(-1, 4).astype(np.int64)
    dm = np.stack([rest[tets[:, k]] - rest[tets[:, 0]] for k in (1, 2, 3)], axis=-1)
    ds = np.stack([pose[tets[:, k]] - pose[tets[:, 0]] for k in (1, 2, 3)], axis=-1)
    f = ds @ np.linalg.inv(dm)
    vol = np.abs(np.linalg.det(dm)) / 6.0
    acc = np.zeros((rest.shape[0], 3, 3))
    tot = np.zeros(rest.shape[0])
    for k in range(4):
        np.add.at(acc, tets[:, k], vol[:, None, None] * f)
        np.add.at(tot, tets[:, k], vol)
    fv = acc / tot[:, None, None]
    u, _, vt = np.linalg.svd(fv)
    return u @ vt  # det F_v > 0 here, so U V^T is the rotation


def _frames(packed):
    # Three padded columns per vertex.
    c = packed.reshape(-1, 3, 4)[:, :, :3]
    return np.transpose(c, (0, 2, 1)).astype(np.float64)


def _max_relative_error(got, want):
    d = np.linalg.norm((got - want).reshape(len(got), 9), axis=1)
    den = np.maximum(1.0, np.maximum(np.linalg.norm(got.reshape(len(got), 9), axis=1),
                                     np.linalg.norm(want.reshape(len(want), 9), axis=1)))
    return float((d / den).max())


def test_expected_frames_are_rotations():
    inp, rest, pose = _fixture()
    r = _expected_frames(inp, rest, pose)
    np.testing.assert_allclose(r @ np.transpose(r, (0, 2, 1)), np.broadcast_to(np.eye(3), r.shape), atol=1e-12)
    assert (np.linalg.det(r) > 0).all()
    # The deformation is far from affine: the frames differ from vertex to vertex.
    assert float(np.abs(r - r[0]).max()) > 1e-2


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_frames_are_polar_averages(precision):
    inp, rest, pose = _fixture()
    cpu = O.OracleSolver(inp, SETTINGS, precision=precision)
    cpu.step_exact_iterations(1)
    err = _max_relative_error(_frames(cpu.read("vertex_rotations")), _expected_frames(inp, rest, pose))
    print(f"oracle f{precision} vertex frames: max relative error {err:.2e}")
    # FP64: the input's rest data are f32 and the step runs a fixed number of
    # polar iterations, so the FP64 run sits near 1e-8 rather than at rounding.
    assert err <= (FRAME_TOL if precision == 32 else 1e-6)
    assert np.isfinite(cpu.read("positions")).all()


@pytest.mark.gpu
def test_gpu_frames_are_polar_averages():
    inp, rest, pose = _fixture()
    camel = dict(timestep=SETTINGS["timestep"], gravity=SETTINGS["gravity"], iterations=1, floorHeight=-100.0,
                 floorStiffness=0.0, maxStep=0.01 * SCALE, parityMode=True)
    gpu = solver.JGS2GpuSolver.create(inp, camel)
    try:
        gpu.stepExactIterations(1)
        frames = _frames(gpu.readVertexRotations())
        positions = gpu.readPositions()
    finally:
        gpu.destroy()
    err = _max_relative_error(frames, _expected_frames(inp, rest, pose))
    cpu = O.OracleSolver(inp, SETTINGS, precision=32)
    cpu.step_exact_iterations(1)
    err_oracle = _max_relative_error(frames, _frames(cpu.read("vertex_rotations")))
    print(f"GPU vertex frames: max relative error {err:.2e} (vs the f32 oracle {err_oracle:.2e})")
    assert err <= FRAME_TOL
    assert np.isfinite(positions).all()
    # The solved pose stays uninverted (the reference's solved min J > 0).
    x = positions.reshape(-1, 4)[:, :3].astype(np.float64)
    tets = inp.tet_indices.reshape(-1, 4).astype(np.int64)
    ds = np.stack([x[tets[:, k]] - x[tets[:, 0]] for k in (1, 2, 3)], axis=-1)
    assert float(np.linalg.det(ds).min()) > 0.0


def _posed(transform, translation):
    inp, rest, _ = _fixture()
    pose = (rest @ np.asarray(transform).T + np.asarray(translation)).astype(np.float32)
    p4 = np.ones((pose.shape[0], 4), dtype=np.float32)
    p4[:, :3] = pose
    out = inp.copy()
    out.positions = p4.reshape(-1)
    return out


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_frames_of_affine_and_rigid_poses(precision):
    # deformation-gradient.test.ts:89-131: an affine pose A X + b gives every
    # vertex, boundary or interior, the polar factor of A; a rigid motion
    # R X + t gives R.
    A = np.array([[1.1, 0.2, -0.05], [-0.1, 0.9, 0.15], [0.08, -0.12, 1.05]])
    u, _, vt = np.linalg.svd(A)
    a = 0.7
    R = np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])
    # The poses and rest data reach the step as f32, which bounds the FP64 run too.
    tol = 1e-5 if precision == 32 else 1e-6
    for transform, want in ((A, u @ vt), (R, R)):
        inp = _posed(transform, (0.01, -0.02, 0.005))
        cpu = O.OracleSolver(inp, SETTINGS, precision=precision)
        cpu.step_exact_iterations(1)
        frames = _frames(cpu.read("vertex_rotations"))
        err = _max_relative_error(frames, np.broadcast_to(want, frames.shape))
        assert err <= tol, f"f{precision}: {err:.2e}"

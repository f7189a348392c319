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

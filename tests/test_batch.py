"""The batched form: independent scenes stepped together must give, scene by
scene, exactly what each scene gives alone.

Per-scene reductions fold the same chunks in the same order alone and in a
batch, and every per-vertex computation is the same, so results are compared
bitwise (body correction, whose double atomics have a run-dependent order,
is off).
"""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver

SETTINGS = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), floorStiffness=2.0e4, parityMode=True, iterations=10)


@pytest.fixture(scope="module")
def bodies():
    return scenes.batched_bodies(count=5, min_cells=2, max_cells=5, seed=4242)


@pytest.fixture(scope="module")
def split(bodies):
    return bodies.split_bodies()


def test_split_bodies_gives_valid_scenes(bodies, split):
    assert len(split) == 5
    assert sum(s.vertex_count for s in split) == bodies.vertex_count
    assert sum(s.tet_count for s in split) == bodies.tet_count
    for s in split:
        solver.validate_input(s)
        info = s.vertex_info.reshape(-1, 4)
        assert (info[:, 3] == 0).all()
        assert int(info[:, 0][-1] + info[:, 1][-1]) == s.adjacency.size


def test_split_bodies_keeps_records(bodies, split):
    K = bodies.cubature_k
    v0 = 0
    for s in split:
        np.testing.assert_array_equal(s.cubature_weights, bodies.cubature_weights[v0 * K:(v0 + s.vertex_count) * K])
        np.testing.assert_array_equal(s.positions, bodies.positions[4 * v0:4 * (v0 + s.vertex_count)])
        v0 += s.vertex_count


@pytest.mark.gpu
def test_batch_matches_scenes_alone_exact_iterations(split):
    batch = solver.JGS2Batch.create(split, SETTINGS)
    alone = [solver.JGS2GpuSolver.create(s, SETTINGS) for s in split]
    for _ in range(3):
        batch.stepFrames(2, exactIterations=6)
        for a in alone:
            a.stepFramesExactIterations(2, 6)
    for i, a in enumerate(alone):
        np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(), err_msg=f"scene {i}")
        np.testing.assert_array_equal(batch.readVelocities(i), a.readVelocities(), err_msg=f"scene {i}")
        db, da = batch.readGlobalizationDiagnostics(i), a.readGlobalizationDiagnostics()
        assert db["historyCount"] == da["historyCount"] == 6
        np.testing.assert_array_equal(db["history"], da["history"], err_msg=f"scene {i}")
        np.testing.assert_array_equal(db["local"], da["local"], err_msg=f"scene {i}")
        a.destroy()
    batch.destroy()


@pytest.mark.gpu
def test_batch_production_latch_is_per_scene(split):
    # Scene 0 rests without gravity (converges and latches early); the others fall.
    per = [dict(SETTINGS, gravity=(0.0, 0.0, 0.0), floorStiffness=0.0) if i == 0 else dict(SETTINGS)
           for i in range(len(split))]
    rest = split[0].copy()
    # A soft material keeps the f32 rest residual far below the tolerance.
    meta = rest.tet_meta.reshape(-1, 4)
    meta[:, 1:3] *= 1e-3
    scenes_in = [rest] + split[1:]
    batch = solver.JGS2Batch.create(scenes_in, per)
    alone = [solver.JGS2GpuSolver.create(s, o) for s, o in zip(scenes_in, per)]
    batch.stepFrames(1)
    for a in alone:
        a.step()
    counts = []
    for i, a in enumerate(alone):
        db, da = batch.readGlobalizationDiagnostics(i), a.readGlobalizationDiagnostics()
        assert db["historyCount"] == da["historyCount"], f"scene {i}"
        counts.append(db["historyCount"])
        np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(), err_msg=f"scene {i}")
        a.destroy()
    assert counts[0] < max(counts[1:])  # the resting scene stopped first
    batch.destroy()


@pytest.mark.gpu
def test_batch_rejects_mixed_schedules(split):
    per = [dict(SETTINGS, schedule="graph-colored-gauss-seidel") if i == 1 else dict(SETTINGS)
           for i in range(len(split))]
    batch = solver.JGS2Batch.create(split, per)
    with pytest.raises(solver.JGS2RangeError):
        batch.stepFrames(1, exactIterations=2)
    batch.destroy()


@pytest.mark.gpu
def test_batch_graph_colored_matches_alone(split):
    opts = dict(SETTINGS, schedule="graph-colored-gauss-seidel")
    batch = solver.JGS2Batch.create(split, opts)
    alone = [solver.JGS2GpuSolver.create(s, opts) for s in split]
    batch.stepFrames(2, exactIterations=4)
    for a in alone:
        a.stepFramesExactIterations(2, 4)
    for i, a in enumerate(alone):
        np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(), err_msg=f"scene {i}")
        a.destroy()
    batch.destroy()

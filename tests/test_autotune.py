"""Launch-shape autotuner (include/jgs2.h: jgs2_autotune and friends).  The
shapes change how many vertices one block of the local-solve kernel takes,
never a vertex's arithmetic, so every shape and every tuning run must give
bit-identical states."""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver

FRAMES, ITERATIONS = 4, 10


def _run(inp, settings, shape=None, tune=0, frames=FRAMES):
    s = solver.JGS2GpuSolver.create(inp, settings)
    if shape is not None:
        s.setLaunchShape(shape)
    if tune:
        s.autotune(tune)
    s.stepFramesExactIterations(frames, ITERATIONS)
    out = (s.readPositions(), s.readVelocities(), s.launchShape())
    s.destroy()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["cube", "trough"])
def test_every_launch_shape_gives_identical_states(scene):
    if scene == "cube":
        inp, settings = scenes.unit_cube(cells=10), {"parityMode": True}
    else:
        inp, settings = scenes.trough(1), scenes.TROUGH_SETTINGS
    base = _run(inp, settings, shape=0)
    assert base[2]["shape"] == 0 and base[2]["solveVerticesPerBlock"] > 0
    for shape in (1, 2):
        pos, vel, info = _run(inp, settings, shape=shape)
        assert info["shape"] == shape
        assert info["solveVerticesPerBlock"] == max(1, base[2]["solveVerticesPerBlock"] >> shape)
        np.testing.assert_array_equal(pos, base[0], err_msg=f"shape {shape}")
        np.testing.assert_array_equal(vel, base[1], err_msg=f"shape {shape}")


@pytest.mark.gpu
def test_autotuning_times_every_shape_and_keeps_the_fastest():
    inp = scenes.unit_cube(cells=10)
    settings = {"parityMode": True}
    base = _run(inp, settings, shape=0, frames=8)
    pos, vel, info = _run(inp, settings, tune=2, frames=8)  # 6 tuned frames, 2 in the chosen shape
    np.testing.assert_array_equal(pos, base[0])
    np.testing.assert_array_equal(vel, base[1])
    assert info["tuning"] == 0 and info["samples"] == 2
    ms = info["frameMs"]
    assert all(m > 0 for m in ms)
    assert info["shape"] == int(np.argmin(ms))


@pytest.mark.gpu
def test_batch_autotuning_matches_an_untuned_batch():
    parts = [scenes.unit_cube(cells=4 + 2 * i) for i in range(3)]
    opts = {"parityMode": True}
    plain = solver.JGS2Batch.create(parts, opts)
    tuned = solver.JGS2Batch.create(parts, opts)
    tuned.autotune(1)
    plain.stepFrames(5, exactIterations=ITERATIONS)
    tuned.stepFrames(5, exactIterations=ITERATIONS)
    for i in range(3):
        np.testing.assert_array_equal(tuned.readPositions(i), plain.readPositions(i), err_msg=f"scene {i}")
    info = tuned.launchShape()
    assert info["tuning"] == 0 and info["samples"] == 1
    plain.destroy()
    tuned.destroy()


@pytest.mark.gpu
def test_launch_shape_arguments_are_checked():
    s = solver.JGS2GpuSolver.create(scenes.unit_cube(cells=3), {"parityMode": True})
    with pytest.raises(solver.JGS2RangeError, match="rounds must be 1-64"):
        s.autotune(0)
    with pytest.raises(solver.JGS2RangeError, match="Launch shape must be below 3"):
        s.setLaunchShape(3)
    s.autotune(1)
    s.setLaunchShape(1)  # a fixed shape ends tuning
    assert s.launchShape()["tuning"] == 0
    s.destroy()

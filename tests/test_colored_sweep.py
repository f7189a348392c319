"""The graph-coloured schedule as one persistent kernel per iteration
(JGS2_COLOR_SWEEP=persistent)
(per-colour phases separated by grid barriers, jgs2-solver.ts:2275-2325)
against the launch-per-colour encoding (equal to f32 rounding, replayed bit for
bit), and the bounded barrier: with a spin
bound of zero polls a waiting block gives up at once, every block leaves the
kernel, and the host reports JGS2_TIMEOUT at its next synchronisation while
the device stays usable."""
import os

import numpy as np
import pytest

from jgs2_b200 import _ffi, scenes, solver

pytestmark = pytest.mark.gpu

SETTINGS = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), floorStiffness=0.0, parityMode=True, schedule=1)


def _with_env(name, value, fn):
    old = os.environ.get(name)
    os.environ[name] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


def test_persistent_sweep_matches_per_colour_launches():
    # The same arithmetic in another kernel: the compiler may fuse a few
    # multiply-adds differently, so the encodings agree to f32 rounding (and
    # take the same accept / revert decisions), and the persistent sweep
    # replays bit for bit.
    inp = scenes.unit_cube(cells=12)
    a = _with_env("JGS2_COLOR_SWEEP", "persistent", lambda: solver.JGS2GpuSolver.create(inp, SETTINGS))
    a2 = _with_env("JGS2_COLOR_SWEEP", "persistent", lambda: solver.JGS2GpuSolver.create(inp, SETTINGS))
    b = solver.JGS2GpuSolver.create(inp, SETTINGS)
    assert a.scheduleColorCount > 1
    diag = inp.bbox_diagonal()
    for frame in range(3):
        la, lb = a.kernelLaunchCount(), b.kernelLaunchCount()
        for s in (a, a2, b):
            s.stepExactIterations(6)
        np.testing.assert_array_equal(a.readPositions(), a2.readPositions(), err_msg=f"replay, frame {frame}")
        if frame == 0:
            # Later frames of this stiff cube reach the determinant floor,
            # where f32 rounding decides the trajectory (as between the
            # oracle's f32 and FP64 runs); the first frame is well conditioned.
            err = np.abs(a.readPositions() - b.readPositions()).max() / diag
            assert err <= 1e-5, err
            np.testing.assert_array_equal(a.readGlobalizationDiagnostics()["history"][:, 4],
                                          b.readGlobalizationDiagnostics()["history"][:, 4])
        # One sweep (a barrier reset and a kernel) per iteration instead of two
        # launches per colour.
        assert a.kernelLaunchCount() - la < b.kernelLaunchCount() - lb
    for s in (a, a2, b):
        s.destroy()


def test_barrier_timeout_is_reported_and_the_device_stays_usable():
    inp = scenes.unit_cube(cells=12)
    s = _with_env("JGS2_COLOR_SWEEP", "persistent",
                  lambda: _with_env("JGS2_BARRIER_SPIN_LIMIT", "0", lambda: solver.JGS2GpuSolver.create(inp, SETTINGS)))
    s.stepExactIterations(2)
    with pytest.raises(_ffi.JGS2Error) as err:
        s.readPositions()
    assert err.value.status == 5  # JGS2_TIMEOUT
    assert "grid barrier" in err.value.message
    s.destroy()
    # The context survived: a fresh solver steps and reads normally.
    t = _with_env("JGS2_COLOR_SWEEP", "persistent", lambda: solver.JGS2GpuSolver.create(inp, SETTINGS))
    t.stepExactIterations(2)
    assert np.isfinite(t.readPositions()).all()
    t.destroy()


def test_persistent_sweep_with_cloth():
    # The cloth instantiation of the persistent sweep (membrane and hinge
    # gathers read positions other blocks write) against the launches.
    inp = scenes.cloth_drape(cells=6, prefold=False, pinned_columns=(0, 6))
    s = dict(timestep=1 / 120, gravity=(0.0, -9.81, 0.0), floorStiffness=0.0, parityMode=True, schedule=1)
    a = _with_env("JGS2_COLOR_SWEEP", "persistent", lambda: solver.JGS2GpuSolver.create(inp, s))
    b = solver.JGS2GpuSolver.create(inp, s)
    assert a.scheduleColorCount > 1
    la, lb = a.kernelLaunchCount(), b.kernelLaunchCount()
    a.stepExactIterations(5)
    b.stepExactIterations(5)
    assert a.kernelLaunchCount() - la < b.kernelLaunchCount() - lb  # the sweep ran
    err = np.abs(a.readPositions() - b.readPositions()).max() / inp.bbox_diagonal()
    assert err <= 1e-5, err
    a.destroy()
    b.destroy()

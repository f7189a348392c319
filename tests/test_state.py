"""Checkpoint / resume through the C-ABI (jgs2_export_state /
jgs2_import_state): a solver created from the same input and given an
exported image continues bit for bit as the exporting solver does, with
objectives, static IPC contact with lagged friction, and the device broad
phase."""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver

pytestmark = pytest.mark.gpu


def _replay(inp, settings, before, after, step, prepare=None):
    a = solver.JGS2GpuSolver.create(inp, settings)
    if prepare:
        prepare(a)
    for _ in range(before):
        step(a)
    image = a.exportState()
    for _ in range(after):
        step(a)
    b = solver.JGS2GpuSolver.create(inp, settings)
    b.importState(image)
    assert b.exportState() == image  # the restore is complete
    assert b.objectiveActivity == a.objectiveActivity
    for _ in range(after):
        step(b)
    np.testing.assert_array_equal(b.readPositions(), a.readPositions())
    np.testing.assert_array_equal(b.readVelocities(), a.readVelocities())
    np.testing.assert_array_equal(b.readGlobalizationDiagnostics()["history"],
                                  a.readGlobalizationDiagnostics()["history"])
    a.destroy()
    b.destroy()


def test_replay_with_objectives():
    inp = scenes.cantilever(cells=(10, 2, 2), size=(0.5, 0.1, 0.1))
    settings = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), iterations=9)

    def prepare(s):
        free = np.flatnonzero(inp.vertex_info.reshape(-1, 4)[:, 2] == 0)
        s.setExternalForce(int(free[-1]), (0.0, 2.0, 1.0))
        s.setQuadraticTarget(int(free[-3]), inp.rest_positions[free[-3]] + np.array([0.0, 0.03, 0.0]), 400.0)

    _replay(inp, settings, 6, 6, lambda s: s.step(), prepare)


def test_replay_with_static_contact_and_friction():
    _replay(scenes.trough(4), scenes.TROUGH_SETTINGS, 40, 12, lambda s: s.step())


def test_replay_with_the_broad_phase():
    inp = scenes.box_trough(boxes=3, cells=3, heights=(1.0, 1.3), plate_cells=(8, 2),
                            method=scenes.PRECOMPUTE_PATCH)
    _replay(inp, dict(scenes.BOX_TROUGH_SETTINGS), 30, 8, lambda s: s.stepExactIterations(15))


def test_import_refuses_another_solver_shape():
    a = solver.JGS2GpuSolver.create(scenes.cantilever(cells=(4, 1, 1), size=(0.4, 0.1, 0.1)),
                                    dict(timestep=1 / 60))
    b = solver.JGS2GpuSolver.create(scenes.cantilever(cells=(5, 1, 1), size=(0.5, 0.1, 0.1)),
                                    dict(timestep=1 / 60))
    image = a.exportState()
    with pytest.raises(solver.JGS2RangeError, match="state image"):
        b.importState(image)
    with pytest.raises(solver.JGS2RangeError, match="state image"):
        a.importState(image[:-4])
    bad = bytearray(image)
    bad[0:8] = b"NOTJGS2!"
    with pytest.raises(solver.JGS2RangeError, match="state image"):
        a.importState(bytes(bad))
    a.destroy()
    b.destroy()


def test_asynchronous_position_reads():
    # The reference's readPositions resolves later; jgs2_read_positions_async
    # enqueues the copy after the submitted frames and jgs2_wait_reads waits.
    import torch

    inp = scenes.cantilever(cells=(10, 2, 2), size=(0.5, 0.1, 0.1))
    settings = dict(timestep=1 / 60, iterations=9)
    a = solver.JGS2GpuSolver.create(inp, settings)
    b = solver.JGS2GpuSolver.create(inp, settings)
    bufs = [torch.full((4 * inp.vertex_count,), float("nan"), dtype=torch.float32).pin_memory().numpy()
            for _ in range(2)]
    expect = []
    for i in range(2):
        a.step()
        a.readPositionsAsync(bufs[i])
        b.step()
        expect.append(b.readPositions())
    a.awaitReads()
    for got, want in zip(bufs, expect):
        np.testing.assert_array_equal(got, want)
    a.destroy()
    b.destroy()

"""The continuous-batching request loop: every request's result must be the
same as its scene stepped alone through the plain solver path, whichever
requests it shared a wave with, however the memory budget split them into
waves.  Results are compared bitwise: a wave keeps each scene's reductions to
itself, and body correction (double atomics in a run-dependent order) is off.
"""
import numpy as np
import pytest

from jgs2_b200 import _ffi, scenes, server, solver

BASE = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), floorStiffness=0.0, parityMode=True, iterations=5)


@pytest.fixture(scope="module")
def bars():
    return [scenes.cantilever(cells=(4 + 2 * i, 2, 2), size=(0.2 + 0.1 * i, 0.1, 0.1)) for i in range(4)]


def _alone(inp, settings, frames, exact):
    s = solver.JGS2GpuSolver.create(inp, settings)
    if exact:
        s.stepFramesExactIterations(frames, exact)
    else:
        s.stepFrames(frames)
    out = s.readPositions(), s.readVelocities()
    s.destroy()
    return out


def test_server_rejects_requests_larger_than_the_budget(bars):
    srv = server.JGS2Server(memoryBudgetBytes=1024)
    with pytest.raises(_ffi.JGS2Error, match="more device memory than the whole serving budget"):
        srv.submit(bars[0], BASE, frames=1)
    srv.destroy()


def test_server_rejects_invalid_input(bars):
    srv = server.JGS2Server(memoryBudgetBytes=1 << 30)
    bad = bars[0].copy()
    bad.tet_meta[0] = 0.0
    with pytest.raises(solver.JGS2RangeError, match="positive volume"):
        srv.submit(bad, BASE, frames=1)
    srv.destroy()


@pytest.mark.gpu
def test_served_results_equal_results_alone(bars):
    requests = [(bars[0], dict(BASE), 3, 4), (bars[1], dict(BASE, gravity=(0.0, -3.0, 0.0)), 5, 4),
                (bars[2], dict(BASE), 2, 4), (bars[3], dict(BASE), 4, 6), (bars[1], dict(BASE), 3, 0)]
    srv = server.JGS2Server(memoryBudgetBytes=1 << 32)
    ids = [srv.submit(inp, o, frames=f, exactIterations=e) for inp, o, f, e in requests]
    results = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.destroy()
    assert stats["completed"] == len(requests) and stats["failed"] == 0
    for (inp, o, f, e), r in zip(requests, results):
        assert r["status"] == 0 and r["frames"] == f
        pos, vel = _alone(inp, o, f, e)
        np.testing.assert_array_equal(r["positions"], pos)
        np.testing.assert_array_equal(r["velocities"], vel)


@pytest.mark.gpu
def test_memory_budget_splits_waves_without_changing_results(bars):
    budget = max(server.estimate_device_bytes(b) for b in bars) + 1  # one scene at a time
    srv = server.JGS2Server(memoryBudgetBytes=budget)
    ids = [srv.submit(b, BASE, frames=2, exactIterations=4) for b in bars]
    results = [srv.wait(i) for i in ids]
    stats = srv.stats()
    srv.destroy()
    assert stats["waves_created"] == len(bars)
    assert stats["peak_resident_bytes"] <= budget
    for b, r in zip(bars, results):
        assert r["wave_scenes"] == 1
        pos, _vel = _alone(b, BASE, 2, 4)
        np.testing.assert_array_equal(r["positions"], pos)


@pytest.mark.gpu
def test_batch_without_colouring_refuses_graph_coloured_steps(bars):
    batch = solver.JGS2Batch.create(bars[:2], BASE)
    with pytest.raises(_ffi.JGS2Error, match="without graph colouring"):
        batch.stepFrames(1, exactIterations=2, overrides={"schedule": "graph-colored-gauss-seidel"})
    batch.destroy()


@pytest.mark.gpu
def test_served_contact_surface_requests_equal_results_alone():
    # Trough requests through the device broad phase share waves; each keeps
    # its own rows, list span and reductions, so it runs as it runs alone.
    # (Alone here is a one-scene batch: the contact scenes' static twins
    # would colour past 256 colours, and a batch does not colour.)
    troughs = [scenes.trough(n, contact=scenes.CONTACT_SURFACE) for n in (1, 2, 3)]
    st = dict(scenes.TROUGH_SETTINGS)
    requests = [(troughs[0], 6), (troughs[1], 4), (troughs[2], 6), (troughs[1], 2)]
    srv = server.JGS2Server(memoryBudgetBytes=1 << 32)
    ids = [srv.submit(inp, st, frames=f, exactIterations=3) for inp, f in requests]
    results = [srv.wait(i) for i in ids]
    srv.destroy()
    for (inp, f), r in zip(requests, results):
        assert r["status"] == 0 and r["frames"] == f
        alone = solver.JGS2Batch.create([inp], [st])
        alone.stepFrames(f, exactIterations=3)
        np.testing.assert_array_equal(r["positions"], alone.readPositions(0))
        alone.destroy()

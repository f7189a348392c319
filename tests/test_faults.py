"""Failure detection without a GPU fault: a device allocation that fails
partway through create (injected on the host with JGS2_FAIL_ALLOCATION)
returns JGS2_OUT_OF_MEMORY with the failing call named, releases every
allocation the create made, and leaves the device usable; invalid poses are
refused by validation before any kernel runs."""
import os

import numpy as np
import pytest
import torch

from jgs2_b200 import _ffi, scenes, solver

pytestmark = pytest.mark.gpu

SETTINGS = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0))


def _bar():
    return scenes.cantilever(cells=(6, 2, 2), size=(0.6, 0.2, 0.2))


def _create_failing_at(n, make):
    os.environ["JGS2_FAIL_ALLOCATION"] = str(n)
    try:
        return make()
    finally:
        del os.environ["JGS2_FAIL_ALLOCATION"]


@pytest.mark.parametrize("n", [0, 4, 12, 24])
def test_injected_allocation_failure_releases_everything(n):
    inp = _bar()
    torch.cuda.init()
    warm = solver.JGS2GpuSolver.create(inp, SETTINGS)  # module load and first-use allocations
    warm.destroy()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    with pytest.raises(_ffi.JGS2Error) as err:
        _create_failing_at(n, lambda: solver.JGS2GpuSolver.create(inp, SETTINGS))
    assert err.value.status == 3  # JGS2_OUT_OF_MEMORY
    assert "JGS2_FAIL_ALLOCATION" in err.value.message
    torch.cuda.synchronize()
    assert abs(torch.cuda.mem_get_info()[0] - free_before) <= 4 << 20
    # The device and library stay usable.
    s = solver.JGS2GpuSolver.create(inp, SETTINGS)
    s.step()
    assert np.isfinite(s.readPositions()).all()
    s.destroy()


def test_injected_allocation_failure_in_a_batch():
    parts = [_bar(), _bar()]
    with pytest.raises(_ffi.JGS2Error) as err:
        _create_failing_at(6, lambda: solver.JGS2Batch.create(parts, SETTINGS))
    assert err.value.status == 3
    b = solver.JGS2Batch.create(parts, SETTINGS)
    b.stepFrames(1)
    b.destroy()


def test_nonfinite_and_inverted_initial_poses_are_refused():
    inp = _bar()
    bad = inp.copy()
    pos = bad.positions.reshape(-1, 4).copy()
    pos[3, 1] = np.nan
    bad.positions = pos.reshape(-1)
    with pytest.raises(solver.JGS2RangeError):
        solver.JGS2GpuSolver.create(bad, SETTINGS)
    inv = inp.copy()
    pos = inv.positions.reshape(-1, 4).copy()
    pos[:, 0] *= -1.0  # a mirrored mesh: every tet inverted
    inv.positions = pos.reshape(-1)
    with pytest.raises(_ffi.JGS2Error) as err:
        solver.JGS2GpuSolver.create(inv, SETTINGS)
    assert err.value.status in (1, 2)  # invalid argument or infeasible input

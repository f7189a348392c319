"""Device broad phase over the static IPC candidate superset (contact
surfaces, jgs2_input.contact_surface).

The reference lists every candidate of its surface up front
(buildStaticIpcContactCandidates, src/simulation/cpu/ipc-contact.ts:591-665);
the broad phase lists, each iteration, the candidates that can act in it, in
the same canonical order, so a contact-surface run is the static run.

CPU tests: the surface enumeration's exact minimum distance equals the static
superset's over interpenetrating poses (same pairs, same exclusions), the
packer's surface gives the reference's candidate count, and the input checks.
GPU tests: contact-surface runs against static runs of the same scenes
(positions bitwise), the listed candidates against the superset (canonical
order, every candidate within the activation distance listed), the capacity
and settings errors, and a box pile that stays intersection-free under the
exact check.
"""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

D_HAT = 0.08


def _small(contact, **kw):
    args = dict(boxes=3, cells=3, heights=(1.0, 1.3), plate_cells=(8, 2), method=scenes.PRECOMPUTE_PATCH)
    args.update(kw)
    return scenes.box_trough(contact=contact, **args)


# ---- CPU --------------------------------------------------------------------------------

def test_surface_minimum_matches_static_superset():
    a = _small(scenes.CONTACT_STATIC)
    b = _small(scenes.CONTACT_SURFACE)
    assert a.vertex_count == b.vertex_count
    rng = np.random.default_rng(7)
    base = a.positions.reshape(-1, 4).copy()
    info = a.vertex_info.reshape(-1, 4)
    bodies = info[:, 3]
    for trial in range(8):
        pos = base.copy()
        # Drop every box onto the apex and into each other: many close and
        # interpenetrating pairs, so a missed or extra pair shows.
        for body in range(1, bodies.max() + 1):
            sel = bodies == body
            centre = pos[sel, :3].mean(axis=0)
            target = np.array([rng.uniform(-0.05, 0.05), rng.uniform(0.1, 0.3), rng.uniform(-0.1, 0.1)])
            pos[sel, :3] += target - centre
        d_static = solver.minimum_contact_distance(a, pos)
        d_surface = solver.minimum_contact_distance(b, pos, cutoff=100.0)
        assert d_surface == d_static, (trial, d_static, d_surface)
        # A cutoff above the minimum finds the same pair.
        assert solver.minimum_contact_distance(b, pos, cutoff=d_static + 1e-3) == d_static


def test_packed_surface_gives_the_reference_superset():
    a = scenes.trough(10)
    b = scenes.trough(10, contact=scenes.CONTACT_SURFACE)
    assert b.contact_indices is None and b.contact_surface is not None
    cand, vt, ee = scenes.static_contact_candidates(b.vertex_count, b.contact_surface)
    assert (vt, ee) == tuple(int(x) for x in a.contact_counts) and vt + ee == 31801
    np.testing.assert_array_equal(cand, a.contact_indices)
    assert solver.contact_superset_size(b) == 31801
    small = _small(scenes.CONTACT_STATIC)
    assert solver.contact_superset_size(_small(scenes.CONTACT_SURFACE)) == small.contact_candidate_count


def test_surface_input_checks():
    b = scenes.trough(1, contact=scenes.CONTACT_SURFACE)
    solver.validate_input(b)
    both = b.copy()
    a = scenes.trough(1)
    both.contact_indices, both.contact_counts = a.contact_indices, a.contact_counts
    with pytest.raises(solver.JGS2RangeError, match="either static IPC candidates or a contact surface"):
        solver.validate_input(both)
    bad = b.copy()
    bad.contact_surface = bad.contact_surface.copy()
    bad.contact_surface[4] = bad.vertex_count
    with pytest.raises(solver.JGS2RangeError, match="outside vertexCount"):
        solver.validate_input(bad)
    bad.contact_surface[4] = bad.contact_surface[3]
    with pytest.raises(solver.JGS2RangeError, match="three distinct vertices"):
        solver.validate_input(bad)
    big = b.copy()
    big.contact_capacity = 1 << 28
    with pytest.raises(solver.JGS2RangeError, match="capacity"):
        solver.validate_input(big)


# ---- GPU --------------------------------------------------------------------------------

@pytest.mark.gpu
def test_reference_trough_surface_run_is_the_static_run():
    static = scenes.trough(10)
    surface = scenes.trough(10, contact=scenes.CONTACT_SURFACE)
    a = solver.JGS2GpuSolver.create(static, scenes.TROUGH_SETTINGS)
    b = solver.JGS2GpuSolver.create(surface, scenes.TROUGH_SETTINGS)
    assert b.info()["contact_candidate_capacity"] > 0
    for block in range(8):
        a.stepFrames(12)
        b.stepFrames(12)
        np.testing.assert_array_equal(b.readPositions(), a.readPositions(), err_msg=f"frame {12 * (block + 1)}")
        np.testing.assert_array_equal(b.readVelocities(), a.readVelocities())
    # Minimum determinants and the accept decision of the last iteration; the
    # energies sum the same terms in another order.
    da, db = a.readGlobalizationDiagnostics(), b.readGlobalizationDiagnostics()
    np.testing.assert_array_equal(db["control"][:8], da["control"][:8])
    a.destroy()
    b.destroy()


@pytest.mark.gpu
def test_listed_candidates_are_the_acting_part_of_the_superset():
    static = scenes.trough(10)
    surface = scenes.trough(10, contact=scenes.CONTACT_SURFACE)
    gpu = solver.JGS2GpuSolver.create(surface, scenes.TROUGH_SETTINGS)
    superset = static.contact_indices.reshape(-1, 4).astype(np.int64)
    vt, ee = (int(x) for x in static.contact_counts)
    keys = {(0,) + tuple(c): i for i, c in enumerate(superset[:vt])}
    keys.update({(1,) + tuple(c): vt + i for i, c in enumerate(superset[vt:])})
    lib = O.lib()
    for frames in (30, 30, 36):
        gpu.stepFrames(frames)
        listed = gpu.readContactCandidates().astype(np.int64)
        assert listed.shape[0] == gpu.contactCandidateCount > 0
        kind = listed[:, 3] >> 31
        listed[:, 3] &= 0x7FFFFFFF
        idx = np.array([keys[(int(k),) + tuple(int(x) for x in c)] for k, c in zip(kind, listed)])
        assert (np.diff(idx) > 0).all(), "listed candidates leave the superset's canonical order"
        # Every superset candidate within the activation distance of the
        # final pose was listed by the last iteration.
        pos = gpu.readPositions().reshape(-1, 4)[:, :3].astype(np.float64)
        near = []
        for i, c in enumerate(superset):
            x = pos[c].reshape(-1)
            d = _distance(lib, 0 if i < vt else 1, x)
            if d <= D_HAT:
                near.append(i)
        assert set(near) <= set(idx.tolist()), sorted(set(near) - set(idx.tolist()))[:10]
    gpu.destroy()


def _distance(lib, kind, x):
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    lib.jgs2_oracle_ipc_contact.argtypes = [ctypes.c_uint32, D, D]
    out = np.zeros(9)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    lib.jgs2_oracle_ipc_contact(kind, xx.ctypes.data_as(D), out.ctypes.data_as(D))
    return out[0]


@pytest.mark.gpu
def test_box_trough_surface_run_is_the_static_run():
    # The static superset of this pile needs more than the 256 colours a
    # solver's create-time colouring allows, so both run as one-scene batches
    # (which colour only for the coloured schedule).
    static = _small(scenes.CONTACT_STATIC)
    surface = _small(scenes.CONTACT_SURFACE)
    s = scenes.BOX_TROUGH_SETTINGS
    a = solver.JGS2Batch.create([static], [s])
    b = solver.JGS2Batch.create([surface], [s])
    for _ in range(4):
        a.stepFrames(10, exactIterations=15)
        b.stepFrames(10, exactIterations=15)
        np.testing.assert_array_equal(b.readPositions(0), a.readPositions(0))
    assert b.info(0)["contact_candidate_count"] > 0
    d = solver.minimum_contact_distance(surface, b.readPositions(0), cutoff=1.0)
    assert d > s["ipcMinimumDistance"], d
    a.destroy()
    b.destroy()


@pytest.mark.gpu
def test_box_pile_stays_intersection_free():
    inp = scenes.box_trough(boxes=6, cells=4, heights=(1.0, 1.6), method=scenes.PRECOMPUTE_PATCH)
    s = scenes.BOX_TROUGH_SETTINGS
    gpu = solver.JGS2GpuSolver.create(inp, s)
    p0 = gpu.readPositions().reshape(-1, 4)[:, :3].copy()
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    closest = np.inf
    for block in range(12):
        gpu.stepFramesExactIterations(10, s["iterations"])
        pos4 = gpu.readPositions()
        pos = pos4.reshape(-1, 4)[:, :3]
        assert np.isfinite(pos).all()
        assert np.abs(pos[pinned] - p0[pinned]).max() < 2e-5
        d = solver.minimum_contact_distance(inp, pos4, cutoff=0.05)
        assert d > s["ipcMinimumDistance"], f"frame {10 * (block + 1)}: distance {d}"
        closest = min(closest, d)
    # The boxes landed: some pair came inside the activation band.
    assert closest < s["ipcActivationDistance"], closest
    gpu.destroy()


@pytest.mark.gpu
def test_capacity_overflow_fails_the_step_without_faulting():
    inp = scenes.trough(4, contact=scenes.CONTACT_SURFACE, capacity=16)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    gpu.stepFrames(90)
    with pytest.raises(solver._ffi.JGS2Error, match="above its capacity"):
        gpu.awaitIdle()
    gpu.destroy()


@pytest.mark.gpu
def test_surface_settings_checks():
    inp = scenes.trough(1, contact=scenes.CONTACT_SURFACE)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    with pytest.raises(solver.JGS2RangeError, match="Jacobi schedule only"):
        gpu.step({"schedule": "graph-colored-gauss-seidel"})
    with pytest.raises(solver.JGS2RangeError, match="maxStep must be positive"):
        gpu.step({"maxStep": 0.0})
    gpu.step()
    gpu.destroy()


@pytest.mark.gpu
def test_surface_batch_matches_alone():
    # The serving loop steps contact-surface requests as one batch: each
    # scene's rows, list span, reductions and active rows stay its own, so a
    # scene runs bitwise as it runs alone.
    parts = [scenes.trough(2, contact=scenes.CONTACT_SURFACE), _small(scenes.CONTACT_SURFACE),
             scenes.trough(1, contact=scenes.CONTACT_SURFACE)]
    opts = [dict(scenes.TROUGH_SETTINGS), dict(scenes.BOX_TROUGH_SETTINGS), dict(scenes.TROUGH_SETTINGS)]
    batch = solver.JGS2Batch.create(parts, opts)
    alone = [solver.JGS2Batch.create([p], [o]) for p, o in zip(parts, opts)]
    for frames in (10, 30):
        batch.stepFrames(frames, exactIterations=3)
        for a in alone:
            a.stepFrames(frames, exactIterations=3)
        for i, a in enumerate(alone):
            np.testing.assert_array_equal(batch.readPositions(i), a.readPositions(0), err_msg=f"scene {i}")
            assert batch.info(i)["contact_candidate_count"] == a.info(0)["contact_candidate_count"]
    for a in alone:
        a.destroy()
    batch.destroy()

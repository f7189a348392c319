"""jgs2_gate_candidate_no_alloc, the allocation-free gate, against
jgs2_evaluate_assembled_candidate on the same poses: two calls in a row
through the C-ABI, on device arrays the test owns.

Tolerances: minimum determinants, validity bits, accept / revert flags and
the sweep aggregates equal exactly (minima and flags do not depend on the
reduction order); assembled energies within rtol 1e-6 (the two kernels sum
the same per-element f32 energies in double with different block groupings,
then round to f32).
"""
from ctypes import POINTER, c_int, c_uint32, c_void_p

import numpy as np
import pytest
import torch

from jgs2_b200 import _ffi, scenes, solver

pytestmark = pytest.mark.gpu

ENERGY_RTOL = 1e-6
SETTINGS = dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), floorStiffness=0.0, parityMode=True)


def _entry():
    lib = _ffi.step_lib()
    f = lib.jgs2_gate_candidate_no_alloc
    f.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, POINTER(_ffi.Settings), c_uint32, c_void_p, c_void_p]
    f.restype = c_int
    return f


@pytest.fixture(scope="module")
def bar():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((24, 4, 4), (0.0, 0.0, 0.0), (1.2, 0.2, 0.2), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=1 / 60, cubature_k=6)
    return sc.pack()


def _poses(inp):
    rng = np.random.default_rng(20240611)
    src = inp.positions.astype(np.float32).reshape(-1, 4).copy()
    src[:, :3] += rng.normal(0.0, 2e-3, size=(inp.vertex_count, 3)).astype(np.float32)
    accepted = src.copy()
    accepted[:, :3] += rng.normal(0.0, 1e-3, size=(inp.vertex_count, 3)).astype(np.float32)
    # Push one free vertex through the opposite face of its first tet.
    rejected = src.copy()
    q = inp.tet_indices.reshape(-1, 4)[0]
    free = [v for v in q if inp.vertex_info.reshape(-1, 4)[v, 2] == 0]
    v = int(free[0])
    others = [int(u) for u in q if int(u) != v]
    centroid = src[others, :3].mean(axis=0)
    rejected[v, :3] = centroid + 1.5 * (centroid - src[v, :3])
    return src.reshape(-1), [("accepted", accepted.reshape(-1)), ("rejected", rejected.reshape(-1))]


def _cloth_poses(inp):
    """An accepted small perturbation of the sheet and a rejected one that
    mirrors a free cloth vertex through the opposite edge of its triangle
    (the triangle's signed area stretch turns negative)."""
    rng = np.random.default_rng(20240612)
    info = inp.vertex_info.reshape(-1, 4)
    src = inp.positions.astype(np.float32).reshape(-1, 4).copy()
    free = info[:, 2] == 0
    accepted = src.copy()
    accepted[free, :3] += rng.normal(0.0, 1e-4, size=(int(free.sum()), 3)).astype(np.float32)
    tris = inp.cloth_triangles.reshape(-1, 3).astype(np.int64)
    rejected = src.copy()
    for t in tris[::-1]:
        if all(info[int(q), 2] == 0 for q in t):
            v, a, c = (int(q) for q in t)
            mid = 0.5 * (src[a, :3] + src[c, :3])
            rejected[v, :3] = mid + (mid - src[v, :3])
            break
    else:
        raise AssertionError("no free cloth triangle")
    return src.reshape(-1), [("accepted", accepted.reshape(-1)), ("rejected", rejected.reshape(-1))]


def _to_device(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to("cuda")


def _check_against_existing_entry(inp, settings, src, cases):
    gate = _entry()
    gpu = solver.JGS2GpuSolver.create(inp, settings)
    # The existing entry point, once per candidate.
    refs = [gpu.evaluateAssembledCandidateForTest(src, cand) for _name, cand in cases]
    assert refs[0]["history"][4] == 1.0 and refs[1]["history"][5] == 1.0  # one accepted, one reverted

    d_src = _to_device(src)
    d_pred = _to_device(src)
    d_cands = [_to_device(cand) for _name, cand in cases]
    d_ctls = [torch.full((16,), float("nan"), dtype=torch.float32, device="cuda") for _ in cases]
    assert all(t.data_ptr() % 16 == 0 for t in [d_src, d_pred, *d_cands, *d_ctls])
    torch.cuda.synchronize()
    # Two calls in a row on the solver's stream, then one wait.
    for d_cand, d_ctl in zip(d_cands, d_ctls):
        status = gate(gpu._h, d_src.data_ptr(), d_cand.data_ptr(), d_pred.data_ptr(), None, 0, d_ctl.data_ptr(),
                      None)
        assert status == 0, _ffi.step_lib().jgs2_last_error(gpu._h)
    gpu.awaitIdle()
    for (name, _cand), ref, d_ctl in zip(cases, refs, d_ctls):
        ctl = d_ctl.cpu().numpy()
        h = ref["history"]
        np.testing.assert_array_equal(ctl[0:4], h[0:4], err_msg=name)    # minima, validity bits
        np.testing.assert_array_equal(ctl[4:7], h[4:7], err_msg=name)    # accepted, reverted, failures
        assert ctl[7] == 0.0, name                                       # history slot
        np.testing.assert_allclose(ctl[8:11], h[8:11], rtol=ENERGY_RTOL, err_msg=name)
        assert ctl[11] == h[11], name                                    # energy validity
        np.testing.assert_array_equal(ctl[12:16], ref["control"][12:16], err_msg=name)  # sweep aggregates
    # The gate changed no solver state: the canonical pose is still the one
    # the last existing-entry call left.
    np.testing.assert_array_equal(gpu.readPositions(), refs[1]["positions"])
    gpu.destroy()


def test_no_alloc_gate_matches_assembled_candidate(bar):
    src, cases = _poses(bar)
    _check_against_existing_entry(bar, SETTINGS, src, cases)


def test_no_alloc_gate_matches_on_cloth():
    # A tet collider and a 6x6-cell StVK sheet: the membrane and hinge terms
    # of the allocation-free kernel against the existing entry point.
    inp = scenes.cloth_drape(cells=6, prefold=False, pinned_columns=(0, 6))
    assert inp.cloth_triangle_count > 0 and inp.hinge_count > 0
    src, cases = _cloth_poses(inp)
    _check_against_existing_entry(inp, dict(SETTINGS, timestep=1 / 120), src, cases)


def test_no_alloc_gate_refuses_contact_solvers():
    inp = scenes.trough(boxes=2)
    assert inp.contact_candidate_count > 0
    gate = _entry()
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    d = torch.zeros(4 * inp.vertex_count, dtype=torch.float32, device="cuda")
    ctl = torch.zeros(16, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    status = gate(gpu._h, d.data_ptr(), d.data_ptr(), d.data_ptr(), None, 0, ctl.data_ptr(), None)
    assert status == 7  # JGS2_UNSUPPORTED
    assert b"contact" in _ffi.step_lib().jgs2_last_error(gpu._h)
    gpu.destroy()


def test_no_alloc_gate_rejects_misaligned_arrays(bar):
    gate = _entry()
    gpu = solver.JGS2GpuSolver.create(bar, SETTINGS)
    d = torch.zeros(4 * bar.vertex_count + 4, dtype=torch.float32, device="cuda")
    ctl = torch.zeros(16, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    status = gate(gpu._h, d.data_ptr() + 4, d.data_ptr(), d.data_ptr(), None, 0, ctl.data_ptr(), None)
    assert status == 1
    assert b"16-byte aligned" in _ffi.step_lib().jgs2_last_error(gpu._h)
    gpu.destroy()

"""Assembled determinant gate + whole-pose revert on the single-tetrahedron
fixture, after the reference's known-answer cases
(tests/e2e/nonlinear-globalization-gpu.spec.ts:181-384): two shears that each
keep J = 1 are accepted, their Jacobi-assembled combination (J = 1 - 1.1^2 =
-0.21) is reverted to the source, and a finite pose whose f32 edge overflows
is reverted with invalid candidate geometry.

The oracle cases run on the CPU and pin the oracle's gate to those answers;
the GPU cases run the same poses through the C-ABI and compare with both.
"""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver
from oracle import oracle as O

SETTINGS = dict(timestep=1 / 60, gravity=(0.0, 0.0, 0.0), iterations=1, floor_stiffness=0.0,
                velocity_damping=1.0, contact_tangential_damping=0.0, contact_margin=0.0,
                horizontal_body_correction=0, parity_mode=1)

BITS = dict(source_geometry=1, candidate_geometry=2, accepted_minimum=4, local_numerics=8)


def decode_history(h):
    """The fields of one 32-float history record the reference's test reads
    (decodeJGS2GlobalizationHistoryRecord, src/simulation/gpu/jgs2-globalization.ts:341-510)."""
    h = np.asarray(h, dtype=np.float32)
    fin = lambda x: bool(np.isfinite(x))
    bits = int(h[3])
    sgv = bool(bits & BITS["source_geometry"]) and fin(h[0])
    cgv = bool(bits & BITS["candidate_geometry"]) and fin(h[1])
    amv = bool(bits & BITS["accepted_minimum"]) and fin(h[2])
    lnv = bool(bits & BITS["local_numerics"])
    all_valid = bool(np.all(np.isfinite(h[[0, 1, 2, 8, 9, 10]]))) and bool(np.all(np.isfinite(h[12:22])))
    return dict(
        source_min=float(h[0]), candidate_min=float(h[1]), accepted_min=float(h[2]),
        source_geometry_valid=sgv, candidate_geometry_valid=cgv, accepted_min_valid=amv,
        local_numerics_valid=lnv, geometry_valid=sgv and cgv,
        accepted=h[4] == 1.0, reverted=h[5] == 1.0, local_failures=int(h[6]), revert_count=int(h[7]),
        source_energy=float(h[8]), candidate_energy=float(h[9]), accepted_energy=float(h[10]),
        energy_valid=h[11] == 1.0 and bool(np.all(np.isfinite(h[8:11]))),
        maximum_update=float(h[20]), converged=h[24] == 1.0,
        finite=h[25] == 1.0 and all_valid and sgv and cgv and amv and lnv,
        iteration_index=int(h[26]), active=h[31] == 1.0)


def _cases(source):
    src = source.reshape(-1).astype(np.float32).copy()
    b, c, combined, nonfinite = src.copy(), src.copy(), src.copy(), src.copy()
    b[1 * 4 + 1] += 1.1
    c[2 * 4] += 1.1
    combined[1 * 4 + 1] += 1.1
    combined[2 * 4] += 1.1
    nonfinite[0] = -3e38
    nonfinite[1 * 4] = 3e38
    return src, [("candidate-b", b), ("candidate-c", c), ("combined", combined), ("nonfinite", nonfinite)]


def _check_known_answers(src, cases, results):
    for (name, cand), r in zip(cases, results):
        h = decode_history(r["history"])
        assert h["source_min"] == pytest.approx(1.0, abs=5e-6), name
        assert h["source_geometry_valid"] and h["accepted_min_valid"] and h["local_numerics_valid"], name
        assert h["local_failures"] == 0, name
        assert h["iteration_index"] == 0 and h["active"], name
        if name in ("candidate-b", "candidate-c"):
            assert h["candidate_min"] == pytest.approx(1.0, abs=5e-6), name
            assert h["accepted_min"] == pytest.approx(1.0, abs=5e-6), name
            assert h["accepted"] and not h["reverted"] and h["revert_count"] == 0, name
            np.testing.assert_array_equal(r["positions"], cand, err_msg=name)
            assert h["energy_valid"] and h["candidate_geometry_valid"] and h["geometry_valid"], name
            assert h["finite"], name
            assert h["candidate_energy"] > h["source_energy"], name
            assert h["accepted_energy"] == h["candidate_energy"], name
        elif name == "combined":
            assert h["candidate_min"] == pytest.approx(-0.21, abs=5e-6)
            assert h["candidate_geometry_valid"] and h["geometry_valid"]
            assert h["accepted_min"] == pytest.approx(1.0, abs=5e-6)
            assert not h["accepted"] and h["reverted"] and h["revert_count"] == 1
            np.testing.assert_array_equal(r["positions"], src)
            assert h["maximum_update"] == 0.0 and not h["converged"]
            assert not h["energy_valid"] and h["finite"]
        else:
            assert h["candidate_min"] == 0.0
            assert not h["candidate_geometry_valid"] and not h["geometry_valid"]
            assert h["accepted_min"] == pytest.approx(1.0, abs=5e-6)
            assert not h["accepted"] and h["reverted"] and h["revert_count"] == 1
            np.testing.assert_array_equal(r["positions"], src)
            assert h["maximum_update"] == 0.0 and not h["converged"]
            assert not h["energy_valid"] and not h["finite"]


@pytest.fixture(scope="module")
def tet():
    return scenes.single_tetrahedron()


@pytest.mark.parametrize("precision", [32, 64])
def test_oracle_assembled_candidate_known_answers(tet, precision):
    cpu = O.OracleSolver(tet, SETTINGS, precision=precision)
    src, cases = _cases(tet.positions)
    results = [cpu.evaluate_assembled_candidate(src, cand) for _name, cand in cases]
    _check_known_answers(src, cases, results)


@pytest.mark.gpu
def test_gpu_assembled_candidate_known_answers_and_oracle(tet):
    inv = {v: k for k, v in solver.CAMEL.items()}
    camel = {inv.get(k, k): (bool(v) if k in ("parity_mode", "horizontal_body_correction") else v)
             for k, v in SETTINGS.items()}
    gpu = solver.JGS2GpuSolver.create(tet, camel)
    cpu = O.OracleSolver(tet, SETTINGS, precision=32)
    src, cases = _cases(tet.positions)
    results = []
    for name, cand in cases:
        g = gpu.evaluateAssembledCandidateForTest(src, cand)
        c = cpu.evaluate_assembled_candidate(src, cand)
        np.testing.assert_array_equal(g["positions"].reshape(-1, 4)[:, :3], c["positions"].reshape(-1, 4)[:, :3],
                                      err_msg=name)
        # Geometry, decisions and counts agree exactly; energies and norms to
        # f32 reduction-order tolerance.
        gh, ch = g["history"], c["history"]
        exact = [0, 1, 2, 3, 4, 5, 6, 7, 11, 22, 23, 24, 25, 26, 28, 29, 30, 31]
        np.testing.assert_array_equal(gh[exact], ch[exact], err_msg=name)
        np.testing.assert_allclose(gh[8:11], ch[8:11], rtol=1e-5, atol=1e-6, err_msg=name)
        np.testing.assert_allclose(gh[12:22], ch[12:22], rtol=1e-4, atol=1e-6, err_msg=name)
        d = gpu.readGlobalizationDiagnostics()
        assert d["historyCount"] == 1, name
        results.append(g)
    gpu.destroy()
    _check_known_answers(src, cases, results)


def _pinned_target_input(tet):
    """A feasible 180-degree rigid rotation (J = +1) whose newly pinned vertex B
    proposes its rest target, making the complete candidate J = -1
    (tests/e2e/nonlinear-globalization-gpu.spec.ts:243-296)."""
    inp = tet.copy()
    inp.positions = np.array([0, 0, 0, 1, -1, 0, 0, 1, 0, -1, 0, 1, 0, 0, 1, 1], np.float32)
    inp.velocities = np.zeros(16, np.float32)
    inp.vertex_info = inp.vertex_info.copy()
    inp.vertex_info[1 * 4 + 2] = 1
    return inp


def _check_pinned_target(inp, positions, h):
    h = decode_history(h)
    assert h["source_min"] == pytest.approx(1.0, abs=5e-6)
    assert h["candidate_min"] == pytest.approx(-1.0, abs=5e-6)
    assert h["accepted_min"] == pytest.approx(1.0, abs=5e-6)
    assert not h["accepted"] and h["reverted"]
    np.testing.assert_array_equal(positions.reshape(-1, 4)[:, :3], inp.positions.reshape(-1, 4)[:, :3])


def test_oracle_pinned_target_revert(tet):
    inp = _pinned_target_input(tet)
    cpu = O.OracleSolver(inp, SETTINGS, precision=32)
    cpu.step_exact_iterations(1)
    _check_pinned_target(inp, cpu.read("positions"), cpu.read("history")[:32])


@pytest.mark.gpu
def test_gpu_pinned_target_revert(tet):
    inp = _pinned_target_input(tet)
    inv = {v: k for k, v in solver.CAMEL.items()}
    camel = {inv.get(k, k): (bool(v) if k in ("parity_mode", "horizontal_body_correction") else v)
             for k, v in SETTINGS.items()}
    gpu = solver.JGS2GpuSolver.create(inp, camel)
    gpu.stepExactIterations(1)
    d = gpu.readGlobalizationDiagnostics()
    assert d["historyCount"] == 1
    _check_pinned_target(inp, gpu.readPositions(), np.asarray(d["history"][0], dtype=np.float32))
    gpu.destroy()


@pytest.mark.parametrize("precision", [64, 32])
def test_gate_reports_the_exact_determinant_of_an_affine_candidate(precision):
    # nonlinear-oracle.test.ts:304-330: an affine pose A X gives every tet the
    # deformation gradient A, so the gate's candidate minimum is det A.
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((2, 1, 1), (0.0, 0.0, 0.0), (0.2, 0.1, 0.1), m, 0, 0)
    sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    inp = sc.pack()
    A = np.array([[0.9, 0.1, 0.0], [-0.05, 1.1, 0.2], [0.0, 0.05, 0.85]])
    rest = inp.positions.reshape(-1, 4).copy()
    cand = rest.copy()
    cand[:, :3] = (rest[:, :3].astype(np.float64) @ A.T).astype(np.float32)
    cpu = O.OracleSolver(inp, SETTINGS, precision=precision)
    control = cpu.evaluate_assembled_candidate(rest.reshape(-1), cand.reshape(-1))["control"]
    assert abs(control[0] - 1.0) < 1e-6  # the source is the rest shape
    assert abs(control[1] - np.linalg.det(A)) < (1e-6 if precision == 64 else 1e-5)

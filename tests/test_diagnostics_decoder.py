"""The host mirror's globalization record decoders against the reference's
decoder tests (src/simulation/gpu/jgs2-globalization.test.ts:35-470)."""
import math

import numpy as np
import pytest

from jgs2_b200 import diagnostics as D
from jgs2_b200.solver import JGS2RangeError

NAN, INF = math.nan, math.inf


def test_frozen_policy_strides_and_status_codes():
    assert (D.HISTORY_CAPACITY, D.LOCAL_DIAGNOSTIC_VEC4S, D.CONTROL_VEC4S, D.HISTORY_VEC4S) == (64, 4, 4, 8)
    assert D.RELATIVE_EIGENVALUE_FLOOR == 2.0 ** -16 and D.MAX_NORMALIZED_SHIFT == 1e-3
    assert D.DETERMINANT_FLOOR == 1e-4 and D.ARMIJO_C1 == 1e-4
    assert D.BACKTRACK_FACTOR == 0.5 and D.MAX_BACKTRACKS == 12
    assert (D.SOURCE_GEOMETRY_VALID_BIT, D.CANDIDATE_GEOMETRY_VALID_BIT, D.ACCEPTED_MINIMUM_VALID_BIT,
            D.LOCAL_NUMERICS_VALID_BIT, D.VALIDITY_BITS_MASK) == (1, 2, 4, 8, 15)
    assert D.LOCAL_STATUS_CODES == {"accepted": 0, "pinned": 1, "zeroGradient": 2, "shiftLimit": 3,
                                    "nonDescent": 4, "lineSearchFailed": 5, "nonfinite": 6, "choleskyFailed": 7}


def test_decodes_every_lane_of_a_local_record():
    decoded = D.decode_local_diagnostic([1, 2, 3, 0.5, -0.25, 10, 0.01, 0.001, -4, -3.5, -8, 2e-5,
                                         0.125, 2, 3, 0])
    assert decoded == {
        "direction": [1, 2, 3], "alpha": 0.5, "minimumEigenvalue": -0.25, "scale": 10, "diagonalShift": 0.01,
        "normalizedShift": 0.001, "acceptedEnergyDelta": -4, "armijoDeltaBound": -3.5,
        "gradientDotDirection": -8, "shiftedLinearResidual": 2e-5, "minimumTrialDeformationDeterminant": 0.125,
        "backtrackCount": 2, "energyEvaluationCount": 3, "statusCode": 0, "status": "accepted",
        "accepted": True, "directionValid": True, "alphaValid": True, "positiveDefiniteDiagnosticsValid": True,
        "energyDiagnosticsValid": True, "minimumTrialDeformationDeterminantValid": True, "finite": True,
    }


def test_nonfinite_local_numerics_become_finite_zero_sentinels():
    d = D.decode_local_diagnostic([NAN, 2, 3, INF, -INF, 10, 0.01, 0.001, NAN, -3.5, -8, INF, NAN, 0, 0, 6])
    assert d["direction"] == [0, 2, 3]
    assert (d["alpha"], d["minimumEigenvalue"], d["acceptedEnergyDelta"], d["shiftedLinearResidual"],
            d["minimumTrialDeformationDeterminant"]) == (0, 0, 0, 0, 0)
    for key in ("directionValid", "alphaValid", "positiveDefiniteDiagnosticsValid", "energyDiagnosticsValid",
                "minimumTrialDeformationDeterminantValid", "finite"):
        assert d[key] is False


def test_geometry_result_versus_no_trial_and_nonfinite_sentinels():
    record = np.zeros(16, dtype=np.float32)
    record[5] = 1
    record[15] = 2  # zero gradient: no trial was evaluated
    no_trial = D.decode_local_diagnostic(record)
    assert no_trial["minimumTrialDeformationDeterminant"] == 0
    assert not no_trial["minimumTrialDeformationDeterminantValid"] and no_trial["finite"]
    record[15] = 6
    nonfinite = D.decode_local_diagnostic(record)
    assert not nonfinite["minimumTrialDeformationDeterminantValid"] and not nonfinite["finite"]
    record[12] = 0.25
    nonfinite_energy = D.decode_local_diagnostic(record)
    assert nonfinite_energy["minimumTrialDeformationDeterminant"] == 0.25
    assert nonfinite_energy["minimumTrialDeformationDeterminantValid"] and not nonfinite_energy["finite"]
    record[15] = 5
    rejected = D.decode_local_diagnostic(record)
    assert rejected["minimumTrialDeformationDeterminantValid"] and rejected["finite"]


def test_rejects_malformed_local_records():
    for n in (15, 17):
        with pytest.raises(JGS2RangeError, match="expected exactly 16"):
            D.decode_local_diagnostic(np.zeros(n))
    packed = np.zeros(16)
    packed[5] = 1
    for value in (0.5, D.MAX_BACKTRACKS + 1):
        packed[13] = value
        with pytest.raises(JGS2RangeError, match="backtrackCount must be a nonnegative integer"):
            D.decode_local_diagnostic(packed)
    packed[13] = 0
    packed[14] = -1
    with pytest.raises(JGS2RangeError, match="energyEvaluationCount must be a nonnegative integer"):
        D.decode_local_diagnostic(packed)
    packed[14] = 0
    packed[15] = 8
    with pytest.raises(JGS2RangeError, match="status must be an integer from 0 through 7"):
        D.decode_local_diagnostic(packed)


def test_decodes_every_validity_mask():
    packed = np.zeros(32, dtype=np.float32)
    packed[[0, 1, 2]] = [0.5, 0.4, 0.4]
    packed[[18, 25, 31]] = 1
    for mask in range(16):
        packed[3] = mask
        d = D.decode_history_record(packed)
        src, cand, acc, loc = (bool(mask & b) for b in (1, 2, 4, 8))
        assert (d["sourceGeometryValid"], d["candidateGeometryValid"],
                d["acceptedMinimumDeformationDeterminantValid"], d["localNumericsValid"]) == (src, cand, acc, loc)
        assert d["geometryValid"] == (src and cand)
        assert d["finite"] == (mask == 15)


def test_decodes_every_lane_of_a_history_record():
    d = D.decode_history_record([1, -0.21, 1, 15, 0, 1, 2, 1, 20, 19, 20, 1, 3, 4, 5, 6, 7, 8, 9, 0.25,
                                 10, 0.5, 0, 1, 0, 1, 5, 0.0007, 3, 4, 5, 1])
    assert d == {
        "sourceMinimumDeformationDeterminant": 1, "candidateMinimumDeformationDeterminant": -0.21,
        "acceptedMinimumDeformationDeterminant": 1, "sourceGeometryValid": True, "candidateGeometryValid": True,
        "acceptedMinimumDeformationDeterminantValid": True, "localNumericsValid": True, "geometryValid": True,
        "assembledAccepted": False, "assembledReverted": True, "localFailureCount": 2, "revertCount": 1,
        "sourceEnergy": 20, "candidateEnergy": 19, "acceptedEnergy": 20, "energyValid": True,
        "componentGradientNorms": {"inertia": 3, "material": 4, "externalForce": 5, "target": 6, "contact": 7},
        "componentGradientNormsValid": True, "gradientNorm": 8, "residualDenominator": 9, "relativeResidual": 0.25,
        "residualDiagnosticsValid": True, "maximumUpdate": 10, "normalizedMaximumUpdate": 0.5,
        "updateDiagnosticsValid": True, "residualSatisfied": False, "updateSatisfied": True, "converged": False,
        "finite": True, "iterationIndex": 5, "maximumLocalNormalizedShift": 0.0007,
        "maximumLocalNormalizedShiftValid": True, "maximumBacktrackCount": 3, "infeasibleTrialCount": 4,
        "energyEvaluationCount": 5, "active": True,
    }


def test_validity_flags_combine_with_zero_sentinels():
    d = D.decode_history_record([NAN, INF, 1, 0, 0, 1, 0, 1, NAN, 2, -INF, 0, NAN, 4, 5, 6,
                                 7, INF, 1, NAN, NAN, 0.5, 0, 0, 0, 1, 0, NAN, 0, 0, 0, 1])
    for key in ("sourceGeometryValid", "candidateGeometryValid", "acceptedMinimumDeformationDeterminantValid",
                "localNumericsValid", "geometryValid", "energyValid", "componentGradientNormsValid",
                "residualDiagnosticsValid", "updateDiagnosticsValid", "maximumLocalNormalizedShiftValid", "finite"):
        assert d[key] is False, key
    scalars = [d["sourceMinimumDeformationDeterminant"], d["candidateMinimumDeformationDeterminant"],
               d["sourceEnergy"], d["acceptedEnergy"], *d["componentGradientNorms"].values(), d["gradientNorm"],
               d["relativeResidual"], d["maximumUpdate"], d["maximumLocalNormalizedShift"]]
    assert all(math.isfinite(x) for x in scalars)
    assert d["sourceMinimumDeformationDeterminant"] == 0 and d["componentGradientNorms"]["inertia"] == 0


def test_reverted_source_minimum_survives_a_nonfinite_candidate():
    packed = np.zeros(32, dtype=np.float32)
    packed[[0, 2]] = 0.5
    packed[3] = 1 | 4 | 8
    packed[[5, 7, 18, 25, 31]] = 1
    d = D.decode_history_record(packed)
    assert d["sourceGeometryValid"] and not d["candidateGeometryValid"]
    assert d["acceptedMinimumDeformationDeterminant"] == 0.5 and d["acceptedMinimumDeformationDeterminantValid"]
    assert d["localNumericsValid"] and not d["geometryValid"] and not d["finite"]


def test_finite_infeasible_geometry_versus_invalid_local_numerics():
    packed = np.zeros(32, dtype=np.float32)
    packed[[0, 1, 2, 3]] = [0.5, -0.25, 0.5, 15]
    packed[[5, 7, 18, 25, 31]] = 1
    d = D.decode_history_record(packed)
    assert d["geometryValid"] and d["assembledReverted"] and d["finite"]
    packed[3] = 15 & ~8
    d = D.decode_history_record(packed)
    assert d["geometryValid"] and not d["localNumericsValid"] and not d["finite"]


def test_bounded_history_sequences():
    record = np.zeros(32, dtype=np.float32)
    record[3] = 15
    record[[11, 18, 25, 31]] = 1
    packed = np.concatenate([record, record])
    packed[32 + 26] = 1
    records = D.decode_history(packed)
    assert [r["iterationIndex"] for r in records] == [0, 1]
    assert isinstance(records, tuple)
    with pytest.raises(JGS2RangeError, match="complete 32-float records"):
        D.decode_history(np.zeros(31))
    with pytest.raises(JGS2RangeError, match="no more than 64 records"):
        D.decode_history(np.zeros(65 * 32))


def test_rejects_malformed_history_records():
    with pytest.raises(JGS2RangeError, match="expected exactly 32"):
        D.decode_history_record(np.zeros(31))
    cases = [(6, 0.5, "localFailureCount"), (7, 2, "revertCount"), (26, 64, "iterationIndex"),
             (3, 16, "geometryValidityBits"), (3, 0.5, "geometryValidityBits"), (3, -1, "geometryValidityBits"),
             (28, 13, "maximumBacktrackCount")]
    for lane, value, label in cases:
        packed = np.zeros(32)
        packed[lane] = value
        with pytest.raises(JGS2RangeError, match=f"{label} must be a nonnegative integer"):
            D.decode_history_record(packed)


def test_decode_globalization_of_a_raw_read():
    local = np.zeros((3, 16), dtype=np.float32)
    local[:, 5] = 1
    local[1, 15] = 1  # pinned
    history = np.zeros((2, 32), dtype=np.float32)
    history[:, 3] = 15
    history[:, [11, 18, 25, 31]] = 1
    history[1, 26] = 1
    out = D.decode_globalization({"local": local, "control": np.zeros(16), "history": history, "historyCount": 2})
    assert [r["status"] for r in out["local"]] == ["accepted", "pinned", "accepted"]
    assert out["historyCount"] == 2 and [r["iterationIndex"] for r in out["history"]] == [0, 1]
    with pytest.raises(JGS2RangeError, match="invalid globalization history count"):
        D.decode_globalization({"local": local, "control": np.zeros(16), "history": history, "historyCount": 65})


def test_oracle_records_decode_under_the_reference_rules():
    # The oracle writes the step's records in the layout the GPU writes
    # (the GPU parity tests compare them); a few production frames of a bar
    # decode without a range error and with consistent flags.
    from jgs2_b200 import scenes
    from oracle import oracle as O

    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4)
    sc.add_cuboid((6, 2, 2), (0.0, 0.0, 0.0), (0.3, 0.1, 0.1), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    inp = sc.pack()
    cpu = O.OracleSolver(inp, dict(timestep=1 / 60, gravity=(0.0, -9.8, 0.0), iterations=6), precision=32)
    cpu.step_frames(3)
    control = cpu.read("control")
    count = int(control[7])
    out = D.decode_globalization({"local": cpu.read("local").reshape(-1, 16), "control": control,
                                  "history": cpu.read("history").reshape(64, 32), "historyCount": count})
    # Production steps round an even iteration count up to the next odd one.
    assert 0 < count <= O.normalize_odd_iterations(6) and out["historyCount"] == count
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    assert all(r["status"] == "pinned" for r, p in zip(out["local"], pinned) if p)
    assert all(r["finite"] for r, p in zip(out["local"], pinned) if not p)
    for i, h in enumerate(out["history"]):
        assert h["iterationIndex"] == i and h["active"] and h["finite"]
        assert h["assembledAccepted"] != h["assembledReverted"]
        assert h["revertCount"] == int(h["assembledReverted"])


def test_diagnostic_relative_error_is_symmetric_and_scale_safe():
    # jgs2-diagnostics.test.ts:369-384.
    assert D.relative_error([1, 2], [1, 1]) == pytest.approx(1 / math.sqrt(5), abs=1e-12)
    assert D.relative_error([3, 4], [0, 0]) == 1.0
    assert D.relative_error([0, 0], [0, 0]) == 0.0
    assert D.relative_error([1, 1], [1, 2]) == D.relative_error([1, 2], [1, 1])
    with pytest.raises(JGS2RangeError, match="matching lengths"):
        D.relative_error([1], [1, 2])

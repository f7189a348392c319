"""Decoders for the step's globalization records, the reference's
src/simulation/gpu/jgs2-globalization.ts:1-560.

`JGS2GpuSolver.readGlobalizationDiagnostics()` returns the raw float
records, as the C-ABI (`jgs2_read_globalization`) delivers them:
- per vertex, a 4-vec4 local record;
- the 4-vec4 control record;
- up to 64 history records of 8 vec4 each.

`decode_globalization` turns that result into the reference's decoded form:
`{"local": [...], "history": [...], "historyCount": n}`, with the
reference's field names. The per-record decoders follow the reference's
rules:
- non-finite (or negative, for nonnegative fields) lanes become finite
  zero sentinels with a matching validity flag;
- counts, flags and status codes must be exact integers in range, or a
  JGS2RangeError (the reference's RangeError) is raised with the
  reference's wording.
"""
from __future__ import annotations

import math
from typing import Sequence

from .solver import JGS2RangeError

HISTORY_CAPACITY = 64
LOCAL_DIAGNOSTIC_VEC4S = 4
CONTROL_VEC4S = 4
HISTORY_VEC4S = 8

RELATIVE_EIGENVALUE_FLOOR = 2.0 ** -16
MAX_NORMALIZED_SHIFT = 1e-3
DETERMINANT_FLOOR = 1e-4
ARMIJO_C1 = 1e-4
BACKTRACK_FACTOR = 0.5
MAX_BACKTRACKS = 12

SOURCE_GEOMETRY_VALID_BIT = 1
CANDIDATE_GEOMETRY_VALID_BIT = 2
ACCEPTED_MINIMUM_VALID_BIT = 4
LOCAL_NUMERICS_VALID_BIT = 8
VALIDITY_BITS_MASK = 15

LOCAL_STATUS_CODES = {"accepted": 0, "pinned": 1, "zeroGradient": 2, "shiftLimit": 3, "nonDescent": 4,
                      "lineSearchFailed": 5, "nonfinite": 6, "choleskyFailed": 7}
LOCAL_STATUS_NAMES = ("accepted", "pinned", "zero-gradient", "shift-limit", "non-descent", "line-search-failed",
                      "nonfinite", "cholesky-failed")
STATUS_ACCEPTED, STATUS_LINE_SEARCH_FAILED, STATUS_NONFINITE, STATUS_CHOLESKY_FAILED = 0, 5, 6, 7

_LOCAL_FLOATS = 4 * LOCAL_DIAGNOSTIC_VEC4S
_HISTORY_FLOATS = 4 * HISTORY_VEC4S
_MAX_SAFE_INTEGER = 2 ** 53 - 1


def _range_error(message: str):
    return JGS2RangeError(1, message)


def _exact_length(packed: Sequence[float], expected: int, label: str):
    if len(packed) != expected:
        raise _range_error(f"{label} contains {len(packed)} floats; expected exactly {expected}.")


def _finite_or_zero(value: float):
    value = float(value)
    return (value, True) if math.isfinite(value) else (0.0, False)


def _finite_nonnegative_or_zero(value: float):
    value = float(value)
    return (value, True) if math.isfinite(value) and value >= 0 else (0.0, False)


def _flag(value: float, label: str) -> bool:
    value = float(value)
    if value not in (0.0, 1.0):
        raise _range_error(f"{label} must be encoded as exactly 0 or 1.")
    return value == 1.0


def _count(value: float, label: str, maximum: int = _MAX_SAFE_INTEGER) -> int:
    value = float(value)
    if not (math.isfinite(value) and value == math.floor(value) and abs(value) <= _MAX_SAFE_INTEGER) \
            or value < 0 or value > maximum:
        raise _range_error(f"{label} must be a nonnegative integer no greater than {maximum}.")
    return int(value)


def _status(value: float) -> int:
    value = float(value)
    if not (math.isfinite(value) and value == math.floor(value)) or value < STATUS_ACCEPTED \
            or value > STATUS_CHOLESKY_FAILED:
        raise _range_error(f"Local globalization status must be an integer from {STATUS_ACCEPTED} through "
                           f"{STATUS_CHOLESKY_FAILED}.")
    return int(value)


def decode_local_diagnostic(packed: Sequence[float]) -> dict:
    """decodeJGS2GlobalizationLocalDiagnostic (jgs2-globalization.ts:237-340):
    one 16-float local record."""
    _exact_length(packed, _LOCAL_FLOATS, "Local globalization diagnostic")
    direction = [_finite_or_zero(packed[i]) for i in range(3)]
    alpha = _finite_nonnegative_or_zero(packed[3])
    min_eig = _finite_or_zero(packed[4])
    scale = _finite_nonnegative_or_zero(packed[5])
    shift = _finite_nonnegative_or_zero(packed[6])
    normalized_shift = _finite_nonnegative_or_zero(packed[7])
    energy_delta = _finite_or_zero(packed[8])
    armijo_bound = _finite_or_zero(packed[9])
    gdd = _finite_or_zero(packed[10])
    residual = _finite_nonnegative_or_zero(packed[11])
    min_trial_det = _finite_or_zero(packed[12])
    backtracks = _count(packed[13], "Local globalization backtrackCount", MAX_BACKTRACKS)
    evaluations = _count(packed[14], "Local globalization energyEvaluationCount")
    code = _status(packed[15])
    # A zero determinant is a sentinel unless the status says the trial
    # geometry was evaluated (accepted, a failed search, or a non-finite
    # energy after feasible geometry).
    geometry_before_nonfinite_energy = code == STATUS_NONFINITE and min_trial_det[0] > DETERMINANT_FLOOR
    geometry_evaluated = code in (STATUS_ACCEPTED, STATUS_LINE_SEARCH_FAILED) or geometry_before_nonfinite_energy
    direction_valid = all(v for _, v in direction)
    pd_valid = all(v for _, v in (min_eig, scale, shift, normalized_shift))
    energy_valid = all(v for _, v in (energy_delta, armijo_bound, gdd, residual))
    finite = (direction_valid and alpha[1] and pd_valid and energy_valid and min_trial_det[1]
              and code != STATUS_NONFINITE)
    return {
        "direction": [d for d, _ in direction],
        "alpha": alpha[0],
        "minimumEigenvalue": min_eig[0],
        "scale": scale[0],
        "diagonalShift": shift[0],
        "normalizedShift": normalized_shift[0],
        "acceptedEnergyDelta": energy_delta[0],
        "armijoDeltaBound": armijo_bound[0],
        "gradientDotDirection": gdd[0],
        "shiftedLinearResidual": residual[0],
        "minimumTrialDeformationDeterminant": min_trial_det[0],
        "backtrackCount": backtracks,
        "energyEvaluationCount": evaluations,
        "statusCode": code,
        "status": LOCAL_STATUS_NAMES[code],
        "accepted": code == STATUS_ACCEPTED,
        "directionValid": direction_valid,
        "alphaValid": alpha[1],
        "positiveDefiniteDiagnosticsValid": pd_valid,
        "energyDiagnosticsValid": energy_valid,
        "minimumTrialDeformationDeterminantValid": min_trial_det[1] and geometry_evaluated,
        "finite": finite,
    }


def decode_history_record(packed: Sequence[float]) -> dict:
    """decodeJGS2GlobalizationHistoryRecord (jgs2-globalization.ts:342-510):
    one 32-float convergence-history record."""
    _exact_length(packed, _HISTORY_FLOATS, "Globalization history record")
    src_min, cand_min, acc_min = (_finite_or_zero(packed[i]) for i in range(3))
    bits = _count(packed[3], "geometryValidityBits", VALIDITY_BITS_MASK)
    assembled_accepted = _flag(packed[4], "assembledAccepted")
    assembled_reverted = _flag(packed[5], "assembledReverted")
    failures = _count(packed[6], "localFailureCount")
    reverts = _count(packed[7], "revertCount", 1)
    src_e, cand_e, acc_e = (_finite_or_zero(packed[i]) for i in (8, 9, 10))
    packed_energy_valid = _flag(packed[11], "energyValid")
    norms = [_finite_nonnegative_or_zero(packed[i]) for i in range(12, 17)]
    gnorm, den, rel = (_finite_nonnegative_or_zero(packed[i]) for i in (17, 18, 19))
    max_update, norm_update = (_finite_nonnegative_or_zero(packed[i]) for i in (20, 21))
    residual_ok = _flag(packed[22], "residualSatisfied")
    update_ok = _flag(packed[23], "updateSatisfied")
    converged = _flag(packed[24], "converged")
    packed_finite = _flag(packed[25], "finite")
    index = _count(packed[26], "iterationIndex", HISTORY_CAPACITY - 1)
    max_shift = _finite_nonnegative_or_zero(packed[27])
    max_backtracks = _count(packed[28], "maximumBacktrackCount", MAX_BACKTRACKS)
    infeasible = _count(packed[29], "infeasibleTrialCount")
    evaluations = _count(packed[30], "energyEvaluationCount")
    active = _flag(packed[31], "active")

    source_valid = bool(bits & SOURCE_GEOMETRY_VALID_BIT) and src_min[1]
    candidate_valid = bool(bits & CANDIDATE_GEOMETRY_VALID_BIT) and cand_min[1]
    accepted_valid = bool(bits & ACCEPTED_MINIMUM_VALID_BIT) and acc_min[1]
    local_valid = bool(bits & LOCAL_NUMERICS_VALID_BIT)
    norms_valid = all(v for _, v in norms)
    residual_valid = all(v for _, v in (gnorm, den, rel))
    update_valid = all(v for _, v in (max_update, norm_update))
    all_numerics = (all(v for _, v in (src_min, cand_min, acc_min)) and all(v for _, v in (src_e, cand_e, acc_e))
                    and norms_valid and residual_valid and update_valid and max_shift[1])
    names = ("inertia", "material", "externalForce", "target", "contact")
    return {
        "sourceMinimumDeformationDeterminant": src_min[0],
        "candidateMinimumDeformationDeterminant": cand_min[0],
        "acceptedMinimumDeformationDeterminant": acc_min[0],
        "sourceGeometryValid": source_valid,
        "candidateGeometryValid": candidate_valid,
        "acceptedMinimumDeformationDeterminantValid": accepted_valid,
        "localNumericsValid": local_valid,
        "geometryValid": source_valid and candidate_valid,
        "assembledAccepted": assembled_accepted,
        "assembledReverted": assembled_reverted,
        "localFailureCount": failures,
        "revertCount": reverts,
        "sourceEnergy": src_e[0],
        "candidateEnergy": cand_e[0],
        "acceptedEnergy": acc_e[0],
        "energyValid": packed_energy_valid and all(v for _, v in (src_e, cand_e, acc_e)),
        "componentGradientNorms": {n: v for n, (v, _) in zip(names, norms)},
        "componentGradientNormsValid": norms_valid,
        "gradientNorm": gnorm[0],
        "residualDenominator": den[0],
        "relativeResidual": rel[0],
        "residualDiagnosticsValid": residual_valid,
        "maximumUpdate": max_update[0],
        "normalizedMaximumUpdate": norm_update[0],
        "updateDiagnosticsValid": update_valid,
        "residualSatisfied": residual_ok,
        "updateSatisfied": update_ok,
        "converged": converged,
        "finite": packed_finite and all_numerics and source_valid and candidate_valid and accepted_valid
        and local_valid,
        "iterationIndex": index,
        "maximumLocalNormalizedShift": max_shift[0],
        "maximumLocalNormalizedShiftValid": max_shift[1],
        "maximumBacktrackCount": max_backtracks,
        "infeasibleTrialCount": infeasible,
        "energyEvaluationCount": evaluations,
        "active": active,
    }


def decode_history(packed: Sequence[float]) -> tuple:
    """decodeJGS2GlobalizationHistory (jgs2-globalization.ts:517-560): a
    tightly packed run of complete records, at most the capacity."""
    if len(packed) % _HISTORY_FLOATS != 0 or len(packed) > HISTORY_CAPACITY * _HISTORY_FLOATS:
        raise _range_error(f"Globalization history must contain complete {_HISTORY_FLOATS}-float records and no "
                           f"more than {HISTORY_CAPACITY} records.")
    return tuple(decode_history_record(packed[o:o + _HISTORY_FLOATS]) for o in range(0, len(packed), _HISTORY_FLOATS))


def decode_globalization(raw: dict) -> dict:
    """The reference's readGlobalizationDiagnostics result
    (jgs2-solver.ts:2548-2604) from JGS2GpuSolver.readGlobalizationDiagnostics():
    every vertex's decoded local record and the executed history records."""
    count = raw["historyCount"]
    if not (isinstance(count, int) and 0 <= count <= HISTORY_CAPACITY):
        raise _range_error(f"GPU returned invalid globalization history count {count}.")
    local = [decode_local_diagnostic(list(map(float, rec))) for rec in raw["local"]]
    history = decode_history([float(x) for rec in raw["history"][:count] for x in rec])
    return {"local": local, "history": list(history), "historyCount": count}


def relative_error(actual: Sequence[float], reference: Sequence[float]) -> float:
    """jgs2DiagnosticRelativeError (src/simulation/gpu/jgs2-diagnostics.ts:
    296-317): |a - b| / max(1, |a|, |b|) over two equal-length vectors,
    symmetric and safe at zero. Vectors of different lengths raise
    JGS2RangeError."""
    if len(actual) != len(reference):
        raise _range_error("Diagnostic vectors must have matching lengths.")
    diff = act = ref = 0.0
    for a, b in zip(actual, reference):
        diff += (float(a) - float(b)) ** 2
        act += float(a) ** 2
        ref += float(b) ** 2
    return math.sqrt(diff) / max(1.0, math.sqrt(act), math.sqrt(ref))

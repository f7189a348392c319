"""The globalization policy constants and status codes, frozen as the
reference freezes them (src/simulation/gpu/jgs2-globalization-wgsl.test.ts:
42-104; values from src/simulation/gpu/jgs2-globalization.ts:2-46):

- position resolution multiplier 8, relative eigenvalue floor 2^-16,
  maximum normalised shift 1e-3, Armijo c1 1e-4, backtrack factor 0.5,
  determinant floor 1e-4, 12 backtracks and 13 trials, history capacity 64;
- local statuses accepted 0, pinned 1, zero gradient 2, shift limit 3,
  non-descent 4, line search failed 5, non-finite 6, Cholesky failed 7,
  distinct;
- validity bits source geometry 1, candidate geometry 2, accepted minimum 4,
  local numerics 8.

The device header, the oracle and the host decoder each hold a copy. The
test reads each copy from its source, as the reference's test reads its WGSL
source, and checks them against these values and against one another.
"""
import os
import re

import pytest

from jgs2_b200 import diagnostics

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEVICE = os.path.join(ROOT, "webgpu-physics_b200", "csrc", "jgs2_device.cuh")
ORACLE = os.path.join(ROOT, "oracle", "jgs2_oracle.cpp")
HEADER = os.path.join(ROOT, "include", "jgs2.h")

POLICY = {
    "kPositionResolutionMultiplier": 8.0,
    "kRelativeEigenvalueFloor": 2.0 ** -16,
    "kMaxNormalizedShift": 1e-3,
    "kArmijoC1": 1e-4,
    "kBacktrackFactor": 0.5,
    "kDeterminantFloor": 1e-4,
    "kMaxBacktracks": 12,
}
STATUS = {"Accepted": 0, "Pinned": 1, "ZeroGradient": 2, "ShiftLimit": 3, "NonDescent": 4,
          "LineSearchFailed": 5, "Nonfinite": 6, "CholeskyFailed": 7}
VALIDITY = {"kSourceGeometryValid": 1, "kCandidateGeometryValid": 2, "kAcceptedMinimumValid": 4,
            "kLocalNumericsValid": 8}


def _constants(path):
    text = open(path).read()
    found = {}
    for name, value in re.findall(r"constexpr\s+(?:float|double|uint32_t)\s+(k\w+)\s*=\s*([0-9.eE+-]+)u?f?\s*;",
                                  text):
        found[name] = float(value)
    return found


def _enum_values(path, prefix):
    text = open(path).read()
    return {name[len(prefix):]: int(value) for name, value in re.findall(rf"\b({prefix}\w+)\s*=\s*(\d+)u?", text)}


@pytest.mark.parametrize("path", [DEVICE, ORACLE])
def test_policy_constants_match_the_reference(path):
    found = _constants(path)
    for name, value in POLICY.items():
        assert name in found, f"{os.path.basename(path)} lacks {name}"
        # The f32 literal of each value, as the WGSL library writes it.
        assert found[name] == pytest.approx(value, rel=1e-7), name


def test_trial_count_and_history_capacity():
    device = _constants(DEVICE)
    assert device["kTrialCount"] == POLICY["kMaxBacktracks"] + 1
    assert device["kHistoryCapacity"] == 64
    assert re.search(r"#define\s+JGS2_HISTORY_CAPACITY\s+64u", open(HEADER).read())


def test_local_status_codes_are_stable_and_distinct():
    device = _enum_values(DEVICE, "k")
    oracle = _enum_values(ORACLE, "kStatus")
    for name, code in STATUS.items():
        assert device[name] == code, f"device {name}"
        assert oracle[name] == code, f"oracle {name}"
    assert len(set(STATUS.values())) == len(STATUS)
    assert diagnostics.LOCAL_STATUS_CODES == {name[0].lower() + name[1:]: code for name, code in STATUS.items()}


def test_validity_bits_do_not_overlap():
    device = _enum_values(DEVICE, "")
    bits = [device[name] for name in VALIDITY]
    assert bits == list(VALIDITY.values())
    assert device["kValidityMask"] == sum(bits)

"""The cubature trainer's greedy nonnegative column selection against the
reference's own cases (src/simulation/cpu/cubature.test.ts:33-160), through
jgs2_select_nonnegative_columns (the CPU trainer's selection core, which the
GPU selection matches bit for bit)."""
import math

import pytest

from jgs2_b200 import scenes
from jgs2_b200.solver import JGS2RangeError

select = scenes.select_nonnegative_columns


def test_selects_an_exact_deterministic_nonnegative_representation():
    r = select([[1, 0, 0], [0, 1, 0], [0, 0, 1]], [2, 3, 0], 2)
    assert r["selected"] == [1, 0]
    assert r["weights"] == [3, 2]
    assert r["normalizedResidual"] == 0


def test_exact_ties_take_the_original_order_and_zero_columns_are_ignored():
    cols = [[0, 0], [1, 0], [1, 0]]
    first, second = select(cols, [1, 0], 1), select(cols, [1, 0], 1)
    assert first["selected"] == [1] == second["selected"]
    assert first["weights"] == [1] and first["normalizedResidual"] == 0


def test_reports_the_residual_of_a_sample_budget():
    r = select([[1, 0], [0, 1]], [1, 1], 1)
    assert r["selected"] == [0] and r["weights"] == [1]
    assert abs(r["normalizedResidual"] - 1 / math.sqrt(2)) < 1e-14


def test_uses_the_configured_stopping_tolerance():
    loose = select([[1, 0], [0, 1]], [1, 1], 2, refinement_passes=0, residual_tolerance=0.8)
    exact = select([[1, 0], [0, 1]], [1, 1], 2, refinement_passes=0, residual_tolerance=0)
    assert loose["selected"] == [0] and abs(loose["normalizedResidual"] - 1 / math.sqrt(2)) < 1e-14
    assert exact["selected"] == [0, 1] and exact["normalizedResidual"] == 0


def test_never_introduces_a_negative_weight():
    r = select([[-1, 0], [0, 1]], [1, 1], 2)
    assert r["selected"] == [1] and r["weights"] == [1]
    assert abs(r["normalizedResidual"] - 1 / math.sqrt(2)) < 1e-14


def test_zero_target_and_missing_candidates():
    zero = select([[1, 0]], [0, 0], 1)
    assert zero["selected"] == [] and zero["normalizedResidual"] == 0
    none = select([], [2, -1], 4)
    assert none["selected"] == [] and none["normalizedResidual"] == 1


def test_rejects_malformed_input():
    with pytest.raises(JGS2RangeError):
        select([[1, 0]], [1, 0], 13)  # more than the 12 columns the exhaustive fit takes
    with pytest.raises(JGS2RangeError):
        select([[math.nan, 0]], [1, 0], 1)
    with pytest.raises(JGS2RangeError):
        select([[1, 0]], [1, 0], 1, residual_tolerance=1.5)


def test_linear_training_is_bounded_and_nonnegative():
    # precompute.test.ts:580-606 on a co-rotated (linear) bar trained with
    # K = 6: at most K records per vertex, nonnegative weights, a raw
    # gradient residual below 0.3, and some record incident to its source.
    import numpy as np

    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e5, 0.4, scenes.MATERIAL_COROTATED_LINEAR)
    sc.add_cuboid((6, 2, 2), (0.0, 0.0, 0.0), (0.6, 0.2, 0.2), m, 0, scenes.FACE_X_MIN)
    stats = sc.precompute(timestep=1 / 60, cubature_k=6)
    inp = sc.pack()
    K = inp.cubature_k
    assert K <= 6
    ids = inp.cubature_tet_ids.reshape(-1, K)
    w = inp.cubature_weights.reshape(-1, K)
    assert (w >= 0).all()
    tets = inp.tet_indices.reshape(-1, 4)
    incident = any(v in tets[t] for v in range(inp.vertex_count) for t in ids[v] if t != scenes.EMPTY_TET)
    assert incident
    assert stats["max_residual"] < 0.3
    print(f"linear training: max residual {stats['max_residual']:.4f}, "
          f"records per vertex <= {int((w > 0).sum(axis=1).max())}")
    assert np.isfinite(inp.cubature_basis).all()

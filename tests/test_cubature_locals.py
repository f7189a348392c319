"""Local globalization invariants on the trained nonlinear cubature fixture:
the per-local checks of the reference's production cubature test
(tests/e2e/nonlinear-cubature-gpu.spec.ts:440-528), run on the oracle.

The fixture is the reference's 12-tet nonlinear cubature definition
(src/scenes/phase1.ts:287-319): a 2x1x1-hex unit bar, E 5000, nu 0.3, an edge
pinned, six trained samples per vertex. It has 10 active locals. The
reference's frozen pose corpus is replaced by seeded poses: every free
vertex displaced by up to 4 cm, with the inertial target at the rest shape.
Two exact iterations run from each pose.

After each iteration, every active local record must be finite, with:
- scale > 0, diagonal shift >= 0, normalised shift <= 1e-3, and shifted
  linear residual < 2e-5;
- if accepted: a nonzero direction, 0 < alpha <= 1, g.d < 0, accepted energy
  delta <= its Armijo bound, and minimum trial determinant > 1e-4;
- otherwise zero-gradient, with alpha, the energy delta and the Armijo bound
  all zero.

Each assembled candidate must be accepted and not reverted, with no local
failure.
"""
import numpy as np
import pytest

from jgs2_b200 import diagnostics, scenes
from oracle import oracle as O

H = 1 / 60
SETTINGS = dict(timestep=H, gravity=(0.0, 0.0, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=2)


def _fixture():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 5000.0, 0.3)
    sc.add_cuboid((2, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), m, 0, 0)
    rest = sc.rest_positions()
    sc.set_pinned((np.isclose(rest[:, 0], 0) & np.isclose(rest[:, 1], 0)).astype(np.uint8))
    stats = sc.precompute(timestep=H, cubature_k=6)
    assert stats["max_residual"] <= 0.01
    return sc, rest.astype(np.float64)


def _posed(sc, rest, seed):
    free = sc.pack().vertex_info.reshape(-1, 4)[:, 2] == 0
    rng = np.random.default_rng(seed)
    x = rest.copy()
    x[free] += rng.uniform(-0.04, 0.04, size=(int(free.sum()), 3))
    pos = np.ones((rest.shape[0], 4), dtype=np.float32)
    pos[:, :3] = x
    vel = np.zeros((rest.shape[0], 4), dtype=np.float32)
    vel[:, :3] = (rest - pos[:, :3].astype(np.float64)) / H
    sc.set_initial_state(pos.reshape(-1), vel.reshape(-1), pin_at_initial=False)
    return sc.pack(), free


def _check_locals(locals_, free):
    active = [diagnostics.decode_local_diagnostic(locals_[16 * v:16 * v + 16]) for v in np.flatnonzero(free)]
    assert len(active) == 10
    for k, d in enumerate(active):
        label = f"local {k}: {d}"
        assert d["finite"], label
        assert np.isfinite(d["minimumEigenvalue"]), label
        assert d["scale"] > 0 and d["diagonalShift"] >= 0, label
        assert 0 <= d["normalizedShift"] <= 1e-3, label
        assert d["shiftedLinearResidual"] < 2e-5, label
        if d["status"] == "accepted":
            assert np.linalg.norm(d["direction"]) > 0, label
            assert 0 < d["alpha"] <= 1, label
            assert d["gradientDotDirection"] < 0, label
            assert d["acceptedEnergyDelta"] <= d["armijoDeltaBound"], label
            assert d["minimumTrialDeformationDeterminant"] > 1e-4, label
        else:
            assert d["status"] == "zero-gradient", label
            assert d["alpha"] == 0 and d["acceptedEnergyDelta"] == 0 and d["armijoDeltaBound"] == 0, label
    return sum(d["status"] == "accepted" for d in active)


@pytest.mark.parametrize("precision", [32, 64])
def test_trained_cubature_locals_meet_the_reference_invariants(precision):
    sc, rest = _fixture()
    accepted = 0
    for seed in range(3):
        inp, free = _posed(sc, rest, seed)
        for iterations in (1, 2):
            o = O.OracleSolver(inp, dict(SETTINGS, iterations=iterations), precision=precision)
            o.step_exact_iterations(iterations)
            accepted += _check_locals(o.read("local"), free)
            history = diagnostics.decode_history(o.read("history")[:32 * iterations])
            assert len(history) == iterations
            for rec in history:
                assert rec["finite"] and rec["assembledAccepted"] and not rec["assembledReverted"], rec
                assert rec["localFailureCount"] == 0, rec
                assert rec["maximumLocalNormalizedShift"] <= 1e-3
                assert rec["acceptedMinimumDeformationDeterminant"] > 1e-4
    # The poses are far from equilibrium: most locals take a step.
    print(f"f{precision}: {accepted} accepted locals of {3 * 2 * 10}")
    assert accepted >= 30

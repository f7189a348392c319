"""The step's convergence reduction (the oracle's reduceConvergence) on the
reference's synthetic cases (src/simulation/cpu/nonlinear-iteration.test.ts:
181-400). The relative residual is |sum of components| / max(1, sum of
component norms), and the normalised update is max update / max(scene
scale, 1e-12). Convergence needs both gates, an assembled accept, no revert,
no local failure and finite diagnostics."""
import ctypes
import math

import numpy as np
import pytest

from jgs2_b200 import scenes
from oracle import oracle as O

# History record lanes (jgs2-globalization.ts:342-510).
DEN, REL, MAX_UPDATE, NORM_UPDATE, RES_OK, UPD_OK, CONVERGED, FINITE = 18, 19, 20, 21, 22, 23, 24, 25
INERTIA_NORM, MATERIAL_NORM = 12, 13


def _reduce(components, update, scene_scale, residual_tol, update_tol, feasible=True, accepted=True,
            reverted=False, failures=0, precision=64):
    inp = scenes.single_tetrahedron()
    L = O.lib()
    F = ctypes.POINTER(ctypes.c_float)
    L.jgs2_oracle_reduce_convergence.argtypes = [ctypes.c_void_p, ctypes.c_void_p, F, F, F, ctypes.c_double, F]
    settings = dict(residual_tolerance=residual_tol, normalized_update_tolerance=update_tol)
    o = O.OracleSolver(inp, settings, precision=precision)
    comp = np.zeros((inp.vertex_count, 5, 4), dtype=np.float32)
    for c, g in enumerate(components):
        comp[0, c, :3] = g
    upd = np.zeros(inp.vertex_count, dtype=np.float32)
    upd[0] = update
    control = np.zeros(16, dtype=np.float32)
    control[:4] = [1.0, 1.0, 1.0, 15.0 if feasible else 0.0]
    control[4:8] = [1.0 if accepted else 0.0, 1.0 if reverted else 0.0, float(failures), 0.0]
    out = np.zeros(32, dtype=np.float32)
    rec = O._settings_struct(O.resolve_settings(None, **settings))
    L.jgs2_oracle_reduce_convergence(o._h, ctypes.byref(rec), comp.ctypes.data_as(F), upd.ctypes.data_as(F),
                                     control.ctypes.data_as(F), float(scene_scale), out.ctypes.data_as(F))
    return out


def _zero():
    return [(0.0, 0.0, 0.0)] * 5


@pytest.mark.parametrize("precision", [64, 32])
def test_both_gates_are_required(precision):
    base = _zero()
    base[0], base[1] = (1.0, 0.0, 0.0), (-1.0, 0.0, 0.0)
    conv = _reduce(base, 1e-5, 2.0, 1e-6, 1e-4, precision=precision)
    assert conv[DEN] == 2.0 and conv[REL] == 0.0 and conv[CONVERGED] == 1.0
    high_update = _reduce(base, 1e-3, 2.0, 1e-6, 1e-4, precision=precision)
    assert (high_update[RES_OK], high_update[UPD_OK], high_update[CONVERGED]) == (1.0, 0.0, 0.0)
    high_residual = list(base)
    high_residual[1] = (-0.5, 0.0, 0.0)
    hr = _reduce(high_residual, 0.0, 2.0, 1e-6, 1e-4, precision=precision)
    assert (hr[RES_OK], hr[UPD_OK], hr[CONVERGED]) == (0.0, 1.0, 0.0)


@pytest.mark.parametrize("precision", [64, 32])
def test_invalid_diagnostics_stay_finite_and_failures_block_convergence(precision):
    bad = _zero()
    bad[0] = (math.nan, 0.0, 0.0)
    r = _reduce(bad, 0.0, 1.0, 1e-5, 1e-5, feasible=False, failures=1, precision=precision)
    assert r[FINITE] == 0.0 and r[CONVERGED] == 0.0
    assert np.isfinite(r).all()
    ok = _zero()
    r = _reduce(ok, 0.0, 1.0, 1e-5, 1e-5, failures=1, precision=precision)
    assert r[FINITE] == 1.0 and r[CONVERGED] == 0.0


@pytest.mark.parametrize("precision", [64, 32])
def test_update_normalised_by_the_scene_scale_floor(precision):
    r = _reduce(_zero(), 5e-16, 0.0, 1e-5, 1e-3, precision=precision)
    assert abs(r[NORM_UPDATE] - 5e-4) < 1e-9
    assert r[CONVERGED] == 1.0


@pytest.mark.parametrize("precision", [64, 32])
def test_an_assembled_revert_cannot_converge(precision):
    r = _reduce(_zero(), 0.0, 1.0, 1e-5, 1e-5, accepted=False, reverted=True, precision=precision)
    assert r[RES_OK] == 1.0 and r[UPD_OK] == 1.0 and r[CONVERGED] == 0.0


@pytest.mark.parametrize("precision", [64, 32])
def test_large_representable_norms_stay_valid(precision):
    # Components whose squares overflow f32 still give finite scaled norms.
    big = _zero()
    big[0], big[1] = (3e20, 0.0, 0.0), (-3e20, 0.0, 0.0)
    r = _reduce(big, 0.0, 1.0, 1e-5, 1e-5, precision=precision)
    assert r[FINITE] == 1.0 and r[CONVERGED] == 1.0
    assert abs(r[INERTIA_NORM] / 3e20 - 1) < 1e-6 and abs(r[MATERIAL_NORM] / 3e20 - 1) < 1e-6

"""The oracle's local globalization solve pinned to the reference's
globalization tests (src/simulation/cpu/nonlinear-globalization.test.ts:
38-158). The solve normalises the symmetric system by
max(inertia, largest diagonal, Frobenius / sqrt 3), shifts its diagonal up to
the relative eigenvalue floor 2^-16, refuses shifts above 1e-3, and solves
by Cholesky. With inertia 1 and entries at most one the normalisation is the
identity, so the reference's raw-matrix answers apply directly. The
constants are those of jgs2-globalization-wgsl.ts:29-36.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

EIGENVALUE_FLOOR = 2.0 ** -16
MAX_SHIFT = 1e-3
ACCEPTED, SHIFT_LIMIT = 0, 3


def _lib():
    L = O.lib()
    D = ctypes.POINTER(ctypes.c_double)
    L.jgs2_oracle_local_solve.argtypes = [D, D, ctypes.c_double, ctypes.c_int, D]
    L.jgs2_oracle_local_solve.restype = ctypes.c_int
    L.jgs2_oracle_min_symmetric_eigenvalue.argtypes = [D, ctypes.c_int]
    L.jgs2_oracle_min_symmetric_eigenvalue.restype = ctypes.c_double
    return L


def _solve(hessian, gradient, inertia=1.0, precision=64):
    D = ctypes.POINTER(ctypes.c_double)
    h = np.ascontiguousarray(hessian, dtype=np.float64).reshape(9)
    g = np.ascontiguousarray(gradient, dtype=np.float64)
    out = np.zeros(10)
    assert _lib().jgs2_oracle_local_solve(h.ctypes.data_as(D), g.ctypes.data_as(D), inertia, precision,
                                          out.ctypes.data_as(D)) == 0
    return dict(status=int(out[0]), direction=out[1:4].copy(), gdd=out[4], scale=out[5], min_eig=out[6],
                shift=out[7], asym=out[8], residual=out[9])


def _min_eig(m, precision=64):
    D = ctypes.POINTER(ctypes.c_double)
    a = np.ascontiguousarray(m, dtype=np.float64).reshape(9)
    return _lib().jgs2_oracle_min_symmetric_eigenvalue(a.ctypes.data_as(D), precision)


def test_minimum_eigenvalue_of_diagonal_and_coupled_systems():
    assert _min_eig(np.diag([3.0, -2.0, 5.0])) == -2.0
    # Q diag(-0.0005, 2, 4) Q^T for a 45-degree xy rotation.
    lo, hi = -5e-4, 2.0
    mean, off = 0.5 * (lo + hi), 0.5 * (lo - hi)
    coupled = np.array([[mean, off, 0.0], [off, mean, 0.0], [0.0, 0.0, 4.0]])
    assert abs(_min_eig(coupled) - lo) < 1e-12
    assert abs(_min_eig(coupled, 32) - lo) < 1e-6
    r = _solve([[2, 0.2, 0], [0.1, 3, 0], [0, 0, 4]], [1.0, 0.0, 0.0])
    assert abs(r["asym"] - 0.025) < 1e-12


@pytest.mark.parametrize("precision", [64, 32])
def test_capped_shift_and_descent(precision):
    r = _solve(np.diag([-5e-4, 1.0, 0.75]), [1.0, -2.0, 0.5], precision=precision)
    tol = 1e-12 if precision == 64 else 1e-7
    assert r["status"] == ACCEPTED
    assert abs(r["min_eig"] - (-5e-4)) < tol
    assert abs(r["shift"] - (5e-4 + EIGENVALUE_FLOOR)) < tol
    assert r["shift"] <= MAX_SHIFT
    assert r["gdd"] < 0.0
    assert r["residual"] < (1e-10 if precision == 64 else 1e-6)


def test_shift_cap_is_refused_not_raised():
    r = _solve(np.diag([-2e-3, 1.0, 1.0]), [1.0, 0.0, 0.0])
    assert r["status"] == SHIFT_LIMIT
    assert r["shift"] > MAX_SHIFT
    assert list(r["direction"]) == [0.0, 0.0, 0.0]
    exact = _solve(np.diag([EIGENVALUE_FLOOR - MAX_SHIFT, 1.0, 1.0]), [1.0, 0.0, 0.0])
    assert exact["status"] == ACCEPTED
    assert abs(exact["shift"] - MAX_SHIFT) < 1e-14


def test_shift_and_solve_are_scale_invariant():
    ref = None
    for scale in (1e-12, 1.0, 1e12):
        r = _solve(scale * np.diag([-5e-4, 1.0, 0.75]), scale * np.array([1.0, -2.0, 0.5]), inertia=scale)
        assert r["status"] == ACCEPTED
        assert r["residual"] < 1e-9
        if ref is None:
            ref = r
        else:
            np.testing.assert_allclose(r["direction"], ref["direction"], rtol=0, atol=1e-8)
            assert abs(r["shift"] - ref["shift"]) < 1e-12


def _shift_cases():
    # nonlinear-globalization-gpu.spec.ts:851-886: f32 inputs.
    f = np.float32
    cases = [("indefinite-accepted", [-5e-4, 1, 0.75], [1, -2, 0.5], 1.0),
             ("inside-shift-cap", [f(EIGENVALUE_FLOOR - 0.000999), 1, 1], [1, -2, 0.5], 1.0),
             ("outside-shift-cap", [f(EIGENVALUE_FLOOR - 0.001001), 1, 1], [1, -2, 0.5], 1.0)]
    for s in (1e-12, 1.0, 1e12):
        cases.append((f"scale-{s}", [-5e-4 * s, s, 0.75 * s], [s, -2 * s, 0.5 * s], float(f(s))))
    out = []
    for name, diag, grad, inertia in cases:
        h = np.diag(np.array(diag, dtype=np.float32)).astype(np.float64)
        g = np.array(grad, dtype=np.float32).astype(np.float64)
        out.append((name, h, g, inertia))
    return out


@pytest.mark.parametrize("name,h,g,inertia", _shift_cases(), ids=[c[0] for c in _shift_cases()])
def test_f32_solve_matches_the_fp64_policy(name, h, g, inertia):
    # The same cases' bounds (:1040-1062): the f32 solve against the policy
    # evaluated in double on the same f32 inputs.
    f32 = _solve(h, g, inertia, precision=32)
    f64 = _solve(h, g, inertia, precision=64)
    accepted = f64["status"] == ACCEPTED
    assert accepted == (name != "outside-shift-cap")
    assert f32["status"] == (ACCEPTED if accepted else SHIFT_LIMIT)
    rel = np.linalg.norm(f32["direction"] - f64["direction"]) / max(1.0, np.linalg.norm(f32["direction"]),
                                                                  np.linalg.norm(f64["direction"]))
    assert rel < 2e-4
    assert abs(f32["min_eig"] - f64["min_eig"]) < 2e-6
    assert abs(f32["shift"] - f64["shift"]) < 2e-6
    assert abs(f32["scale"] - f64["scale"]) / max(1e-30, abs(f64["scale"])) < 2e-6
    if accepted:
        assert abs(f32["gdd"] - f64["gdd"]) / abs(f64["gdd"]) < 2e-4
        assert f32["residual"] < 2e-5
    else:
        assert f32["gdd"] == 0.0 and f32["residual"] == 0.0

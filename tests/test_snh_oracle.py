"""The oracle's stable Neo-Hookean density pinned to the reference's density
tests (src/simulation/cpu/stable-neo-hookean.test.ts:53-232), which use
E = 8e4, nu = 0.3:

- the scene builder's reparameterisation of the Lame constants
  (mu = 4/3 mu_L, lambda = lambda_L + 5/6 mu_L; :53-69), read back from a
  packed input's per-tet material;
- the linear Hooke response of the tangent at the identity
  (mu_L (D + D^T) + lambda_L tr(D) I; :71-94);
- zero energy and stress at rest and under a rigid rotation (:96-122);
- finite energy, stress and tangent through collapse and inversion
  (:124-159);
- a symmetric tangent (:161-183) and objectivity of energy, stress and the
  tangent action under rotation (:185-231);
- the WGSL library's numeric cases
  (src/simulation/gpu/stable-neo-hookean-wgsl.test.ts:211-296): rest,
  rank-one collapse and inversion, finite differences at three poses to
  relative error 2e-10, and the adjusted Hooke response to 1e-14.

The reference's error measure is ||a - b|| / max(1, ||a||, ||b||)
(src/simulation/cpu/finite-difference.ts:94-118). The FP64 run must meet the
reference's bounds. The f32 mirror, which the GPU step follows, is held to
f32-sized bounds on the same cases.
"""
import ctypes
import math

import numpy as np
import pytest

from jgs2_b200 import scenes
from oracle import oracle as O

YOUNG, POISSON = 8.0e4, 0.3
MU_L = YOUNG / (2 * (1 + POISSON))
LAMBDA_L = YOUNG * POISSON / ((1 + POISSON) * (1 - 2 * POISSON))
MU = 4.0 / 3.0 * MU_L
LAMBDA = LAMBDA_L + 5.0 / 6.0 * MU_L

DEFORMATION = np.array([[1.08, 0.17, -0.04], [0.03, 0.84, 0.12], [-0.09, 0.05, 1.14]])
DIRECTION = np.array([[0.07, -0.02, 0.11], [-0.04, 0.03, 0.08], [0.05, -0.09, -0.01]])


def _lib():
    L = O.lib()
    D = ctypes.POINTER(ctypes.c_double)
    L.jgs2_oracle_snh_density.argtypes = [D, D, ctypes.c_double, ctypes.c_double, ctypes.c_int, D]
    L.jgs2_oracle_snh_density.restype = ctypes.c_int
    return L


def _density(f, h=None, precision=64, lam=LAMBDA, mu=MU):
    """(energy, first Piola, tangent action dP[h], det f) of the oracle."""
    D = ctypes.POINTER(ctypes.c_double)
    f = np.ascontiguousarray(f, dtype=np.float64)
    h = np.zeros((3, 3)) if h is None else np.ascontiguousarray(h, dtype=np.float64)
    out = np.zeros(20)
    assert _lib().jgs2_oracle_snh_density(f.ctypes.data_as(D), h.ctypes.data_as(D), lam, mu, precision,
                                          out.ctypes.data_as(D)) == 0
    return out[0], out[1:10].reshape(3, 3), out[10:19].reshape(3, 3), out[19]


def _relative_error(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(1.0, np.linalg.norm(a), np.linalg.norm(b)))


def _tangent_matrix(f, precision=64):
    """The 9 x 9 tangent, one column per unit direction (rows of h)."""
    cols = []
    for k in range(9):
        e = np.zeros(9)
        e[k] = 1.0
        cols.append(_density(f, e.reshape(3, 3), precision)[2].ravel())
    return np.stack(cols, axis=1)


def test_scene_reparameterises_lame_constants():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, YOUNG, POISSON)
    sc.add_cuboid((1, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), m, 0, 0)
    sc.precompute(timestep=1 / 60, cubature_k=sc.tet_count, exact_complement=1)
    meta = sc.pack().tet_meta.reshape(-1, 4)
    np.testing.assert_allclose(meta[:, 1], np.float32(LAMBDA), rtol=0)
    np.testing.assert_allclose(meta[:, 2], np.float32(MU), rtol=0)
    alpha = 1 + MU / LAMBDA - MU / (4 * LAMBDA)
    # The step folds alpha into the -3/4 mu (J - 1) term: alpha - 1 = 3 mu / (4 lambda).
    assert abs((alpha - 1) - 0.75 * MU / LAMBDA) < 1e-14


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-6)])
def test_hooke_limit_at_identity(precision, tol):
    d = np.array([[0.2, -0.3, 0.1], [0.4, -0.1, 0.25], [-0.2, 0.15, 0.35]])
    _, _, response, _ = _density(np.eye(3), d, precision)
    expected = MU_L * (d + d.T) + LAMBDA_L * np.trace(d) * np.eye(3)
    assert _relative_error(response, expected) < tol


@pytest.mark.parametrize("precision,tol", [(64, 1e-10), (32, 1e-6 * MU)])
def test_zero_rest_response_and_rigid_rotation(precision, tol):
    # f32 bound: rounding at the scale of the stiffness mu (about 4e4).
    a = 0.63
    rotation = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    for f in (np.eye(3), rotation):
        energy, piola, _, det = _density(f, None, precision)
        assert abs(energy) < tol
        assert np.linalg.norm(piola) < tol
        assert abs(det - 1.0) < (1e-14 if precision == 64 else 1e-6)


@pytest.mark.parametrize("precision", [64, 32])
def test_finite_through_collapse_and_inversion(precision):
    for j in (0.5, 0.1, 0.01, 0.0, -0.1, -1.0):
        f = np.diag([j, 1.0, 1.0])
        energy, piola, tangent, det = _density(f, DIRECTION, precision)
        assert abs(det - j) < 1e-7
        assert math.isfinite(energy) and np.isfinite(piola).all() and np.isfinite(tangent).all()


@pytest.mark.parametrize("precision", [64, 32])
def test_tangent_is_symmetric(precision):
    # FP64: the reference's absolute 1e-10 on entries of order 1e5; f32:
    # 1e-6 of the largest entry.
    t = _tangent_matrix(DEFORMATION, precision)
    tol = 1e-10 if precision == 64 else 1e-6 * float(np.abs(t).max())
    assert float(np.abs(t - t.T).max()) < tol


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 5e-6)])
def test_objective_under_rotation(precision, tol):
    a = -0.52
    rotation = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    e0, p0, t0, _ = _density(DEFORMATION, DIRECTION, precision)
    e1, p1, t1, _ = _density(rotation @ DEFORMATION, rotation @ DIRECTION, precision)
    assert abs(e0 - e1) < (1e-10 if precision == 64 else 1e-5 * abs(e0))
    assert _relative_error(p1, rotation @ p0) < tol
    assert _relative_error(t1, rotation @ t0) < tol


def test_stress_and_tangent_match_finite_differences():
    # Central differences of the FP64 energy and stress at the test pose.
    eps = 1e-6
    _, piola, _, _ = _density(DEFORMATION)
    grad = np.zeros((3, 3))
    for r in range(3):
        for c in range(3):
            e = np.zeros((3, 3))
            e[r, c] = eps
            grad[r, c] = (_density(DEFORMATION + e)[0] - _density(DEFORMATION - e)[0]) / (2 * eps)
    assert _relative_error(grad, piola) < 1e-7
    _, _, action, _ = _density(DEFORMATION, DIRECTION)
    fd = (_density(DEFORMATION + eps * DIRECTION)[1] - _density(DEFORMATION - eps * DIRECTION)[1]) / (2 * eps)
    assert _relative_error(fd, action) < 1e-7


def _column_major(values):
    # The WGSL library's test matrices list columns first.
    return np.array(values, dtype=np.float64).reshape(3, 3).T


def test_wgsl_library_cases_rest_collapse_and_inversion():
    # stable-neo-hookean-wgsl.test.ts:211-227 (adjusted lambda 75 000, mu
    # 42 000): zero energy and stress at rest; finite energy and stress for a
    # rank-one collapse and for an inverted gradient.
    lam, mu = 75_000.0, 42_000.0
    energy, piola, _, _ = _density(np.eye(3), lam=lam, mu=mu)
    assert energy == 0.0 and np.linalg.norm(piola) < 1e-11
    collapsed = _column_major([1, 0, 0, 0, 0, 0, 0, 0, 0])
    inverted = _column_major([-0.8, 0.1, 0, 0.2, 1.1, 0.3, 0, -0.1, 0.9])
    assert np.linalg.det(inverted) < 0
    for f in (collapsed, inverted):
        for precision in (64, 32):
            energy, piola, _, _ = _density(f, precision=precision, lam=lam, mu=mu)
            assert math.isfinite(energy) and np.isfinite(piola).all()


def test_wgsl_library_cases_finite_differences():
    # stable-neo-hookean-wgsl.test.ts:229-269 (adjusted lambda 63 000, mu
    # 37 000, step 1e-5): the energy's directional derivative equals P : H to
    # four decimals, and the tangent action matches the central difference
    # of P within relative error 2e-10, at rest, stretched and inverted.
    lam, mu, step = 63_000.0, 37_000.0, 1e-5
    direction = _column_major([0.17, -0.23, 0.09, 0.31, -0.12, 0.26, -0.08, 0.14, 0.19])
    poses = (np.eye(3), _column_major([1.13, 0.07, -0.03, -0.21, 0.91, 0.16, 0.08, -0.12, 1.04]),
             _column_major([-0.72, 0.11, 0.04, 0.09, 1.08, -0.17, -0.06, 0.14, 0.83]))
    for f in poses:
        ep, pp, _, _ = _density(f + step * direction, lam=lam, mu=mu)
        en, pn, _, _ = _density(f - step * direction, lam=lam, mu=mu)
        _, piola, action, _ = _density(f, direction, lam=lam, mu=mu)
        assert abs((ep - en) / (2 * step) - float(np.sum(piola * direction))) < 5e-5
        fd = (pp - pn) / (2 * step)
        err = float(np.linalg.norm(action - fd) / max(1.0, np.linalg.norm(fd)))
        assert err < 2e-10, err


def test_wgsl_library_recovers_the_hooke_response():
    # stable-neo-hookean-wgsl.test.ts:271-296 (Hooke lambda 31 000, mu
    # 19 000): after the adjustment the tangent at the identity is
    # mu (H + H^T) + lambda tr(H) I to relative error 1e-14.
    lam_h, mu_h = 31_000.0, 19_000.0
    h = _column_major([0.21, -0.08, 0.13, 0.17, -0.11, 0.06, -0.04, 0.19, 0.27])
    _, _, action, _ = _density(np.eye(3), h, lam=lam_h + 5.0 / 6.0 * mu_h, mu=4.0 / 3.0 * mu_h)
    expected = mu_h * (h + h.T) + lam_h * np.trace(h) * np.eye(3)
    assert np.linalg.norm(action - expected) / max(1.0, np.linalg.norm(expected)) < 1e-14

"""Precision of the device IPC closest-feature routine on near-degenerate
pairs, stated against the oracle's FP64 run of the same method
(jgs2_ipc_point_triangle_contact / jgs2_ipc_edge_edge_contact,
src/simulation/gpu/ipc-contact-wgsl.ts:151-300).

The step evaluates every contact in f32 and recomputes near-degenerate pairs
(sliver triangles, near-parallel edges, near-touching features) in FP64.
Each case below is a seeded family of such pairs, translated away from the
origin so f32 coordinates carry their full rounding.  Error measure: the
distance error relative to max(FP64 distance, 2^-10 x feature extent).
The FP64 path is held to 1e-6 (f32 rounding of an FP64 result is 6e-8);
the plain f32 arithmetic of the same pairs (the oracle's f32 mirror) is
reported beside it.
"""
import ctypes

import numpy as np
import pytest

from jgs2_b200 import _ffi

D = ctypes.POINTER(ctypes.c_double)
WIDE_RTOL = 1e-6


def _oracle():
    from oracle import oracle as O

    L = O.lib()
    for name in ("jgs2_oracle_ipc_contact", "jgs2_oracle_ipc_contact_f32"):
        getattr(L, name).argtypes = [ctypes.c_uint32, D, D]
        getattr(L, name).restype = ctypes.c_int
    return L


def _oracle_eval(name, kinds, pts):
    L = _oracle()
    out = np.zeros((len(kinds), 9))
    for i, (k, p) in enumerate(zip(kinds, pts)):
        x = np.ascontiguousarray(p, dtype=np.float64).reshape(-1)
        o = np.zeros(9)
        getattr(L, name)(int(k), x.ctypes.data_as(D), o.ctypes.data_as(D))
        out[i] = o
    return out


def _cases(seed=7):
    """(kind, points (4, 3) float32, extent) for four families of pairs."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(64):
        shift = rng.uniform(-20, 20, 3)
        rot, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        fam = i % 4
        d = 10.0 ** rng.uniform(-6, -2)
        if fam == 0:  # near-parallel edges
            ang = 10.0 ** rng.uniform(-5, -2)
            p = np.array([[0, 0, 0], [1, 0, 0], [0.3, d, 0], [1.3, d + np.sin(ang), 0.0]])
            kind = 1
        elif fam == 1:  # crossing edges, near touching
            p = np.array([[-0.5, 0, 0], [0.5, 0, 0], [0.1, -0.5, d], [-0.1, 0.5, d]])
            kind = 1
        elif fam == 2:  # sliver triangle, point above it
            h = 10.0 ** rng.uniform(-5, -2)
            p = np.array([[0.4, 0.0002, d], [0, 0, 0], [1, 0, 0], [0.5, h, 0]])
            kind = 0
        else:  # point near-touching a regular triangle
            p = np.array([[0.3, 0.3, d], [0, 0, 0], [1, 0, 0], [0, 1, 0]])
            kind = 0
        pts = (p @ rot.T + shift).astype(np.float32)
        out.append((kind, pts, 1.0))
    return out


def _relative_errors(kinds, pts, extents, got, ref):
    floor = np.array(extents) * 2.0 ** -10
    return np.abs(got[:, 0] - ref[:, 0]) / np.maximum(ref[:, 0], floor)


def test_oracle_f32_loses_digits_on_these_pairs():
    # CPU-only: the families are hard for plain f32 (the reason for FP64).
    cases = _cases()
    kinds = [c[0] for c in cases]
    pts = [c[1].astype(np.float64) for c in cases]
    ref = _oracle_eval("jgs2_oracle_ipc_contact", kinds, pts)
    f32 = _oracle_eval("jgs2_oracle_ipc_contact_f32", kinds, pts)
    err = _relative_errors(kinds, pts, [c[2] for c in cases], f32, ref)
    assert np.all(ref[:, 8] == 1.0)
    assert err.max() > 1e-3, err.max()


@pytest.mark.gpu
def test_device_contact_features_match_fp64():
    cases = _cases()
    kinds = np.array([c[0] for c in cases], dtype=np.uint32)
    pts = np.stack([c[1] for c in cases]).astype(np.float32)
    out = np.zeros((len(cases), 9), dtype=np.float32)
    wide = np.zeros(len(cases), dtype=np.uint32)
    L = _ffi.step_lib()
    f = L.jgs2_evaluate_contact_features
    f.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
                  ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
    f.restype = ctypes.c_int
    rc = f(_ffi.fptr(pts.reshape(-1)), kinds.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), len(cases),
           _ffi.fptr(out.reshape(-1)), wide.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), 0)
    assert rc == 0
    ref = _oracle_eval("jgs2_oracle_ipc_contact", kinds, [p.astype(np.float64) for p in pts])
    f32 = _oracle_eval("jgs2_oracle_ipc_contact_f32", kinds, [p.astype(np.float64) for p in pts])
    extents = [c[2] for c in cases]
    gpu_err = _relative_errors(kinds, pts, extents, out.astype(np.float64), ref)
    f32_err = _relative_errors(kinds, pts, extents, f32, ref)
    print(f"contact distance error vs FP64 over {len(cases)} near-degenerate pairs: device max {gpu_err.max():.2e} "
          f"({int(wide.sum())} took the FP64 run), plain f32 max {f32_err.max():.2e}")
    assert np.all(out[:, 8] == 1.0)
    assert wide.sum() >= len(cases) // 2
    assert gpu_err[wide == 1].max() <= WIDE_RTOL
    assert gpu_err.max() <= max(WIDE_RTOL, 1e-3)
    # Weights of FP64-path pairs reproduce the FP64 closest points.
    np.testing.assert_allclose(out[wide == 1, 4:8], ref[wide == 1, 4:8], atol=1e-5)

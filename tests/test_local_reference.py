"""The exact-complement local system on a deformed pose: the reference's
nonlinear local-reference case (src/simulation/cpu/jgs2-local.test.ts:242-308).

The fixture:
- a one-hex unit cube (the reference mesh generator's default size), pinned
  at x = 0;
- stable Neo-Hookean, density 1000, E 8e4, nu 0.3;
- exact-complement cubature: every tet at weight one, whole-mesh exact bases;
- every free coordinate i moved by 0.018 sin(0.4 + 1.3 i), with the inertial
  target left at the rest shape;
- an external force of 0.3 cos(0.8 i) on every free coordinate i.

The reference's CPU case projects onto the rest-shape exact basis. Its GPU
step, which the oracle follows, first turns each stored block by the vertex
frames: R_u B_u R_v^T, for a block of vertex u in a record of source v
(src/simulation/gpu/jgs2-shader.ts:1851-1860). R is the polar factor of the
vertex's volume-averaged deformation gradient. At the last free vertex, the
oracle's local system (FP64) must be the exact projection B^T grad E,
B^T hess(E) B of the whole incremental potential E onto that rotated basis
B. E is the inertia, the external-force work and the stable Neo-Hookean
energy. Its restricted energy at the reference's
local displacement (0.003, -0.002, 0.0015) must equal E(x + B d) - E(x).
The expected values are computed here in float64 from the input's own f32
data. The gradient is analytic; the Hessian is taken by central differences
of that gradient along B.
"""
import ctypes

import numpy as np
import pytest

from jgs2_b200 import scenes
from oracle import oracle as O

H = 1 / 60
SETTINGS = dict(timestep=H, gravity=(0.0, 0.0, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=1)
LOCAL_DISPLACEMENT = np.array([0.003, -0.002, 0.0015])


def _fixture():
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 8.0e4, 0.3)
    sc.add_cuboid((1, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=H, cubature_k=sc.tet_count, exact_complement=1, method=scenes.PRECOMPUTE_EXACT)
    rest = sc.rest_positions().astype(np.float64)
    free = sc.pack().vertex_info.reshape(-1, 4)[:, 2] == 0
    coords = rest[free].reshape(-1)
    i = np.arange(coords.size)
    deformed = rest.copy()
    deformed[free] = (coords + 0.018 * np.sin(0.4 + 1.3 * i)).reshape(-1, 3)
    pos = np.ones((rest.shape[0], 4), dtype=np.float32)
    pos[:, :3] = deformed
    # The predictor x + h v lands on the rest shape.
    vel = np.zeros((rest.shape[0], 4), dtype=np.float32)
    vel[:, :3] = (rest - pos[:, :3].astype(np.float64)) / H
    sc.set_initial_state(pos.reshape(-1), vel.reshape(-1), pin_at_initial=False)
    inp = sc.pack()
    force = np.zeros((rest.shape[0], 3))
    force[free] = (0.3 * np.cos(0.8 * i)).reshape(-1, 3)
    inp.external_forces = force.astype(np.float32).reshape(-1)
    return inp, free


def _basis(inp, vertex):
    """Vertex `vertex`'s stored exact basis over every vertex (3V x 3), read
    from the blocks of its records."""
    K = inp.cubature_k
    tets = inp.tet_indices.reshape(-1, 4)
    B = np.zeros((inp.vertex_count, 3, 3))
    for r in range(vertex * K, (vertex + 1) * K):
        t = int(inp.cubature_tet_ids[r])
        if t == 0xFFFFFFFF:
            continue
        blocks = inp.cubature_basis[36 * r:36 * r + 36].reshape(4, 3, 3).astype(np.float64)
        for lane in range(4):
            B[int(tets[t, lane])] = blocks[lane]
    return B.reshape(-1, 3)


class _Potential:
    """The incremental potential in float64 over the input's f32 data."""

    def __init__(self, inp, free):
        h = float(np.float32(H))
        x = inp.positions.reshape(-1, 4)[:, :3].astype(np.float64)
        v = inp.velocities.reshape(-1, 4)[:, :3].astype(np.float64)
        self.target = x + h * v
        self.mass = np.where(free, inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64), 0.0)
        self.inertia = self.mass / (h * h)
        self.force = inp.external_forces.reshape(-1, 3).astype(np.float64)
        self.free = free
        self.tets = inp.tet_indices.reshape(-1, 4).astype(np.int64)
        self.minv = np.transpose(inp.tet_inverse_dm.reshape(-1, 3, 4)[:, :, :3].astype(np.float64), (0, 2, 1))
        meta = inp.tet_meta.reshape(-1, 4).astype(np.float64)
        self.vol, self.lam, self.mu = meta[:, 0], meta[:, 1], meta[:, 2]

    def _gradients(self, y):
        ds = np.stack([y[self.tets[:, k]] - y[self.tets[:, 0]] for k in (1, 2, 3)], axis=-1)
        return ds @ self.minv

    def energy(self, y):
        f = self._gradients(y)
        i1 = np.einsum("tij,tij->t", f, f)
        j = np.linalg.det(f)
        mu, lam = self.mu, self.lam
        psi = 0.5 * mu * (i1 - 3) - 0.75 * mu * (j - 1) + 0.5 * lam * (j - 1) ** 2 - 0.5 * mu * np.log((i1 + 1) / 4)
        d = y - self.target
        return (0.5 * float(np.sum(self.inertia[:, None] * d * d)) - float(np.sum(self.force[self.free] * y[self.free]))
                + float(np.sum(self.vol * psi)))

    def gradient(self, y):
        f = self._gradients(y)
        i1 = np.einsum("tij,tij->t", f, f)
        c0, c1, c2 = f[:, :, 0], f[:, :, 1], f[:, :, 2]
        cof = np.stack([np.cross(c1, c2), np.cross(c2, c0), np.cross(c0, c1)], axis=-1)
        j = np.einsum("ti,ti->t", c0, cof[:, :, 0])
        p = ((self.mu * (1 - 1 / (i1 + 1)))[:, None, None] * f
             + (self.lam * (j - 1) - 0.75 * self.mu)[:, None, None] * cof)
        g_ds = self.vol[:, None, None] * p @ np.transpose(self.minv, (0, 2, 1))
        g = self.inertia[:, None] * (y - self.target)
        g[self.free] -= self.force[self.free]
        for k in (1, 2, 3):
            np.add.at(g, self.tets[:, k], g_ds[:, :, k - 1])
            np.add.at(g, self.tets[:, 0], -g_ds[:, :, k - 1])
        g[~self.free] = 0.0
        return g.reshape(-1)


def _rotated(pot, B, vertex, y):
    """R_u B_u R_v^T over every vertex u, R the polar factor of the vertex's
    volume-weighted average deformation gradient at pose y."""
    f = pot._gradients(y)
    acc = np.zeros((y.shape[0], 3, 3))
    tot = np.zeros(y.shape[0])
    for k in range(4):
        np.add.at(acc, pot.tets[:, k], pot.vol[:, None, None] * f)
        np.add.at(tot, pot.tets[:, k], pot.vol)
    u, _, vt = np.linalg.svd(acc / np.maximum(tot, 1e-300)[:, None, None])
    r = u @ vt
    blocks = B.reshape(-1, 3, 3)
    return np.einsum("uij,ujk,lk->uil", r, blocks, r[vertex]).reshape(-1, 3)


def _oracle_local(inp, vertex, d, precision=64):
    L = O.lib()
    D = ctypes.POINTER(ctypes.c_double)
    L.jgs2_oracle_local_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, D, D]
    o = O.OracleSolver(inp, SETTINGS, precision=precision)
    rec = O._settings_struct(O.resolve_settings(None, **SETTINGS))
    out = np.zeros(14)
    dd = np.ascontiguousarray(d, dtype=np.float64)
    L.jgs2_oracle_local_system(o._h, ctypes.byref(rec), vertex, dd.ctypes.data_as(D), out.ctypes.data_as(D))
    return out[:3], out[3:12].reshape(3, 3).T, out[12]


def _relative_error(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(1.0, np.linalg.norm(b)))


# FP64 bounds: the reference's 1e-13 for the projected gradient; the Hessian
# is compared with central differences (step 1e-6) of the analytic gradient;
# the restricted energy equals the direct difference to rounding. The f32
# mirror, which the GPU step follows, is held to f32-sized bounds.
@pytest.mark.parametrize("precision,tol_g,tol_h,tol_e", [(64, 1e-13, 1e-8, 1e-12), (32, 1e-6, 5e-6, 1e-4)])
def test_local_system_is_the_exact_projection_on_a_deformed_pose(precision, tol_g, tol_h, tol_e):
    inp, free = _fixture()
    vertex = int(np.flatnonzero(free)[-1])
    B = _basis(inp, vertex)
    np.testing.assert_allclose(B.reshape(-1, 3, 3)[vertex], np.eye(3), atol=1e-6)
    pot = _Potential(inp, free)
    x = inp.positions.reshape(-1, 4)[:, :3].astype(np.float64)
    B = _rotated(pot, B, vertex, x)
    g_want = B.T @ pot.gradient(x)
    eps = 1e-6
    h_want = np.stack([B.T @ (pot.gradient(x + eps * (B[:, k]).reshape(-1, 3))
                              - pot.gradient(x - eps * (B[:, k]).reshape(-1, 3))) / (2 * eps) for k in range(3)],
                      axis=1)
    g_loc, h_loc, _ = _oracle_local(inp, vertex, np.zeros(3), precision)
    _, _, delta = _oracle_local(inp, vertex, LOCAL_DISPLACEMENT, precision)
    e_want = pot.energy(x + (B @ LOCAL_DISPLACEMENT).reshape(-1, 3)) - pot.energy(x)
    eg, eh, ee = _relative_error(g_loc, g_want), _relative_error(h_loc, h_want), abs(delta - e_want) / abs(e_want)
    print(f"f{precision} deformed pose, vertex {vertex}: gradient {eg:.1e}, Hessian {eh:.1e}, restricted energy {ee:.1e} "
          f"(|g| {np.linalg.norm(g_want):.3e}, dE {e_want:.4e})")
    assert eg < tol_g and eh < tol_h and ee < tol_e

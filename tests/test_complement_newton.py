"""The exact JGS2 complement reproduces the global Newton step: the
reference's Eq. 7-13 oracle (src/simulation/cpu/precompute.test.ts:438-499).

The fixture is a 3x2x2-hex bar, pinned at x = 0, with exact-complement
cubature (every tet, weight one, whole-mesh exact bases). It is at rest,
given seeded velocities, with no gravity. At rest the stable Neo-Hookean
tangent is the linear Hooke stiffness. So the energy of the first iteration
is the quadratic (1/2) dx^T H dx + g^T dx, with:
- H = K + M / h^2 the assembled rest system;
- g = M (x - x~) / h^2 the inertia gradient.

One vertex's local system, as the oracle's step assembles it (incident tets
plus the complement records), must solve to that vertex's block of the
global Newton step -H^-1 g.
"""
import ctypes

import numpy as np

from jgs2_b200 import scenes
from oracle import oracle as O

from test_exact_basis import DENSITY, POISSON, TIMESTEP, YOUNG, _rest_system

SETTINGS = dict(timestep=TIMESTEP, gravity=(0.0, 0.0, 0.0), floor_stiffness=0.0, parity_mode=1, iterations=1)


def _bar_at_rest_moving(seed=7):
    sc = scenes.Scene()
    m = sc.add_material(DENSITY, YOUNG, POISSON)
    sc.add_cuboid((3, 2, 2), (0.0, 0.0, 0.0), (0.3, 0.2, 0.2), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=TIMESTEP, cubature_k=sc.tet_count, exact_complement=1, method=scenes.PRECOMPUTE_EXACT)
    rest = sc.rest_positions().astype(np.float64)
    base = sc.pack()
    pinned = base.vertex_info.reshape(-1, 4)[:, 2] != 0
    rng = np.random.default_rng(seed)
    vel = np.zeros((rest.shape[0], 4), dtype=np.float32)
    vel[~pinned, :3] = rng.uniform(-0.5, 0.5, size=(int((~pinned).sum()), 3))
    pos = np.ones((rest.shape[0], 4), dtype=np.float32)
    pos[:, :3] = rest
    sc.set_initial_state(pos.reshape(-1), vel.reshape(-1), pin_at_initial=False)
    return sc.pack(), rest, vel[:, :3].astype(np.float64), pinned


def _local_system(inp, vertex):
    L = O.lib()
    D = ctypes.POINTER(ctypes.c_double)
    L.jgs2_oracle_local_system.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, D, D]
    o = O.OracleSolver(inp, SETTINGS, precision=64)
    rec = O._settings_struct(O.resolve_settings(None, **SETTINGS))
    out = np.zeros(14)
    d = np.zeros(3)
    L.jgs2_oracle_local_system(o._h, ctypes.byref(rec), vertex, d.ctypes.data_as(D), out.ctypes.data_as(D))
    return out[:3], out[3:12].reshape(3, 3).T


def _stored_basis(inp, v, dof, n):
    """Vertex v's stored exact basis as a 3 x n block row over the movable
    coordinates (each vertex's block read from a record that holds it)."""
    K = inp.cubature_k
    tets = inp.tet_indices.reshape(-1, 4)
    B = np.zeros((n, 3))
    for r in range(v * K, (v + 1) * K):
        t = int(inp.cubature_tet_ids[r])
        if t == 0xFFFFFFFF:
            continue
        blocks = inp.cubature_basis[36 * r:36 * r + 36].reshape(4, 3, 3).astype(np.float64)
        for l in range(4):
            u = int(tets[t, l])
            if dof[u] >= 0:
                B[dof[u]:dof[u] + 3] = blocks[l]
    return B


def test_exact_complement_local_step_is_the_global_newton_block():
    inp, rest, vel, pinned = _bar_at_rest_moving()
    H, dof = _rest_system(inp, rest)
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    active = np.flatnonzero(~pinned)
    # x - x~ = -h v with no gravity.
    g = np.concatenate([mass[v] / TIMESTEP ** 2 * (-TIMESTEP * vel[v]) for v in active])
    newton = -np.linalg.solve(H, g)
    worst_h = worst_g = worst_step = 0.0
    for v in active:
        g_loc, H_loc = _local_system(inp, int(v))
        # The assembled local system is the reduced system B^T H B, B^T g
        # over the stored bases B.
        B = _stored_basis(inp, int(v), dof, H.shape[0])
        h_red, g_red = B.T @ H @ B, B.T @ g
        worst_h = max(worst_h, float(np.abs(H_loc - h_red).max() / np.abs(h_red).max()))
        worst_g = max(worst_g, float(np.abs(g_loc - g_red).max() / np.abs(g_red).max()))
        # With the exact basis that reduced step is the vertex's block of the
        # global Newton step (Eq. 7-13).
        step = -np.linalg.solve(H_loc, g_loc)
        want = newton[dof[v]:dof[v] + 3]
        worst_step = max(worst_step, float(np.linalg.norm(step - want) / np.linalg.norm(want)))
    print(f"exact complement, {len(active)} vertices: reduced Hessian {worst_h:.1e}, reduced gradient "
          f"{worst_g:.1e} (against the stored bases); step vs global Newton {worst_step:.1e}")
    # The oracle evaluates from the input's f32 data (inverse rest matrices,
    # volumes, materials, masses, velocities), this restatement from the
    # float64 rest shape: the reduced Hessian agrees to f32 rounding, the
    # reduced gradient (a sum over every vertex's inertia force) to a few
    # 1e-5, and the 3x3 solve carries that into the step.
    assert worst_h < 1e-6
    assert worst_g < 1e-4
    assert worst_step < 1e-4


def test_exact_complement_projects_quadratic_targets_densely():
    # nonlinear-restricted-energy.test.ts:343-420: with every tet at unit
    # weight, target springs k |x - t|^2 / 2 on the free vertices enter the
    # local system as the dense projection B^T (H + k) B, B^T (g + k (x - t)).
    inp, rest, vel, pinned = _bar_at_rest_moving()
    active = np.flatnonzero(~pinned)
    rng = np.random.default_rng(11)
    k = np.zeros(inp.vertex_count, dtype=np.float32)
    k[active] = rng.uniform(50.0, 500.0, size=active.size).astype(np.float32)
    targets = (inp.positions.reshape(-1, 4)[:, :3] + rng.uniform(-0.02, 0.02, (inp.vertex_count, 3))).astype(
        np.float32)
    inp.target_positions = targets.reshape(-1)
    inp.target_stiffnesses = k
    H, dof = _rest_system(inp, rest)
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    x = inp.positions.reshape(-1, 4)[:, :3].astype(np.float64)
    g = np.concatenate([mass[v] / TIMESTEP ** 2 * (-TIMESTEP * vel[v]) + float(k[v]) * (x[v] - targets[v])
                        for v in active])
    Ht = H + np.diag(np.repeat(k[active].astype(np.float64), 3))
    worst_h = worst_g = 0.0
    for v in active:
        g_loc, H_loc = _local_system(inp, int(v))
        B = _stored_basis(inp, int(v), dof, H.shape[0])
        h_red, g_red = B.T @ Ht @ B, B.T @ g
        worst_h = max(worst_h, float(np.abs(H_loc - h_red).max() / np.abs(h_red).max()))
        worst_g = max(worst_g, float(np.abs(g_loc - g_red).max() / np.abs(g_red).max()))
    print(f"targets, dense projection: reduced Hessian {worst_h:.1e}, reduced gradient {worst_g:.1e}")
    assert worst_h < 1e-6 and worst_g < 1e-4

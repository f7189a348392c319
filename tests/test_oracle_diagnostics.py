"""Exact all-element oracle diagnostics (readOracleDiagnostics,
src/simulation/gpu/jgs2-solver.ts:2882-2907; the evaluator of
src/simulation/gpu/jgs2-diagnostics.ts:388-1146).

The device evaluation is compared with a float64 numpy restatement of the same
quantities at the pose the solver reports: the five energy components, the
per-vertex active-coordinate gradient and diagonal Hessian block (inertia,
stable Neo-Hookean elasticity, external force, quadratic target, penalty
floor), the per-tet energies and determinants, the component norms and the
force-balance residual.
"""
import numpy as np
import pytest

from jgs2_b200 import scenes, solver


def _snh(F, lam, mu):
    I1 = np.sum(F * F)
    J = np.linalg.det(F)
    cof = np.stack([np.cross(F[:, 1], F[:, 2]), np.cross(F[:, 2], F[:, 0]), np.cross(F[:, 0], F[:, 1])], axis=1)
    a = mu * (1 - 1 / (I1 + 1))
    b = lam * (J - 1) - 0.75 * mu
    c1 = 2 * mu / (I1 + 1) ** 2
    psi = 0.5 * mu * (I1 - 3) - 0.75 * mu * (J - 1) + 0.5 * lam * (J - 1) ** 2 - 0.5 * mu * np.log((I1 + 1) / 4)
    return psi, a * F + b * cof, a, c1, cof, J


def _reference(inp, x, pred, h, forces, targets, floor_height, floor_k):
    """float64 restatement of evaluateDiagnosticTetrahedra / Vertices."""
    V, T = inp.vertex_count, inp.tet_count
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    active = inp.vertex_info.reshape(-1, 4)[:, 2] == 0
    tets = inp.tet_indices.reshape(-1, 4)
    inv = inp.tet_inverse_dm.reshape(-1, 3, 4)[:, :, :3].astype(np.float64)  # three padded columns
    meta = inp.tet_meta.reshape(-1, 4).astype(np.float64)
    grad = np.zeros((V, 3))
    g_el = np.zeros((V, 3))
    H = np.zeros((V, 3, 3))
    tet_e = np.zeros(T)
    tet_det = np.zeros(T)
    w = mass / (h * h)
    for t in range(T):
        q = tets[t]
        Dm_inv = inv[t].T  # columns stored as rows
        Ds = np.stack([x[q[1]] - x[q[0]], x[q[2]] - x[q[0]], x[q[3]] - x[q[0]]], axis=1)
        F = Ds @ Dm_inv
        vol, lam, mu = meta[t, 0], meta[t, 1], meta[t, 2]
        psi, P, a, c1, cof, J = _snh(F, lam, mu)
        tet_e[t], tet_det[t] = vol * psi, J
        rows = Dm_inv
        gs = [-(rows[0] + rows[1] + rows[2]), rows[0], rows[1], rows[2]]
        for s in range(4):
            v = q[s]
            if not active[v]:
                continue
            g = gs[s]
            g_el[v] += vol * P @ g
            u, wv = F @ g, cof @ g
            H[v] += vol * (a * (g @ g) * np.eye(3) + c1 * np.outer(u, u) + lam * np.outer(wv, wv))
    e = dict(inertia=0.0, elasticity=tet_e.sum(), externalForce=0.0, quadraticTarget=0.0, floorContact=0.0)
    sq = dict(inertia=0.0, material=0.0, externalForce=0.0, target=0.0, contact=0.0)
    for v in range(V):
        if not active[v]:
            continue
        d = x[v] - pred[v]
        gi = w[v] * d
        gf = -forces[v]
        gt = targets[v, 3] * (x[v] - targets[v, :3])
        gfl = np.zeros(3)
        H[v] += (w[v] + targets[v, 3]) * np.eye(3)
        dist = x[v, 1] - floor_height
        if floor_k > 0 and dist < 0:
            e["floorContact"] += 0.5 * floor_k * dist * dist
            gfl[1] = floor_k * dist
            H[v, 1, 1] += floor_k
        grad[v] = gi + gf + gt + g_el[v] + gfl
        e["inertia"] += 0.5 * w[v] * d @ d
        e["externalForce"] += -forces[v] @ x[v]
        e["quadraticTarget"] += 0.5 * targets[v, 3] * (x[v] - targets[v, :3]) @ (x[v] - targets[v, :3])
        sq["inertia"] += gi @ gi
        sq["material"] += g_el[v] @ g_el[v]
        sq["externalForce"] += gf @ gf
        sq["target"] += gt @ gt
        sq["contact"] += gfl @ gfl
    return e, {k: np.sqrt(v) for k, v in sq.items()}, grad, H, tet_e, tet_det, active


@pytest.mark.gpu
def test_oracle_diagnostics_match_a_float64_restatement():
    inp = scenes.cantilever(cells=(6, 2, 2), size=(0.6, 0.2, 0.2), cubature_k=6)
    rest = inp.positions.reshape(-1, 4)[:, :3]
    # The bottom row starts inside the floor; the height is the f32 value the
    # device compares against, so both sides decide floor contact alike.
    floor_height = float(np.float32(float(rest[:, 1].min()) + 0.01))
    settings = dict(timestep=1 / 60, floorHeight=floor_height, floorStiffness=2e4, parityMode=True)
    gpu = solver.JGS2GpuSolver.create(inp, settings)
    V = inp.vertex_count
    free = np.flatnonzero(inp.vertex_info.reshape(-1, 4)[:, 2] == 0)
    f_vertex, t_vertex = int(free[-1]), int(free[len(free) // 2])
    gpu.setExternalForce(f_vertex, (0.0, 3.0, -1.0))
    gpu.setQuadraticTarget(t_vertex, rest[t_vertex] + np.array([0.0, 0.05, 0.0]), 500.0)
    for _ in range(3):
        gpu.stepExactIterations(10)
    d = gpu.readOracleDiagnostics()
    x = gpu.readPositions().reshape(-1, 4)[:, :3].astype(np.float64)
    pred = gpu.readPredictedPositions().reshape(-1, 4)[:, :3].astype(np.float64)
    forces = np.zeros((V, 3))
    forces[f_vertex] = (0.0, 3.0, -1.0)
    targets = np.zeros((V, 4))
    targets[t_vertex, :3] = np.float32(rest[t_vertex] + np.array([0.0, 0.05, 0.0]))
    targets[t_vertex, 3] = 500.0
    e, norms, grad, H, tet_e, tet_det, active = _reference(inp, x, pred, 1 / 60, forces, targets, floor_height, 2e4)

    for k, ref in e.items():
        assert d["components"][k] == pytest.approx(ref, rel=1e-4, abs=1e-6), k
    assert d["energy"] == pytest.approx(sum(e.values()), rel=1e-4, abs=1e-6)
    for k, ref in norms.items():
        assert d["componentGradientNorms"][k] == pytest.approx(ref, rel=1e-3, abs=1e-5), k
    rec = d["vertexRecords"]
    gscale = np.abs(grad[active]).max()
    assert np.abs(rec[active, 0, :3] - grad[active]).max() <= 1e-4 * gscale + 1e-5
    hblock = rec[:, 1:4, :3]  # row-major rows of the block
    hscale = np.abs(H[active]).max()
    herr = np.abs(hblock[active] - H[active]).max(axis=(1, 2))
    assert herr.max() <= 1e-4 * hscale, (herr.max() / hscale, np.flatnonzero(active)[herr.argmax()])
    assert (rec[~active, 0, 3] == 0).all() and (rec[active, 0, 3] == 1).all()
    # f32 evaluation of a tet's energy cancels terms of size vol (3 mu + lambda)
    # (I1 is near 3 and J near 1 close to rest): allow one rounding of that.
    meta = inp.tet_meta.reshape(-1, 4).astype(np.float64)
    cancel = 2.0 ** -24 * meta[:, 0] * (3 * meta[:, 2] + meta[:, 1])
    assert (np.abs(d["tetRecords"][:, 0] - tet_e) <= 1e-3 * np.abs(tet_e) + cancel).all()
    np.testing.assert_allclose(d["tetRecords"][:, 1], tet_det, rtol=1e-5)
    assert d["minimumDeformationDeterminant"] == pytest.approx(tet_det.min(), rel=1e-5)
    updates = gpu.readFinalIterationUpdates().reshape(V, -1)[:, 0]  # (magnitude, 0, 0, valid) per vertex
    assert d["maximumUpdate"] == pytest.approx(float(updates[active].max()), rel=1e-6)
    assert d["activeVertexCount"] == int(active.sum())
    bottom = active & (x[:, 1] < floor_height)
    assert d["activeContactCount"] == int(bottom.sum()) > 0
    assert d["minimumContactDistanceValid"]
    assert d["minimumContactDistance"] == pytest.approx(float((x[active, 1] - floor_height).min()), abs=1e-6)
    assert d["finite"] and d["gradientValid"] and d["relativeResidualValid"]
    denom = max(1.0, sum(norms.values()))
    assert d["relativeResidual"] == pytest.approx(np.linalg.norm(grad[active]) / denom, rel=1e-3)
    # A second read of the unchanged state gives the same numbers.
    d2 = gpu.readOracleDiagnostics()
    assert d2["energy"] == d["energy"] and np.array_equal(d2["vertexRecords"], rec)
    gpu.destroy()


@pytest.mark.gpu
def test_oracle_diagnostics_refuse_ipc_contact():
    inp = scenes.trough(1)
    gpu = solver.JGS2GpuSolver.create(inp, scenes.TROUGH_SETTINGS)
    gpu.step()
    with pytest.raises(solver.JGS2RangeError, match="do not yet include IPC contact energy"):
        gpu.readOracleDiagnostics()
    gpu.step({"ipcBarrierStiffness": 0.0})
    assert gpu.readOracleDiagnostics()["finite"]
    gpu.destroy()

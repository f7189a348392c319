"""The precompute's exact vertex bases against a float64 numpy restatement of
the reference's computeExactVertexBasis (src/simulation/cpu/precompute.ts:
141-222) over the assembled rest system (src/simulation/cpu/fem.ts:240-335).

The rest system is H = K + M / h^2 over the movable vertices. K is the
assembled linear (Hooke) element stiffness, which the stable Neo-Hookean
tangent equals at rest. For a source vertex s, the basis is
B = H^-1 S (S^T H^-1 S)^-1, with S selecting s's three coordinates.
Vertex u's block is B's rows for u: the identity at u = s, zero at pinned
vertices. With the exact complement, every record of s holds the blocks of
its tetrahedron's four vertices, row-major, row = u's coordinate and
column = the source direction.
"""
import numpy as np

from jgs2_b200 import scenes

TIMESTEP = 1 / 60
YOUNG, POISSON, DENSITY = 1e5, 0.4, 1000.0
EMPTY = 0xFFFFFFFF


def _bar():
    sc = scenes.Scene()
    m = sc.add_material(DENSITY, YOUNG, POISSON)
    sc.add_cuboid((3, 2, 2), (0.0, 0.0, 0.0), (0.3, 0.2, 0.2), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=TIMESTEP, cubature_k=sc.tet_count, exact_complement=1, method=scenes.PRECOMPUTE_EXACT)
    return sc.pack(), sc.rest_positions().astype(np.float64)


def _rest_system(inp, rest):
    V = inp.vertex_count
    tets = inp.tet_indices.reshape(-1, 4).astype(np.int64)
    pinned = inp.vertex_info.reshape(-1, 4)[:, 2] != 0
    mass = inp.vertex_rest.reshape(-1, 4)[:, 3].astype(np.float64)
    mu = YOUNG / (2 * (1 + POISSON))
    lam = YOUNG * POISSON / ((1 + POISSON) * (1 - 2 * POISSON))
    active = np.flatnonzero(~pinned)
    dof = -np.ones(V, dtype=np.int64)
    dof[active] = 3 * np.arange(len(active))
    n = 3 * len(active)
    H = np.zeros((n, n))
    for t in tets:
        dm = np.stack([rest[t[k]] - rest[t[0]] for k in (1, 2, 3)], axis=1)
        vol = abs(np.linalg.det(dm)) / 6.0
        g = np.linalg.inv(dm)  # rows: shape gradients of vertices 1..3
        grads = np.vstack([-g.sum(axis=0), g])
        for a in range(4):
            if dof[t[a]] < 0:
                continue
            for b in range(4):
                if dof[t[b]] < 0:
                    continue
                ga, gb = grads[a], grads[b]
                blk = vol * (mu * (ga @ gb) * np.eye(3) + mu * np.outer(gb, ga) + lam * np.outer(ga, gb))
                H[dof[t[a]]:dof[t[a]] + 3, dof[t[b]]:dof[t[b]] + 3] += blk
    H[np.arange(n), np.arange(n)] += np.repeat(mass[active], 3) / TIMESTEP ** 2
    return H, dof


def test_exact_bases_match_the_restated_rest_system():
    inp, rest = _bar()
    H, dof = _rest_system(inp, rest)
    Hinv = np.linalg.inv(H)
    K = inp.cubature_k
    tets = inp.tet_indices.reshape(-1, 4)
    worst, checked = 0.0, 0
    for s in range(inp.vertex_count):
        if dof[s] < 0:
            continue
        cols = Hinv[:, dof[s]:dof[s] + 3]
        basis = cols @ np.linalg.inv(0.5 * (cols[dof[s]:dof[s] + 3] + cols[dof[s]:dof[s] + 3].T))
        for r in range(s * K, (s + 1) * K):
            t = int(inp.cubature_tet_ids[r])
            if t == EMPTY:
                continue
            blocks = inp.cubature_basis[36 * r:36 * r + 36].reshape(4, 3, 3).astype(np.float64)
            for l in range(4):
                u = int(tets[t, l])
                want = np.zeros((3, 3)) if dof[u] < 0 else basis[dof[u]:dof[u] + 3]
                worst = max(worst, float(np.abs(blocks[l] - want).max()))
                checked += 1
    print(f"exact bases: {checked} blocks, max deviation {worst:.2e}")
    assert checked > 0
    # f32 storage of entries of order one.
    assert worst < 5e-7


def test_corotated_rest_stiffness_is_symmetric_and_translation_free():
    # precompute.test.ts:296-332: every element's linear rest stiffness is
    # symmetric, annihilates rigid translations, and equals the Hooke
    # element matrix of its rest geometry.
    sc = scenes.Scene()
    m = sc.add_material(DENSITY, YOUNG, POISSON, scenes.MATERIAL_COROTATED_LINEAR)
    sc.add_cuboid((2, 2, 1), (0.0, 0.0, 0.0), (0.2, 0.2, 0.1), m, 0, scenes.FACE_X_MIN)
    sc.precompute(timestep=TIMESTEP, cubature_k=sc.tet_count, exact_complement=1)
    inp = sc.pack()
    rest = sc.rest_positions().astype(np.float64)
    Ks = inp.tet_rest_stiffness.reshape(-1, 12, 12).astype(np.float64)
    tets = inp.tet_indices.reshape(-1, 4).astype(np.int64)
    mu = YOUNG / (2 * (1 + POISSON))
    lam = YOUNG * POISSON / ((1 + POISSON) * (1 - 2 * POISSON))
    for t, K in zip(tets, Ks):
        scale = np.abs(K).max()
        assert np.abs(K - K.T).max() <= 1e-6 * scale
        for axis in range(3):
            shift = np.zeros(12)
            shift[axis::3] = 1.0
            assert np.abs(K @ shift).max() <= 1e-6 * scale
        dm = np.stack([rest[t[k]] - rest[t[0]] for k in (1, 2, 3)], axis=1)
        vol = abs(np.linalg.det(dm)) / 6.0
        g = np.linalg.inv(dm)
        grads = np.vstack([-g.sum(axis=0), g])
        want = np.zeros((12, 12))
        for a in range(4):
            for b in range(4):
                ga, gb = grads[a], grads[b]
                want[3 * a:3 * a + 3, 3 * b:3 * b + 3] = vol * (mu * (ga @ gb) * np.eye(3) + mu * np.outer(gb, ga)
                                                               + lam * np.outer(ga, gb))
        assert np.abs(K - want).max() <= 1e-6 * scale

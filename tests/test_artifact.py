"""Fingerprinted precomputation artifacts (the reference's rules,
src/reproducibility/precomputation-artifact.ts:9-160): a cached input is
reused only when every input component's fingerprint matches and the payload
is intact; any changed option invalidates it."""
import json

import numpy as np
import pytest

from jgs2_b200 import artifact, scenes


def _build(calls, **kw):
    def build():
        calls.append(kw)
        return scenes.unit_cube(cells=3, **kw)
    return build


def test_fingerprints_are_canonical():
    a = artifact.fingerprint({"b": 1, "a": [1.0, np.arange(3, dtype=np.uint32)]})
    b = artifact.fingerprint({"a": [1.0, np.arange(3, dtype=np.uint32)], "b": 1})
    assert a == b and a.startswith("sha256:") and len(a) == 71
    # Array kind, shape and float bits all count.
    assert artifact.fingerprint(np.arange(3, dtype=np.uint32)) != artifact.fingerprint(np.arange(3, dtype=np.int32))
    assert artifact.fingerprint(np.zeros((2, 3))) != artifact.fingerprint(np.zeros((3, 2)))
    assert artifact.fingerprint(0.1) != artifact.fingerprint(0.1 + 1e-17 * 8)
    assert artifact.fingerprint(1) != artifact.fingerprint(1.0)


def test_cached_input_reused_only_for_the_same_inputs(tmp_path):
    calls = []
    comps = scenes.unit_cube_components(cells=3)
    a, reused = scenes.cached_input(str(tmp_path), "cube3", comps, _build(calls))
    assert not reused and len(calls) == 1
    b, reused = scenes.cached_input(str(tmp_path), "cube3", comps, _build(calls))
    assert reused and len(calls) == 1
    for k, v in a.arrays().items():
        np.testing.assert_array_equal(v, b.arrays()[k], err_msg=k)
    # Each changed option changes its component and misses the cache.
    for change, component in ((dict(cubature_k=4), "cubature"), (dict(young=2e6), "materials"),
                              (dict(patch_radius=1), "basis"), (dict(timestep=1 / 120), "timestep"),
                              (dict(seed=7), "topology")):
        other = scenes.unit_cube_components(cells=3, **change)
        pa, pb = artifact.fingerprints(comps), artifact.fingerprints(other)
        assert [c for c in artifact.COMPONENTS if pa[c] != pb[c]] == [component], change
        _, reused = scenes.cached_input(str(tmp_path), "cube3", other, _build(calls, **change))
        assert not reused


def test_stale_or_corrupt_artifacts_are_rejected(tmp_path):
    comps = scenes.unit_cube_components(cells=3)
    prints = artifact.fingerprints(comps)
    inp = scenes.unit_cube(cells=3)
    path = str(tmp_path / "a.npz")
    artifact.save(path, inp, prints)
    assert artifact.load(path, prints, scenes.SceneInput).vertex_count == inp.vertex_count
    other = artifact.fingerprints(scenes.unit_cube_components(cells=3, cubature_k=4))
    with pytest.raises(artifact.ArtifactMismatch, match="cubature"):
        artifact.load(path, other, scenes.SceneInput)
    # A payload changed after the fact fails its fingerprint.
    with np.load(path) as z:
        data = {k: z[k] for k in z.files}
    data["positions"] = data["positions"].copy()
    data["positions"][0] += 1.0
    np.savez(path, **data)
    with pytest.raises(artifact.ArtifactMismatch, match="payload"):
        artifact.load(path, prints, scenes.SceneInput)
    # An unknown schema is refused.
    header = json.loads(str(data["__header"]))
    header["schema"] = "something.else"
    data["__header"] = np.array(json.dumps(header))
    np.savez(path, **data)
    with pytest.raises(artifact.ArtifactMismatch, match="schema"):
        artifact.load(path, prints, scenes.SceneInput)


def test_trainer_revision_is_fingerprinted(monkeypatch):
    # A change to the training arithmetic (its revision) changes the cubature
    # fingerprint alone, so caches made by an earlier trainer are not reused.
    before = artifact.fingerprints(scenes.unit_cube_components(cells=3))
    monkeypatch.setattr(scenes, "TRAINER_REVISION", scenes.TRAINER_REVISION + 1)
    after = artifact.fingerprints(scenes.unit_cube_components(cells=3))
    assert [c for c in artifact.COMPONENTS if before[c] != after[c]] == ["cubature"]

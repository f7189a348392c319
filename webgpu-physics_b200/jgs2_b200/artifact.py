"""Fingerprinted precomputation artifacts.

The precompute (rest data, bases, cubature training) is the slow part of
building a step input; it is kept on disk and reused only when it was made
from the same inputs.  This restates the reference's artifact rules
(src/reproducibility/precomputation-artifact.ts:9-160): a header with a
schema name and version, the producer, one SHA-256 fingerprint per input
component (topology, materials, timestep, basis, cubature, solver schedule)
over a canonical encoding (sorted keys, array kinds and shapes included), and
the payload's byte length and fingerprint.  Fingerprints detect stale or
incompatible artifacts; they are not a trust mechanism.

The payload is a SceneInput's arrays in an .npz file; the header sits in the
same file as a JSON string.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

SCHEMA = "org.jgs2.precomputation-artifact"
SCHEMA_VERSION = 1
PAYLOAD_FORMAT = "jgs2-b200-npz"
PAYLOAD_FORMAT_VERSION = 1
COMPONENTS = ("topology", "materials", "timestep", "basis", "cubature", "solverSchedule")
PRODUCER = {"name": "jgs2_b200", "version": "1"}


class ArtifactMismatch(ValueError):
    """The artifact is missing, malformed, or made from other inputs."""


def _canonical(value) -> bytes:
    """Deterministic encoding: dict keys sorted, arrays tagged with dtype and
    shape, floats by their exact bits (so 0.1 and 0.1000000001 differ)."""
    if isinstance(value, dict):
        parts = [b"{"]
        for k in sorted(value):
            parts += [json.dumps(str(k)).encode(), b":", _canonical(value[k]), b","]
        return b"".join(parts + [b"}"])
    if isinstance(value, (list, tuple)):
        return b"[" + b",".join(_canonical(v) for v in value) + b"]"
    if isinstance(value, np.ndarray):
        a = np.ascontiguousarray(value)
        head = f"ndarray<{a.dtype.str}>{list(a.shape)}:".encode()
        return head + hashlib.sha256(a.tobytes()).hexdigest().encode()
    if isinstance(value, (bool, np.bool_)):
        return b"true" if value else b"false"
    if isinstance(value, (int, np.integer)):
        return f"i{int(value)}".encode()
    if isinstance(value, (float, np.floating)):
        return f"f{float(value).hex()}".encode()
    if value is None:
        return b"null"
    return json.dumps(str(value)).encode()


def fingerprint(value) -> str:
    return "sha256:" + hashlib.sha256(_canonical(value)).hexdigest()


def fingerprints(components: dict) -> dict:
    """One fingerprint per component; every component must be given."""
    missing = [c for c in COMPONENTS if c not in components]
    if missing:
        raise ValueError(f"fingerprint components missing: {missing}")
    return {c: fingerprint(components[c]) for c in COMPONENTS}


def cache_name(prefix: str, prints: dict) -> str:
    """A file name keyed by all component fingerprints."""
    digest = hashlib.sha256("".join(prints[c] for c in COMPONENTS).encode()).hexdigest()[:24]
    return f"{prefix}-{digest}.npz"


def _payload(arrays: dict) -> str:
    return fingerprint({k: arrays[k] for k in sorted(arrays)})


def save(path: str, scene_input, prints: dict) -> None:
    arrays = scene_input.arrays()
    nbytes = int(sum(np.asarray(a).nbytes for a in arrays.values()))
    header = {"schema": SCHEMA, "schemaVersion": SCHEMA_VERSION, "createdBy": PRODUCER,
              "fingerprints": dict(prints),
              "payload": {"format": PAYLOAD_FORMAT, "formatVersion": PAYLOAD_FORMAT_VERSION,
                          "byteLength": nbytes, "fingerprint": _payload(arrays)}}
    tmp = path + ".tmp.npz"
    np.savez(tmp, __header=np.array(json.dumps(header, sort_keys=True)), **arrays)
    os.replace(tmp, path)


def validate_header(header) -> dict:
    """Check an untrusted header's shape and versions (the reference's
    validatePrecomputationArtifactHeader)."""
    if not isinstance(header, dict):
        raise ArtifactMismatch("precomputation artifact header must be an object")
    if header.get("schema") != SCHEMA:
        raise ArtifactMismatch(f"unsupported precomputation schema {header.get('schema')!r}; expected {SCHEMA}")
    if header.get("schemaVersion") != SCHEMA_VERSION:
        raise ArtifactMismatch(f"unsupported schema version {header.get('schemaVersion')!r}")
    prints = header.get("fingerprints")
    if not isinstance(prints, dict) or sorted(prints) != sorted(COMPONENTS):
        raise ArtifactMismatch("artifact fingerprints must name exactly the components " + ", ".join(COMPONENTS))
    for c, v in prints.items():
        if not (isinstance(v, str) and v.startswith("sha256:") and len(v) == 71):
            raise ArtifactMismatch(f"fingerprint {c} is not a sha256 digest")
    payload = header.get("payload")
    if not isinstance(payload, dict) or payload.get("format") != PAYLOAD_FORMAT or \
            payload.get("formatVersion") != PAYLOAD_FORMAT_VERSION:
        raise ArtifactMismatch("unsupported payload format")
    return header


def load(path: str, expected: dict, scene_input_cls):
    """The artifact at `path` if it was made from `expected` fingerprints and
    its payload is intact; ArtifactMismatch otherwise."""
    if not os.path.exists(path):
        raise ArtifactMismatch(f"no artifact at {path}")
    try:
        with np.load(path, allow_pickle=False) as z:
            header = json.loads(str(z["__header"]))
            arrays = {k: z[k] for k in z.files if k != "__header"}
    except ArtifactMismatch:
        raise
    except Exception as e:  # unreadable or truncated file
        raise ArtifactMismatch(f"unreadable artifact {path}: {e}") from e
    header = validate_header(header)
    stale = [c for c in COMPONENTS if header["fingerprints"][c] != expected[c]]
    if stale:
        raise ArtifactMismatch(f"artifact made from other inputs (changed: {', '.join(stale)})")
    nbytes = int(sum(a.nbytes for a in arrays.values()))
    if nbytes != header["payload"]["byteLength"] or _payload(arrays) != header["payload"]["fingerprint"]:
        raise ArtifactMismatch("artifact payload does not match its fingerprint")
    return scene_input_cls.from_arrays(arrays)

"""Test configuration: the `gpu` marker and import paths.

Tests marked gpu need a CUDA device (they run on a B200); every other test
runs on CPU only.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, "webgpu-physics_b200")):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _native_libraries():
    """Build the native libraries once per session if they are missing."""
    from jgs2_b200 import build

    build.build_all()
    import subprocess

    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    yield

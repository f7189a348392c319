"""The checked build (device index checks compiled in, JGS2_BOUNDS_CHECKS=1,
the stand-in for compute-sanitizer, which is closed on this hardware pool):
the same scenes stepped with it and with the default library must raise no
failed check and agree to f32 rounding (the checks only add branches)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(os.path.dirname(HERE), "webgpu-physics_b200", "lib")


def _run(tmp_path, name, lib_dir):
    out = str(tmp_path / f"{name}.npz")
    env = dict(os.environ, JGS2_LIB_DIR=lib_dir)
    res = subprocess.run([sys.executable, os.path.join(HERE, "checked_run.py"), out], env=env,
                         capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-3000:]
    return np.load(out)


def test_checked_build_passes_every_scene_and_agrees(tmp_path):
    assert os.path.exists(os.path.join(LIB, "checked", "libjgs2.so"))
    plain = _run(tmp_path, "plain", LIB)
    checked = _run(tmp_path, "checked", os.path.join(LIB, "checked"))
    for key in plain.files:
        if key.endswith("_diag"):
            continue
        err = float(np.abs(plain[key] - checked[key]).max()) / float(plain[key + "_diag"][0])
        assert err <= 1e-5, (key, err)

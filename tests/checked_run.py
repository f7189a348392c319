"""Steps a fixed set of scenes and saves their final positions: run once with
the default library and once with the checked one (JGS2_LIB_DIR), by
tests/test_bounds_checked.py.  argv: output .npz path."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "webgpu-physics_b200"))

import numpy as np  # noqa: E402

from jgs2_b200 import scenes, solver  # noqa: E402


def main(out):
    bar = scenes.cantilever(cells=(10, 2, 2), size=(0.5, 0.1, 0.1))
    runs = {
        "bar_jacobi": (bar, dict(timestep=1 / 60), lambda s: s.stepFrames(4)),
        "bar_ggs2": (bar, dict(timestep=1 / 60, schedule=1), lambda s: s.stepFrames(4)),
        "trough_static": (scenes.trough(3), dict(scenes.TROUGH_SETTINGS), lambda s: s.stepFrames(20)),
        "boxes_surface": (scenes.box_trough(boxes=2, cells=3, heights=(1.0, 1.3), plate_cells=(8, 2),
                                            method=scenes.PRECOMPUTE_PATCH), dict(scenes.BOX_TROUGH_SETTINGS),
                          lambda s: s.stepFramesExactIterations(10, 15)),
        "cloth": (scenes.cloth_drape(cells=6, prefold=False, pinned_columns=(0, 6)), dict(timestep=1 / 120),
                  lambda s: s.stepFrames(6)),
        "cube_records": (scenes.unit_cube(cells=8), dict(timestep=1 / 60, parityMode=True),
                         lambda s: s.stepFramesExactIterations(2, 20)),
    }
    saved = {}
    for name, (inp, settings, step) in runs.items():
        s = solver.JGS2GpuSolver.create(inp, settings)
        step(s)
        saved[name] = s.readPositions()  # a checked build raises here on a failed index check
        saved[name + "_diag"] = np.array([inp.bbox_diagonal()])
        s.destroy()
    np.savez(out, **saved)


if __name__ == "__main__":
    main(sys.argv[1])

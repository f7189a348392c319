"""The greedy cubature selection on the GPU (select_gpu.cu) against the CPU
trainer: the same training problems, selected by one thread block each on
the device, write the same records bit for bit (tets, weights, bases) and the
same residuals, for the patch and whole-mesh methods, the stable Neo-Hookean
and co-rotated trainings, the 12-column kernel width and the small-mesh
subset audit.  The selection rounds identically on both sides because the
host and device code share cubature_select.hpp and neither contracts
multiply-adds."""
import numpy as np
import pytest

from jgs2_b200 import scenes

pytestmark = pytest.mark.gpu


def _cuboid(cells, size, faces, k, method, model=scenes.MATERIAL_STABLE_NEO_HOOKEAN, poisson=0.45,
            device=scenes.SELECTION_CPU, **extra):
    sc = scenes.Scene()
    m = sc.add_material(1000.0, 1e6, poisson, model)
    sc.add_cuboid(cells, (0.0, 0.0, 0.0), size, m, 0, faces)
    st = sc.precompute(timestep=1 / 60, cubature_k=k, method=method, selection_device=device, **extra)
    return st, sc.pack().arrays()


CASES = {
    "patch cube 8^3, K=6": dict(cells=(8, 8, 8), size=(1.0, 1.0, 1.0), faces=scenes.FACE_Y_MIN, k=6,
                                method=scenes.PRECOMPUTE_PATCH),
    "whole-mesh bar, K=6": dict(cells=(6, 2, 2), size=(0.6, 0.2, 0.2), faces=scenes.FACE_X_MIN, k=6,
                                method=scenes.PRECOMPUTE_EXACT),
    "co-rotated bar, K=6": dict(cells=(5, 2, 2), size=(0.5, 0.2, 0.2), faces=scenes.FACE_X_MIN, k=6,
                                method=scenes.PRECOMPUTE_EXACT, model=scenes.MATERIAL_COROTATED_LINEAR,
                                poisson=0.3),
    "one hex, K=4 (subset audit)": dict(cells=(1, 1, 1), size=(0.1, 0.1, 0.1), faces=scenes.FACE_Y_MIN, k=4,
                                        method=scenes.PRECOMPUTE_EXACT),
    "patch bar, K=10 (12-wide kernel)": dict(cells=(6, 3, 3), size=(0.6, 0.3, 0.3), faces=scenes.FACE_X_MIN,
                                             k=10, method=scenes.PRECOMPUTE_PATCH, patch_radius=1),
}


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_selection_writes_the_cpu_records(name):
    cpu_st, cpu = _cuboid(**CASES[name], device=scenes.SELECTION_CPU)
    gpu_st, gpu = _cuboid(**CASES[name], device=scenes.SELECTION_GPU)
    assert cpu_st["selection_on_gpu"] == 0 and gpu_st["selection_on_gpu"] == 1
    assert gpu_st["selection_batches"] >= 1
    assert sorted(cpu) == sorted(gpu)
    for key in cpu:
        np.testing.assert_array_equal(gpu[key], cpu[key], err_msg=key)
    for key in ("max_residual", "mean_residual", "records_written", "vertices_over_tolerance"):
        assert gpu_st[key] == cpu_st[key], key


def test_gpu_selection_many_classes_in_one_batch():
    # 20^3 cube: a few hundred patch classes selected in one launch.
    cpu_st, cpu = _cuboid((20, 20, 20), (1.0, 1.0, 1.0), scenes.FACE_Y_MIN, 6, scenes.PRECOMPUTE_PATCH)
    gpu_st, gpu = _cuboid((20, 20, 20), (1.0, 1.0, 1.0), scenes.FACE_Y_MIN, 6, scenes.PRECOMPUTE_PATCH,
                          device=scenes.SELECTION_GPU)
    assert gpu_st["training_classes"] > 100
    for key in cpu:
        np.testing.assert_array_equal(gpu[key], cpu[key], err_msg=key)
    assert gpu_st["max_residual"] == cpu_st["max_residual"]


def test_auto_selects_the_gpu():
    st, _ = _cuboid((3, 2, 2), (0.3, 0.2, 0.2), scenes.FACE_X_MIN, 6, scenes.PRECOMPUTE_EXACT,
                    device=scenes.SELECTION_AUTO)
    assert st["selection_on_gpu"] == 1


def test_gpu_selection_in_several_batches(monkeypatch):
    # A small batch budget splits the classes (and the whole-mesh sources)
    # over several launches; each class keeps its own records.
    # Two threads build 8 jobs per group, so the budget closes a batch every
    # group or two.
    monkeypatch.setenv("JGS2_SELECTION_BATCH_BYTES", str(1 << 20))
    for case in ("patch cube 8^3, K=6", "whole-mesh bar, K=6"):
        cpu_st, cpu = _cuboid(**CASES[case], device=scenes.SELECTION_CPU, threads=2)
        gpu_st, gpu = _cuboid(**CASES[case], device=scenes.SELECTION_GPU, threads=2)
        assert gpu_st["selection_batches"] > 1, case
        for key in cpu:
            np.testing.assert_array_equal(gpu[key], cpu[key], err_msg=f"{case}: {key}")
        assert gpu_st["max_residual"] == cpu_st["max_residual"]

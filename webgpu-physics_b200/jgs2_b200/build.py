"""Build recipe of the native libraries (in-tree, into webgpu-physics_b200/lib).

  libjgs2.so        CUDA step for sm_100a + the C-ABI runtime (include/jgs2.h)
  checked/libjgs2.so  the same with device index checks (JGS2_BOUNDS_CHECKS=1)
  libjgs2_scene.so  scene builder / precompute, with the GPU cubature selection
                    (include/jgs2_scene.h)

Run as `python -m jgs2_b200.build` from webgpu-physics_b200/ or through
__graft_entry__.build().  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO_ROOT = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
LIB = os.path.join(PKG_ROOT, "lib")
INCLUDE = os.path.join(REPO_ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # The system g++ carries libgomp; an overriding $CXX may not.
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}): {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return res


def _stale(target, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


CHECKED_LIB = os.path.join(LIB, "checked")


def build_step_library(force=False, verbose=False, checked=False) -> str:
    """libjgs2.so; `checked` builds the variant with device index checks
    (JGS2_BOUNDS_CHECKS=1) into lib/checked/."""
    out_dir = CHECKED_LIB if checked else LIB
    os.makedirs(out_dir, exist_ok=True)
    target = os.path.join(out_dir, "libjgs2.so")
    sources = [os.path.join(CSRC, f) for f in ("jgs2_kernels.cu", "jgs2_runtime.cpp", "jgs2_server.cpp")]
    headers = [os.path.join(CSRC, f) for f in ("jgs2_kernels.cuh", "jgs2_device.cuh", "jgs2_cloth.cuh",
                                                "jgs2_contact.cuh")] + [
        os.path.join(INCLUDE, f) for f in ("jgs2.h", "jgs2_server.h")]
    if not force and not _stale(target, sources + headers):
        return target
    nvcc = _nvcc()
    objs, cmds = [], []
    for src in sources:
        obj = os.path.join(out_dir, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-pthread", "-I", INCLUDE,
               "-I", CSRC, *(["-DJGS2_BOUNDS_CHECKS=1"] if checked else []), "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd.insert(1, "-x")
            cmd.insert(2, "cu")
        cmds.append(cmd)
        objs.append(obj)
    # The translation units compile in parallel.
    with concurrent.futures.ThreadPoolExecutor(len(cmds)) as pool:
        list(pool.map(lambda c: _run(c, verbose), cmds))
    _run([nvcc, *ARCH, "-shared", "-o", target, *objs, "-lcudart", "-Xcompiler", "-pthread"], verbose)
    for obj in objs:
        os.remove(obj)
    return target


def build_scene_library(force=False, verbose=False) -> str:
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libjgs2_scene.so")
    sdir = os.path.join(CSRC, "scene")
    sources = [os.path.join(sdir, f) for f in ("scene.cpp", "precompute.cpp", "select_gpu.cu")]
    headers = [os.path.join(sdir, f) for f in ("scene_internal.hpp", "cubature_select.hpp", "select_gpu.hpp")] + [
        os.path.join(INCLUDE, "jgs2_scene.h"), os.path.join(INCLUDE, "jgs2.h")]
    if not force and not _stale(target, sources + headers):
        return target
    nvcc, cxx = _nvcc(), _cxx()
    # The cubature selection must round identically on the CPU and the GPU:
    # no multiply-add contraction in the host code (-ffp-contract=off) nor in
    # the device code (--fmad=false).
    objs, cmds = [], []
    for src in sources:
        obj = os.path.join(LIB, "scene_" + os.path.basename(src) + ".o")
        if src.endswith(".cu"):
            cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
                   "-I", INCLUDE, "-I", sdir, "-c", src, "-o", obj]
        else:
            cmd = [cxx, "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-std=c++17",
                   "-I", INCLUDE, "-I", sdir, "-c", src, "-o", obj]
        cmds.append(cmd)
        objs.append(obj)
    with concurrent.futures.ThreadPoolExecutor(len(cmds)) as pool:
        list(pool.map(lambda c: _run(c, verbose), cmds))
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "lib64")
    _run([cxx, "-shared", "-fopenmp", "-o", target, *objs, "-L", cuda_lib, "-lcudart"], verbose)
    for obj in objs:
        os.remove(obj)
    return target


def build_all(force=False, verbose=False):
    with concurrent.futures.ThreadPoolExecutor(3) as pool:
        jobs = [pool.submit(build_step_library, force, verbose), pool.submit(build_scene_library, force, verbose),
                pool.submit(build_step_library, force, verbose, True)]
        step, scene, checked = (j.result() for j in jobs)
    # The checked directory is a complete library directory (JGS2_LIB_DIR).
    dst = os.path.join(CHECKED_LIB, "libjgs2_scene.so")
    if not os.path.exists(dst) or os.path.getmtime(dst) < os.path.getmtime(scene):
        shutil.copy2(scene, dst)
    return [step, scene, checked]


if __name__ == "__main__":
    for path in build_all(force="--force" in sys.argv, verbose=True):
        print(path)

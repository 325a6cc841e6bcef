"""Builds the native libraries of the luvas3d package in-tree.

    python luvas.io-3d_b200/build.py            # libluvas3d.so (CUDA, sm_100a) + libl3dscene.so

libluvas3d.so is compiled for sm_100a only.  --fmad=false keeps nvcc from fusing multiplies and
adds on its own: every fused multiply-add in the kernels is an explicit fmaf, which is what makes
the plain FP32 form reproducible bit for bit on the CPU.  The host compiler gets
-ffp-contract=off for the same reason (the dispatch parameters are composed in FP64 on the host).
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "luvas3d", "lib")

CUDA_SOURCES = ["capi.cu", "stereo.cu", "stereo_fast.cu", "tsdf.cu", "noalloc.cu", "grad.cu", "cloud.cu", "scan.cu", "mesh.cu", "image.cu", "probe.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-O3",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libluvas3d.so")
    return cand


def _cxx() -> str:
    # the image also carries a g++ under /opt/gcc without OpenMP support; prefer the system one
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False) -> None:
    os.makedirs(LIB, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "luvas3d.h"))
    sources = [os.path.join(CSRC, f) for f in CUDA_SOURCES if os.path.exists(os.path.join(CSRC, f))]
    target = os.path.join(LIB, "libluvas3d.so")
    if force or _stale(target, sources + headers):
        build_dir = os.path.join(HERE, "_build")
        os.makedirs(build_dir, exist_ok=True)
        cmds, objs = [], []
        for src in sources:
            obj = os.path.join(build_dir, os.path.basename(src) + ".o")
            cmd = [_nvcc(), *NVCC_FLAGS, "-c", src, "-o", obj]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
            objs.append(obj)
        # one nvcc per translation unit, in parallel
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
            for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
                f.result()
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", target, *objs,
               "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    scene_src = os.path.join(CSRC, "scene.cpp")
    scene = os.path.join(LIB, "libl3dscene.so")
    if force or _stale(scene, [scene_src, os.path.join(CSRC, "l3d_fmath.h")]):
        cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-o", scene, scene_src]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)

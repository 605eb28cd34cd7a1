"""Builds libhs_bem.so in-tree: host C++20 (mesh validation, planner, session,
C ABI) and the sm_100a CUDA kernels, linked against the static CUDA runtime.

    python -m hornsculpt_b200.build        # or hornsculpt_b200.build.build()
"""
from __future__ import annotations

import concurrent.futures
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIBRARY = PKG / "libhs_bem.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Sources whose floating-point operations must match the host planner's one
# for one: no multiply-add contraction (explicit fma() only).
NO_CONTRACTION = {"plan_device.cu"}


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = shutil.which("nvcc") or os.path.join(cuda, "bin", "nvcc")
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libhs_bem.so")
    return path


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _compile(src: pathlib.Path, verbose_ptxas: bool) -> pathlib.Path:
    obj = BUILD / (src.name + ".o")
    deps = [src] + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    if obj.exists() and obj.stat().st_mtime > max(d.stat().st_mtime for d in deps) and not verbose_ptxas:
        return obj
    cmd = [_nvcc(), "-std=c++20", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I",
           str(CSRC), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu" and verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    if src.name in NO_CONTRACTION:
        cmd += ["-fmad=false"]
    subprocess.run(cmd, check=True)
    return obj


def build(verbose_ptxas: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objs = list(pool.map(lambda s: _compile(s, verbose_ptxas), _sources()))
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIBRARY.with_suffix(".so.tmp")
        subprocess.run([_nvcc(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-lpthread"], check=True)
        tmp.replace(LIBRARY)
    return LIBRARY


ADAPTER = PKG / "adapter"
ADAPTER_BINARY = ADAPTER / "adapter_solve"


def build_adapter(reference: pathlib.Path) -> pathlib.Path:
    """Compiles the reference-side adapter (adapter/cuda_bem_solver_b200.cpp, the
    reference's hornsculpt::CudaBemSolver over this library's C ABI) and its driver
    against the reference's own headers, linked to libhs_bem.so: proof that the
    drop-in builds against the reference interface as it is declared there."""
    includes = sorted((reference / "modules").glob("*/include"))
    if not includes:
        raise RuntimeError(f"no reference include directories under {reference}")
    cmd = [shutil.which("g++") or "g++", "-std=c++20", "-O2", "-Wall", *[f"-I{d}" for d in includes], "-I",
           str(INCLUDE), str(ADAPTER / "cuda_bem_solver_b200.cpp"), str(ADAPTER / "adapter_solve.cpp"), "-L", str(PKG),
           "-lhs_bem", "-Wl,-rpath,$ORIGIN/..", "-o", str(ADAPTER_BINARY)]
    subprocess.run(cmd, check=True)
    return ADAPTER_BINARY


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))

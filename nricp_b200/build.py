"""Builds the CUDA extension in-tree: nricp_b200/libnricp_b200.so for sm_100a.

Plain nvcc, one shared library with a C ABI (include/nricp_b200.h); no torch
extension machinery.  Host C++ is compiled with -ffp-contract=off so the FP64
template graph rounds exactly as the reference's host code does.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libnricp_b200.so"
SOURCES = ["host.cpp", "lbvh.cu", "wrap_kernels.cu", "graph_build.cu", "session.cu", "capi.cu",
           "static_scratch.cu"]
HEADERS = ["common.cuh", "kernels.cuh", "host.hpp", "session.hpp", "graph_build.hpp", "staging.hpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if candidate and (Path(candidate).exists() or candidate == "nvcc"):
            return candidate
    raise FileNotFoundError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [HERE.parent / "include" / "nricp_b200.h"]
    return any(p.stat().st_mtime > built for p in deps)


# A measurement-only variant: the solve's reductions rounded to FP32
# (NRICP_FP32_REDUCTIONS in wrap_kernels.cu), for the precision comparison of
# `bench.py --precision`.  Loaded only when NRICP_B200_LIBRARY points at it.
FP32_REDUCTIONS_LIB = HERE / "variants" / "fp32_reductions" / "libnricp_b200.so"


def build(force: bool = False, verbose: bool = False, defines: tuple = (), lib: Path | None = None,
          build_dir: Path | None = None) -> Path:
    lib = lib or LIB
    if not force and not defines and not _stale():
        return lib
    build_dir = build_dir or HERE / "_build"
    build_dir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(parents=True, exist_ok=True)
    objects = []
    common = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-fopenmp", *[f"-D{d}" for d in defines]]
    for source in SOURCES:
        obj = build_dir / (Path(source).stem + ".o")
        cmd = [nvcc(), *common, "-c", str(CSRC / source), "-o", str(obj)]
        if source.endswith(".cu"):
            cmd[1:1] = ["-x", "cu"]
        if verbose:
            cmd.append("-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = lib.with_suffix(f".so.{os.getpid()}")
    subprocess.run([nvcc(), *ARCH, "-shared", *objects, "-o", str(tmp), "-Xcompiler", "-fopenmp",
                    "-lcudart"], check=True)
    os.replace(tmp, lib)
    return lib


def build_fp32_reductions() -> Path:
    return build(force=True, defines=("NRICP_FP32_REDUCTIONS",), lib=FP32_REDUCTIONS_LIB,
                 build_dir=HERE / "_build_fp32_reductions")


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))

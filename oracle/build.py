"""Build recipes for the oracle -- TEST INFRASTRUCTURE ONLY.

* ``build_oracle()`` compiles the C restatement (nricp_oracle.c +
  block_cholesky.c) into ``oracle/libnricp_oracle.so`` with gcc.
* ``build_reference()`` compiles the reference's own FP64 route A from its
  sources where they lie under the reference checkout (``NRICP_REFERENCE_DIR``,
  default: a ``reference`` directory beside this repository) into ``oracle/_ref/libnricp_ref.so``.  The
  reference needs Eigen 3.4.0, a submodule that is not vendored with it, in two
  translation units: ``src/solver/direct_solve.cpp`` is replaced by
  ``ref/solve_direct.cpp`` (same signature, the block Cholesky restatement) and
  ``src/core/deformation.cpp``'s ``fit_rigid`` compiles against the minimal
  ``ref/eigen_shim/Eigen/Dense``.  ``ref/ref_driver.cpp`` is a C-ABI driver that
  reproduces ``prepare_solve`` (src/python/bindings.cpp:584-672) around the
  reference's ``solve_route_a``.  No reference source is copied.
"""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libnricp_oracle.so"
REF_DIR = HERE / "_ref"
REF_LIB = REF_DIR / "libnricp_ref.so"

_C_SOURCES = ["nricp_oracle.c", "block_cholesky.c"]
_C_FLAGS = ["-O2", "-std=gnu11", "-ffp-contract=off", "-fPIC", "-shared"]

# The reference's host translation units that route A is made of
# (src/core, src/geometry, src/energy, src/solver), minus direct_solve.cpp.
_REF_SOURCES = [
    "core/build_info.cpp",
    "core/constraints.cpp",
    "core/deformation.cpp",
    "core/graph.cpp",
    "core/mesh.cpp",
    "core/report.cpp",
    "core/sampling.cpp",
    "geometry/closest_point.cpp",
    "energy/energy.cpp",
    "energy/robust.cpp",
    "solver/correspondence.cpp",
    "solver/fused_assembly.cpp",
    "solver/normal_equations.cpp",
    "solver/route_a.cpp",
]


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    built = target.stat().st_mtime
    return any(s.stat().st_mtime > built for s in sources if s.exists())


def build_oracle(force: bool = False) -> Path:
    sources = [HERE / s for s in _C_SOURCES]
    deps = sources + [HERE / "nricp_oracle.h", HERE / "block_cholesky.h",
                      HERE.parent / "include" / "nricp_b200.h"]
    if force or _stale(ORACLE_LIB, deps):
        tmp = ORACLE_LIB.with_suffix(f".so.{os.getpid()}")
        cmd = ["gcc", *_C_FLAGS, *map(str, sources), "-o", str(tmp), "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def reference_dir() -> Path:
    """The reference checkout: NRICP_REFERENCE_DIR, else ``reference`` beside
    this repository's root."""
    env = os.environ.get("NRICP_REFERENCE_DIR")
    return Path(env) if env else HERE.parent.parent / "reference"


def build_reference(force: bool = False) -> Path | None:
    """Compile the reference's route A in place; None when it is absent."""
    src = reference_dir() / "src"
    if not (src / "solver" / "route_a.cpp").exists():
        return REF_LIB if REF_LIB.exists() else None
    REF_DIR.mkdir(exist_ok=True)
    ref_sources = [src / s for s in _REF_SOURCES]
    own = [HERE / "ref" / "ref_driver.cpp", HERE / "ref" / "solve_direct.cpp",
           HERE / "block_cholesky.c"]
    deps = ref_sources + own + [HERE / "ref" / "eigen_shim" / "Eigen" / "Dense"]
    if not (force or _stale(REF_LIB, deps)):
        return REF_LIB
    objects = []
    flags = ["-O2", "-ffp-contract=off", "-fPIC"]
    for source in ref_sources + own:
        obj = REF_DIR / (source.parent.name + "_" + source.stem + ".o")
        if source.suffix == ".c":
            cmd = ["gcc", *flags, "-std=gnu11", "-c", str(source), "-o", str(obj)]
        else:
            cmd = ["g++", *flags, "-std=c++20", f"-I{src}",
                   f"-I{HERE / 'ref' / 'eigen_shim'}", f"-I{HERE}",
                   "-c", str(source), "-o", str(obj)]
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = REF_LIB.with_suffix(f".so.{os.getpid()}")
    subprocess.run(["g++", "-shared", *objects, "-o", str(tmp)], check=True)
    os.replace(tmp, REF_LIB)
    for obj in objects:
        Path(obj).unlink()
    return REF_LIB


REF_GPU_LIB = REF_DIR / "libnricp_ref_gpu.so"
_REF_CUDA_SOURCES = ["assemble.cu", "deform_ops.cu", "gpu_level.cu", "gpu_solver.cu", "graph_build.cu",
                     "host_staging.cu", "lbvh.cu", "level_layout.cu", "local_global.cu", "pcg_solver.cu",
                     "session.cu"]


def build_reference_gpu(force: bool = False) -> Path | None:
    """The reference's own GPU routes (src/cuda, compiled for sm_100a with
    nvcc, as its CMake does with --extended-lambda) beside its host sources,
    with this driver's ref_solve_route_b / ref_solve_route_c and
    ref/ref_lbvh.cu's ref_lbvh_build; None when the checkout is absent.  Route
    B is a timed comparison; route C and the hierarchy anchor the FP64 route-C
    and LBVH restatements in the GPU tests."""
    src = reference_dir() / "src"
    if not (src / "cuda" / "gpu_solver.cu").exists():
        return REF_GPU_LIB if REF_GPU_LIB.exists() else None
    REF_DIR.mkdir(exist_ok=True)
    cuda_sources = [src / "cuda" / s for s in _REF_CUDA_SOURCES]
    host_sources = [src / s for s in _REF_SOURCES]
    own = [HERE / "ref" / "ref_driver.cpp", HERE / "ref" / "solve_direct.cpp", HERE / "block_cholesky.c",
           HERE / "ref" / "ref_lbvh.cu"]
    deps = cuda_sources + host_sources + own
    if not (force or _stale(REF_GPU_LIB, deps)):
        return REF_GPU_LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    arch = ["-gencode", "arch=compute_100a,code=sm_100a"]
    objects = []
    for source in cuda_sources + host_sources + own:
        obj = REF_DIR / ("gpu_" + source.parent.name + "_" + source.stem + ".o")
        if source.suffix == ".c":
            cmd = ["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-std=gnu11", "-c", str(source), "-o", str(obj)]
        elif source.suffix == ".cu":
            cmd = [nvcc, *arch, "-O2", "-std=c++20", "--extended-lambda", "-Xcompiler", "-fPIC",
                   f"-I{src}", "-c", str(source), "-o", str(obj)]
        else:
            cmd = ["g++", "-O2", "-ffp-contract=off", "-fPIC", "-std=c++20", "-DNRICP_REF_GPU", f"-I{src}",
                   f"-I{HERE / 'ref' / 'eigen_shim'}", f"-I{HERE}", "-I/usr/local/cuda/include",
                   "-c", str(source), "-o", str(obj)]
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = REF_GPU_LIB.with_suffix(f".so.{os.getpid()}")
    subprocess.run([nvcc, *arch, "-shared", *objects, "-o", str(tmp), "-lcudart"], check=True)
    os.replace(tmp, REF_GPU_LIB)
    for obj in objects:
        Path(obj).unlink()
    return REF_GPU_LIB


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_reference(force=True))
    print(build_reference_gpu(force=True))

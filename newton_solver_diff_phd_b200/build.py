"""Build the sm_100a shared library ``_build/libpdb200.so`` in the package tree.

``python -m newton_solver_diff_phd_b200.build`` compiles every CUDA source for
``sm_100a`` with nvcc and the host factor builder with g++ (no floating-point
contraction: the factor must round each product before its subtraction).
The build is incremental on file modification times.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
INCLUDE = PACKAGE.parent / "include"
BUILD = PACKAGE / "_build"
LIBRARY = BUILD / "libpdb200.so"

CUDA_SOURCES = ("pd_kernels.cu", "pd_adjoint.cu", "pd_solver.cu", "pd_noalloc.cu", "pd_batch.cu", "pd_contact.cu",
                "pd_friction.cu", "pd_woodbury.cu", "pd_diffpd.cu", "pd_factor_device.cu")
HOST_SOURCES = ("factor.cpp", "runs.cpp")
HEADERS = ("factor.h", "runs.h", "pd_math.cuh", "pd_device.cuh", "pd_forward.cuh", "pd_kernels.h", "pd_batch.cuh",
           "pd_team.cuh", "solver_state.h", "pd_geometry.cuh", "pd_friction.cuh")
ARCH = ("-gencode", "arch=compute_100a,code=sm_100a")


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda) / "bin" / "nvcc"
    return str(candidate) if candidate.exists() else (shutil.which("nvcc") or "nvcc")


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > mtime for s in sources)


def _run(command):
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(command)}\n{result.stdout}\n{result.stderr}")
    return result


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile the library if any source is newer than it; return its path."""
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "pd_b200.h"]
    objects = []
    commands = []
    nvcc = _nvcc()
    for source in CUDA_SOURCES:
        obj = BUILD / (source + ".o")
        if force or _stale(obj, [CSRC / source, *headers]):
            commands.append([
                nvcc, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v",
                "-I", str(INCLUDE), "-c", str(CSRC / source), "-o", str(obj),
            ])
        objects.append(obj)
    for source in HOST_SOURCES:
        obj = BUILD / (source + ".o")
        if force or _stale(obj, [CSRC / source, *headers]):
            commands.append(["g++", "-std=c++17", "-O3", "-fPIC", "-ffp-contract=off", "-fno-fast-math",
                             "-c", str(CSRC / source), "-o", str(obj)])
        objects.append(obj)
    # Translation units compile side by side (the slowest one bounds the build).
    with ThreadPoolExecutor(max(1, min(len(commands), os.cpu_count() or 1))) as pool:
        for result in pool.map(_run, commands):
            if verbose:
                print(result.stderr)
    if force or _stale(LIBRARY, objects):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcudart"])
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))

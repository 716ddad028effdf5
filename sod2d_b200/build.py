"""Build recipe for the native libraries of sod2d_b200 (run in-tree).

* ``_lib/libsod2d_host.so``  -- host-side set-up (mesh, GLL tables, Jacobians);
  plain C++, no GPU needed.
* ``_lib/libsod2d_gpu.so``   -- the sm_100a CUDA kernels behind the C-ABI of
  ``include/sod2d_gpu.h``, linked from one object per translation unit
  (``sod2d_gpu.cu`` context and compressible RHS, ``comp_step.cu`` time
  integrators, ``incomp.cu`` incompressible path, ``precond.cu`` learned
  preconditioner, ``noalloc_analysis.cu``).

Both land inside the package directory so they travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
OBJDIR = PKG / "_build"  # object files (not committed)
INCLUDE = ROOT / "include"

# The image exports CXX=/opt/gcc/bin/g++, which lacks libgomp: use the system
# compiler explicitly.
HOST_CXX = os.environ.get("SOD2D_HOST_CXX", "/usr/bin/g++")
NVCC = os.environ.get("SOD2D_NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"

HOST_SRCS = ["host_setup.cpp"]
GPU_SRCS = ["sod2d_gpu.cu", "comp_step.cu", "incomp.cu", "precond.cu", "noalloc_analysis.cu"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    subprocess.run(cmd, check=True)


def build_host(force: bool = False) -> Path:
    LIBDIR.mkdir(exist_ok=True)
    out = LIBDIR / "libsod2d_host.so"
    srcs = [CSRC / s for s in HOST_SRCS]
    deps = srcs + [INCLUDE / "sod2d_host.h"]
    if force or _stale(out, deps):
        _run([HOST_CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
              "-ffp-contract=off", f"-I{INCLUDE}", *map(str, srcs), "-o", str(out)])
    return out


def build_gpu(force: bool = False) -> Path:
    """Each translation unit is compiled on its own (in parallel, and only
    when it or a header changed), then linked into one shared library."""
    from concurrent.futures import ThreadPoolExecutor
    LIBDIR.mkdir(exist_ok=True)
    OBJDIR.mkdir(exist_ok=True)
    out = LIBDIR / "libsod2d_gpu.so"
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + [INCLUDE / "sod2d_gpu.h"]
    flags = [ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}",
             "--expt-relaxed-constexpr", f"-ccbin={HOST_CXX}"]
    objs = []
    jobs = []
    for name in GPU_SRCS:
        src = CSRC / name
        obj = OBJDIR / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC, *flags, "-c", str(src), "-o", str(obj)])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
            list(ex.map(_run, jobs))
    if force or jobs or _stale(out, objs):
        _run([NVCC, ARCH, "-shared", f"-ccbin={HOST_CXX}", *map(str, objs), "-o", str(out)])
    return out


def build_all(force: bool = False) -> None:
    build_host(force)
    if (CSRC / GPU_SRCS[0]).exists():
        build_gpu(force)


if __name__ == "__main__":
    import sys
    build_all(force="--force" in sys.argv)
    print("built:", *sorted(p.name for p in LIBDIR.glob("*.so")))

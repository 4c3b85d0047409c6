"""Builds the engine library (libsimlab_lbm.so, sm_100a) in-tree with nvcc.

The library is the product: CUDA kernels, the C++ host driver behind the C ABI
of include/simlab_lbm.h and the host voxelizer.  It is compiled for sm_100a
only and placed next to this file so it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libsimlab_lbm.so"

CUDA_SOURCES = ["d3q19_kernels.cu", "lattice.cu", "noalloc.cu", "d3q27_kernels.cu", "mlattice.cu", "gray.cu", "voxel_gpu.cu"]
# the GPU voxelizer rounds every product and sum separately, as the host
# voxelizer does, so its results are bit-identical
FILE_FLAGS = {"voxel_gpu.cu": ["-fmad=false"]}
CXX_SOURCES = ["voxel.cpp"]
HEADERS = ["lbm_device.cuh", "lbm_kernels.h", "voxel.hpp", "d3q27.h", "revoxel.cuh", "spin_math.cuh", "tma.cuh", "reduce.cuh", "host_wait.hpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-prec-div=false", "-prec-sqrt=false", "-Xcompiler", "-fPIC,-fopenmp",
              "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], log: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    log.append(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")


def build_library(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in CUDA_SOURCES + CXX_SOURCES + HEADERS] + [ROOT / "include" / "simlab_lbm.h", Path(__file__)]
    if not force and not _stale(LIB, deps):
        return LIB
    # the library is stamped with the newest source time seen now, so a source
    # edited while the build runs leaves it stale for the next call
    t_src = max(d.stat().st_mtime for d in deps)
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    log: list[str] = []
    cc = nvcc()
    cmds = []
    for src in CUDA_SOURCES:
        obj = objdir / (src + ".o")
        cmds.append(([cc, *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(src, []), "-I", str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)], obj))
    for src in CXX_SOURCES:
        obj = objdir / (src + ".o")
        cmds.append((["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-c", str(CSRC / src), "-o", str(obj)], obj))
    # the translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor

    logs: list[list[str]] = [[] for _ in cmds]
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        futs = [ex.submit(_run, c, logs[k]) for k, (c, _) in enumerate(cmds)]
        for f in futs:
            f.result()
    for lg in logs:
        log.extend(lg)
    objs = [str(o) for _, o in cmds]
    tmp = LIB.with_suffix(".so.tmp")
    _run([cc, *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"], log)
    os.replace(tmp, LIB)
    os.utime(LIB, (t_src, t_src))
    (objdir / "build.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

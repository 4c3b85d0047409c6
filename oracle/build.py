"""TEST INFRASTRUCTURE -- builds the CPU oracle (liboracle.so) with g++.

Compiled with -ffp-contract=off and without fast-math so the FP32
instantiation performs the reference's FP32 operations one by one.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOURCES = [HERE / "oracle_capi.cpp", HERE / "d3q19_oracle.hpp", HERE / "d3q27_oracle.hpp", HERE / "gray_oracle.hpp", HERE.parent / "include" / "simlab_lbm.h"]


def build_oracle(force: bool = False) -> Path:
    if not force and LIB.exists() and all(s.stat().st_mtime <= LIB.stat().st_mtime for s in SOURCES):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           str(HERE / "oracle_capi.cpp"), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))

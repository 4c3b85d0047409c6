"""Small profiling workload for ncu captures: the arm LES case on a
512x256x64 lattice (8.4 M cells; 352 MB of FP16 populations, larger than L2),
a few steps of one storage format.

    python -m simlab_b200.profile_case [fp16|fp32|bf16|fp64] [steps]
"""
from __future__ import annotations

import sys

from .cases import arm_les
from .lbm import Lattice, Storage


def main() -> None:
    storage = Storage[(sys.argv[1] if len(sys.argv) > 1 else "fp16").upper()]
    steps = int(sys.argv[2]) if len(sys.argv) > 2 else 6
    st, vox = arm_les(storage, dims=(512, 256, 64))
    lat = Lattice(st, vox)
    lat.advance(steps)
    lat.synchronize()
    m, bad = lat.mass()
    print(f"profile case {storage.name} 512x256x64: {steps} steps, mass {m:.6e}, non-finite {bad}")


if __name__ == "__main__":
    main()

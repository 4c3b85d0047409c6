"""Small profiling workloads for ncu captures, a few steps of one storage format.

    python -m simlab_b200.profile_case [fp16|fp32|bf16|fp64] [steps]
        the arm LES case on a 512x256x64 lattice (8.4 M cells; 352 MB of FP16
        populations, larger than L2), D3Q19
    python -m simlab_b200.profile_case d3q27 [fp16|fp32|bf16|fp64] [steps]
        a single-level D3Q27 wind tunnel, 256x128x128 (4.2 M cells; 453 MB of
        FP16 populations in two sets), velocity inlet, open faces, sponges
"""
from __future__ import annotations

import sys

from .cases import arm_les
from .lbm import FaceBc, Lattice, Storage


def d3q27_tunnel(storage: Storage):
    from .mlattice import MultiSetup

    F = FaceBc
    return MultiSetup(dims0=[256, 128, 128], faces=[F.VELOCITY] + [F.OPEN] * 5, nu0=0.001, u_inf=[0.05, 0, 0], u_init=[0.05, 0, 0],
                      sponge=[0, 16, 8, 8, 8, 8], sponge_tau=1.0, sponge_sigma=0.1, total_pressure_inlet=True, storage=storage)


def main() -> None:
    args = sys.argv[1:]
    if args and args[0] == "d3q27":
        from .mlattice import MultiLattice

        storage = Storage[(args[1] if len(args) > 1 else "fp16").upper()]
        steps = int(args[2]) if len(args) > 2 else 6
        lat = MultiLattice(d3q27_tunnel(storage))
        lat.advance(steps)
        lat.synchronize()
        m, bad = lat.mass(0)
        print(f"profile case D3Q27 {storage.name} 256x128x128: {steps} steps, mass {m:.6e}, non-finite {bad}")
        return
    storage = Storage[(args[0] if args else "fp16").upper()]
    steps = int(args[1]) if len(args) > 1 else 6
    st, vox = arm_les(storage, dims=(512, 256, 64))
    lat = Lattice(st, vox)
    lat.advance(steps)
    lat.synchronize()
    m, bad = lat.mass()
    print(f"profile case {storage.name} 512x256x64: {steps} steps, mass {m:.6e}, non-finite {bad}")


if __name__ == "__main__":
    main()

"""Small profiling workloads for ncu captures, a few steps of one storage format.

    python -m simlab_b200.profile_case [fp16|fp32|bf16|fp64] [steps]
        the arm LES case on a 512x256x64 lattice (8.4 M cells; 352 MB of FP16
        populations, larger than L2), D3Q19
    python -m simlab_b200.profile_case d3q27 [fp16|fp32|bf16|fp64] [steps]
        a single-level D3Q27 wind tunnel, 256x128x128 (4.2 M cells; 453 MB of
        FP16 populations in two sets), velocity inlet, open faces, sponges
    python -m simlab_b200.profile_case levels [fp16|fp32] [finest steps]
        the refined rotor case on a 128x64x64 coarse level with its two boxes
        (3.6 M cells; 392 MB of FP16 populations): ghosts, restriction, faces,
        force reduction and the D3Q27 re-voxelizer of the spinning rotor
    python -m simlab_b200.profile_case spin [steps]
        the two-blade rotor (radius 40) spinning on one 256x128x128 D3Q19 level,
        FP16: the D3Q19 re-voxelizer and moving-wall records
    python -m simlab_b200.profile_case probes [steps]
        the arm case on 512x256x64, FP16, with 10,000 surface probes and two
        slices sampled every step, then the FP64 mass check
    python -m simlab_b200.profile_case gray [steps]
        the gray-level design case (192x96x96, FP32): forward steps, then one
        adjoint sweep over the same steps (checkpoint every 10)
    python -m simlab_b200.profile_case voxel [19|27]
        the static voxelizer on the GPU: a sphere of radius 100 cells (81,920
        triangles) in a 222^3 lattice, two calls
    python -m simlab_b200.profile_case levelprobes [finest steps]
        three D3Q27 levels (coarse 128x64x64, FP16) with a sphere of radius 12
        on the finest, its surface vertices and two slices sampled every
        finest step, then the mass of each level and the finest level's dump
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


def _levels(args) -> None:
    from .cases import prop_refined, spin_schedule
    from .mlattice import MultiLattice

    storage = Storage[(args[0] if args else "fp16").upper()]
    steps = int(args[1]) if len(args) > 1 else 8
    s, geo, om = prop_refined(storage, radius=30.0, dims0=(128, 64, 64))
    lat = MultiLattice(s, geo)
    f = lat.run(spin_schedule(steps, om, 1))
    print(f"profile case levels {storage.name} {lat.level_cells()}: {steps} finest steps, last force {f[-1][:3]}")


def _spin(args) -> None:
    from .cases import rotor_tunnel, spin_schedule

    steps = int(args[0]) if args else 6
    st, geo, om = rotor_tunnel(Storage.FP16, spinning=True)
    lat = Lattice(st, geo)
    f = lat.run(spin_schedule(steps, om, 1))
    print(f"profile case spin: {steps} steps, {lat.nrec} records, last force {f[-1][:3]}")


def _probes(args) -> None:
    import numpy as np

    from .lbm import Probes, SliceDef

    steps = int(args[0]) if args else 6
    st, vox = arm_les(Storage.FP16, dims=(512, 256, 64))
    rng = np.random.default_rng(7)
    c = np.asarray(st.center)
    verts = [(rng.uniform(-20, 20, 3), np.array([1.0, 0.0, 0.0])) for _ in range(10000)]
    sl = [SliceDef(origin=(1, int(c[1]), 1), u=(1, 0, 0), v=(0, 0, 1), nu=510, nv=62),
          SliceDef(origin=(int(c[0]), 1, 1), u=(0, 1, 0), v=(0, 0, 1), nu=254, nv=62)]
    lat = Lattice(st, vox, Probes(verts=verts, slices=sl, vertex_offset=1.0))
    lat.run(steps_array_sampled(steps))
    m, bad = lat.mass()
    print(f"profile case probes: {steps} sampled steps, {lat.npix} pixels, mass {m:.6e}, non-finite {bad}")


def steps_array_sampled(n: int):
    from .lbm import steps_array

    return steps_array(n, sample=True)


def _gray(args) -> None:
    from .cases import gray_design
    from .gray import AdjointSpec, GrayLattice

    steps = int(args[0]) if args else 20
    st, gam, _ = gray_design()
    lat = GrayLattice(st, gam)
    lat.run(steps)
    lat.reset()
    spec = AdjointSpec(steps=steps, t0=steps // 2 + 1, t1=steps, checkpoint_every=10, objective=0, dir=[1.0, 0.0, 0.0], recompute=True)
    j, g = lat.backward(spec)
    print(f"profile case gray: {steps} steps forward, adjoint objective {j:.6e}, |grad| {float((g * g).sum()) ** 0.5:.3e}")


def _voxel(args) -> None:
    from .lbm import voxelize_static
    from .shapes import sphere

    q = int(args[0]) if args else 19
    v, t = sphere([110.3, 110.7, 110.1], 100.0, 6)
    for _ in range(2):
        vox = voxelize_static(v, t, [222] * 3, q, device=True)
    print(f"profile case voxel D3Q{q}: {len(t)} triangles, {len(vox.solid)} solid cells, {len(vox.walls)} wall records")


def _levelprobes(args) -> None:
    import numpy as np

    from .lbm import Probes, SliceDef, steps_array, voxelize_static
    from .mlattice import LevelBox, MultiLattice, MultiSetup
    from .shapes import sphere

    steps = int(args[0]) if args else 8
    F = FaceBc
    s = MultiSetup(dims0=[128, 64, 64], faces=[F.VELOCITY] + [F.OPEN] * 5, nu0=0.001, u_inf=[0.05, 0, 0], u_init=[0.05, 0, 0],
                   sponge=[0, 16, 8, 8, 8, 8], sponge_tau=1.0, sponge_sigma=0.1, total_pressure_inlet=True, storage=Storage.FP16,
                   debug_dump=True)
    for l in range(1, 3):
        d = s.dims(l - 1)
        n = [int(d[k] * 0.63) for k in range(3)]
        s.boxes.append(LevelBox(lo=[(d[k] - n[k]) // 2 for k in range(3)], n=n))
    fd = s.dims(2)
    c = [fd[0] * 0.4 + 0.3, fd[1] * 0.5 + 0.2, fd[2] * 0.5 + 0.1]
    s.center = c
    v, t = sphere(c, 12.0, 4)
    vox = voxelize_static(v, t, list(fd), 27)
    rel = np.asarray(v) - np.asarray(c)
    verts = [(tuple(p), tuple(p / np.linalg.norm(p))) for p in rel]
    # slices in finest-level units over the whole domain: the finest level's
    # node 0 sits at 4 lo(box 1) + 2 lo(box 2)
    org = [4 * s.boxes[0].lo[k] + 2 * s.boxes[1].lo[k] for k in range(3)]
    yc, zc = org[1] + int(round(c[1])), org[2] + int(round(c[2]))
    slices = [SliceDef(origin=[0, 0, zc], u=[2, 0, 0], v=[0, 2, 0], nu=256, nv=128),
              SliceDef(origin=[0, yc, 0], u=[2, 0, 0], v=[0, 0, 2], nu=256, nv=128)]
    lat = MultiLattice(s, vox, probes=Probes(verts=verts, slices=slices, vertex_offset=0.5))
    lat.run(steps_array(steps, sample=True))
    masses = [lat.mass(l) for l in range(lat.levels())]
    m = lat.macros(2)
    print(f"profile case levelprobes {lat.level_cells()}: {steps} sampled finest steps, {lat.nvert} vertices, {lat.npix} pixels, "
          f"masses {[f'{x[0]:.4e}' for x in masses]}, finest macros {m.shape}")


def main() -> None:
    args = sys.argv[1:]
    cases = {"levels": _levels, "spin": _spin, "probes": _probes, "gray": _gray, "voxel": _voxel, "levelprobes": _levelprobes}
    if args and args[0] in cases:
        cases[args[0]](args[1:])
        return
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

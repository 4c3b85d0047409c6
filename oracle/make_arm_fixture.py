"""TEST INFRASTRUCTURE -- writes oracle/fixtures/arm_les_512x256x256.npz.

The CPU baseline (bench.py's cpu_baseline leg and its --impl reference arm)
runs the oracle on the 512x256x256 LES arm case.  So that those runs load
nothing of the engine, the case's inputs are frozen here once: the lattice
setup (every field of lbm_setup) and the arm's solid cells and wall links, as
the engine's voxelizer (a port of crates/cfd/src/voxel.rs) produces them for
simlab_b200.cases.arm_les with FP16 storage.

    python -m oracle.make_arm_fixture
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "fixtures" / "arm_les_512x256x256.npz"


def main() -> None:
    from simlab_b200.cases import arm_les
    from simlab_b200.lbm import Storage

    st, vox = arm_les(Storage.FP16)
    setup = {"dims": [int(d) for d in st.dims], "faces": [int(f) for f in st.faces], "nu": float(st.nu), "smagorinsky": float(st.smagorinsky),
             "u_inf": [float(v) for v in st.u_inf], "u_init": [float(v) for v in st.u_init], "body_force": [float(v) for v in st.body_force],
             "sponge": [int(v) for v in st.sponge], "sponge_tau": float(st.sponge_tau), "sponge_sigma": float(st.sponge_sigma),
             "absorb_velocity": int(bool(st.absorb_velocity)), "total_pressure_inlet": int(bool(st.total_pressure_inlet)),
             "storage": int(st.storage), "collision": int(st.collision), "center": [float(v) for v in st.center],
             "debug_dump": 0, "wall_model": int(bool(st.wall_model))}
    OUT.parent.mkdir(exist_ok=True)
    np.savez_compressed(OUT, setup=np.frombuffer(json.dumps(setup).encode(), dtype=np.uint8),
                        solid=np.asarray(vox.solid, dtype=np.uint32), walls=np.asarray(vox.walls))
    print(OUT)


if __name__ == "__main__":
    main()

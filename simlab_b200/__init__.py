"""simlab_b200: a B200-native lattice-Boltzmann time step for SimLab's
`crates/cfd` wind tunnel, behind the reference's solver API (C ABI in
include/simlab_lbm.h, Python mirror in `simlab_b200.lbm`)."""
from .lbm import (  # noqa: F401
    Collision,
    FaceBc,
    Lattice,
    LatticeSetup,
    LbmError,
    Probes,
    SliceDef,
    SpinGeometry,
    SpinVoxels,
    StaticVoxels,
    StepIn,
    Storage,
    halfway,
    inside_grid,
    library,
    steps_array,
    voxelize_spin,
    voxelize_static,
)

"""The spinning-part path (Geometry::Spin, the GPU re-voxelizer of
crates/cfd/src/shader.rs:865-1104) against the CPU oracle and the
reference's own check (crates/cfd/tests/geometry.rs:79-161: at angle zero the
re-voxelizer finds the static voxelizer's walls).  The re-voxelizer's
geometric arithmetic is f32 rounded per operation in both, so links agree bit
for bit; tolerances: FP32 relative L2 of u <= 1e-5, forces <= 1e-5 of their
largest value, FP64 engine vs FP64 oracle forces <= 1e-9."""
import numpy as np
import pytest

from oracle import OracleLattice
from simlab_b200.lbm import FaceBc, Lattice, LatticeSetup, SpinGeometry, Storage, steps_array, voxelize_spin, voxelize_static
from simlab_b200.shapes import cuboid, merge, sphere

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def rotz(a):
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def spin_steps(n, w, a0=0.0):
    a = steps_array(n)
    for k in range(n):
        a[k]["rot"] = rotz(a0 + w * (k + 1))
        a[k]["rot_prev"] = rotz(a0 + w * k)
        a[k]["omega"] = [0.0, 0.0, w]
    return a


def paddle():
    """A two-blade paddle in body coordinates: a hub and two offset plates."""
    return merge(cuboid([-2.2, -2.1, -2.3], [2.1, 2.3, 2.2]), cuboid([2.0, -0.9, -1.7], [9.3, 0.8, 1.6]),
                 cuboid([-9.1, -0.7, -1.4], [-2.0, 1.1, 1.9]))


def spin_case(storage=Storage.FP32, n=(40, 36, 24), c=(19.6, 18.3, 11.7)):
    v, t = paddle()
    sv = voxelize_spin(v, t, [0.0, 0.0, 1.0], 0.125)
    r = int(np.ceil(sv.radius)) + 3
    box_lo = [int(c[0]) - r, int(c[1]) - r, int(c[2]) - 5]
    box_n = [2 * r + 1, 2 * r + 1, 11]
    F = FaceBc
    st = LatticeSetup(dims=list(n), faces=[F.VELOCITY, F.OPEN, F.PERIODIC, F.PERIODIC, F.PERIODIC, F.PERIODIC], nu=0.02,
                      u_inf=[0.03, 0.0, 0.0], u_init=[0.03, 0.0, 0.0], storage=storage, center=list(c), debug_dump=True)
    return st, SpinGeometry(vox=sv, box_lo=box_lo, box_n=box_n)


def test_revoxelizer_at_angle_zero_finds_the_static_walls():
    """geometry.rs:79-161: links that differ <= 6 % of the common ones, q
    differing by more than 0.05 on <= 0.2 % of them."""
    st, geo = spin_case()
    v, t = paddle()
    c = st.center
    vs = voxelize_static(np.asarray(v) + np.asarray(c), t, st.dims)
    lat = Lattice(st, geo)
    lat.run(spin_steps(1, 0.0))
    recs = lat.records().reshape(-1, 40)
    gpu = {int(r[1]): r for r in recs if r[0] != 0}
    same = diff = qbad = 0
    for w in vs.walls:
        r = gpu.get(int(w["cell"]))
        if r is None:
            diff += bin(int(w["mask"])).count("1")
            continue
        m = int(r[0])
        common = m & int(w["mask"])
        diff += bin(m ^ int(w["mask"])).count("1")
        same += bin(common).count("1")
        q = np.concatenate([[np.nan], np.frombuffer(r[2:11].astype(np.uint32).tobytes(), dtype=np.float16).astype(np.float32)])
        for d in range(1, 19):
            if common & (1 << d) and abs(q[d] - w["q"][d]) > 0.05:
                qbad += 1
    assert same > 100
    assert diff <= 0.06 * same, (diff, same)
    assert qbad <= 0.002 * same + 1, (qbad, same)


@pytest.mark.parametrize("storage", [Storage.FP32, Storage.FP64])
def test_spinning_paddle_matches_oracle(storage):
    st, geo = spin_case(storage)
    g, o = Lattice(st, geo), OracleLattice(st, geo, real64=storage == Storage.FP64)
    steps = spin_steps(90, 0.02)
    hg, ho = g.run(steps), o.run(steps)
    rg, ro = g.records().reshape(-1, 40), o.records().reshape(-1, 40)
    assert np.array_equal(rg[:, :11], ro[:, :11])  # masks, cells and q bit-equal
    mg, mo = g.macros(), o.macros()
    assert np.array_equal(np.isnan(mg[:, 0]), np.isnan(mo[:, 0]))
    # macros() reads back float32, so the FP64 velocity bar is the readback's
    assert rel_l2(mg[:, 1:4], mo[:, 1:4]) <= (1e-5 if storage == Storage.FP32 else 1e-6)
    assert np.max(np.abs(hg - ho)) <= (1e-5 if storage == Storage.FP32 else 1e-9) * np.max(np.abs(ho))


def test_spinning_part_mass_follows_the_oracle():
    """Covering and uncovering cells does not conserve mass in this scheme
    (a covered cell's populations leave the fluid, an uncovered one is refilled
    at its neighbours' density); the engine's mass follows the FP64 oracle's."""
    st, geo = spin_case(Storage.FP64)
    st.faces = [FaceBc.PERIODIC] * 6
    g, o = Lattice(st, geo), OracleLattice(st, geo, real64=True)
    steps = spin_steps(150, 0.03)
    g.run(steps)
    o.run(steps)
    m1, bad = g.mass()
    mo = o.macros()
    assert bad == 0
    assert abs(m1 / np.nansum(mo[:, 0]) - 1.0) < 1e-9


def test_spinning_checkpoint_round_trip_is_exact():
    st, geo = spin_case(Storage.FP16)
    g = Lattice(st, geo)
    g.run(spin_steps(13, 0.02))
    blob = g.save_state()
    a = g.run(spin_steps(21, 0.02, a0=13 * 0.02))
    g.load_state(blob)
    b = g.run(spin_steps(21, 0.02, a0=13 * 0.02))
    assert np.array_equal(a, b)

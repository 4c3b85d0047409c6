"""Host voxelizer against crates/cfd/tests/geometry.rs:13-76 (CPU)."""
import numpy as np

from simlab_b200.lbm import inside_grid, voxelize_static
from simlab_b200.shapes import cuboid, merge, sphere

C19 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0], [-1, -1, 0], [1, 0, 1],
                [-1, 0, -1], [0, 1, 1], [0, -1, -1], [1, -1, 0], [-1, 1, 0], [1, 0, -1], [-1, 0, 1], [0, 1, -1], [0, -1, 1]])


def test_sphere_volume_and_links():
    r = 10.3
    v, t = sphere([20.2, 19.7, 20.4], r, 5)
    vox = voxelize_static(v, t, [41, 41, 41])
    exact = 4.0 / 3.0 * np.pi * r ** 3
    assert abs(len(vox.solid) / exact - 1.0) < 0.03
    net = np.zeros(3, dtype=np.int64)
    for w in vox.walls:
        for d in range(1, 19):
            if w["mask"] & (1 << d):
                assert 0.0 < w["q"][d] <= 1.0
                net += C19[d]
    assert np.all(net == 0)


def test_holes_and_overlaps_do_not_flood():
    v, t = cuboid([3.3, 3.3, 3.3], [16.7, 12.6, 14.2])
    t = t[2:]
    ins = inside_grid(v, t, [0.0, 0.0, 0.0], 1.0, [20, 16, 18])
    n = int(ins.sum())
    exact = (16 - 4 + 1) * (12 - 4 + 1) * (14 - 4 + 1)
    assert abs(n - exact) <= exact // 20
    a = cuboid([2.3, 2.3, 2.3], [10.6, 10.6, 10.6])
    b = cuboid([6.4, 6.4, 6.4], [14.7, 14.7, 14.7])
    v, t = merge(a, b)
    ins = inside_grid(v, t, [0.0, 0.0, 0.0], 1.0, [17, 17, 17])
    assert ins[(8 * 17 + 8) * 17 + 8]


def test_thin_plate_blocks_links():
    v, t = cuboid([2.0, 2.0, 5.4], [12.0, 12.0, 5.6])
    vox = voxelize_static(v, t, [15, 15, 12])
    assert len(vox.solid) == 0
    up = int(np.sum((vox.walls["mask"] >> 5) & 1))
    down = int(np.sum((vox.walls["mask"] >> 6) & 1))
    assert up > 50 and up == down


def test_voxelizer_deterministic_and_d3q27():
    v, t = sphere([12.3, 11.8, 12.1], 5.2, 4)
    a = voxelize_static(v, t, [25, 25, 25])
    b = voxelize_static(v, t, [25, 25, 25])
    assert np.array_equal(a.solid, b.solid) and a.walls.tobytes() == b.walls.tobytes()
    c = voxelize_static(v, t, [25, 25, 25], lattice=27)
    assert np.array_equal(a.solid, c.solid)
    assert len(c.walls) >= len(a.walls)

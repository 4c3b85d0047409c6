"""The GPU static voxelizer (lbm_voxelize_static_gpu) against the host one
(voxel.cpp, the restatement of crates/cfd/src/voxel.rs:73-490): solid cells,
wall cells, link masks and every q bit for bit, on the shapes the
reference's geometry tests use and on the bench's arm."""
import numpy as np
import pytest

from simlab_b200 import shapes
from simlab_b200.cases import arm_les
from simlab_b200.lbm import voxelize_static

pytestmark = pytest.mark.gpu


def same(v, t, dims, lattice):
    a = voxelize_static(v, t, dims, lattice)
    b = voxelize_static(v, t, dims, lattice, device=True)
    assert np.array_equal(a.solid, b.solid)
    assert len(a.walls) == len(b.walls)
    assert np.array_equal(a.walls["cell"], b.walls["cell"])
    assert np.array_equal(a.walls["mask"], b.walls["mask"])
    assert np.array_equal(a.walls["q"].view(np.uint32), b.walls["q"].view(np.uint32))
    return a


@pytest.mark.parametrize("lattice", [19, 27])
@pytest.mark.parametrize("center,radius,sub", [((20.3, 21.7, 19.1), 9.6, 3), ((32.0, 32.0, 32.0), 12.0, 5), ((40.37, 30.11, 33.9), 21.3, 4)])
def test_spheres(lattice, center, radius, sub):
    v, t = shapes.sphere(center, radius, sub)
    a = same(v, t, [80, 64, 64], lattice)
    assert len(a.solid) > 0 and len(a.walls) > 0


@pytest.mark.parametrize("lattice", [19, 27])
def test_grid_aligned_cuboid_and_thin_plate(lattice):
    # faces on lattice planes (crossings at grid points) and a plate thinner
    # than a cell (thin-sheet links both ways)
    v1, t1 = shapes.cuboid([10.0, 10.0, 10.0], [30.0, 22.0, 18.0])
    v2, t2 = shapes.cuboid([40.2, 8.5, 6.5], [40.5, 30.5, 26.5])
    v, t = shapes.merge((v1, t1), (v2, t2))
    a = same(v, t, [64, 40, 36], lattice)
    assert len(a.walls) > 0


@pytest.mark.parametrize("lattice", [19, 27])
def test_part_crossing_the_lattice_boundary(lattice):
    v, t = shapes.sphere([2.2, 30.4, 61.3], 10.5, 4)
    same(v, t, [48, 48, 64], lattice)


def test_open_surface_and_empty():
    v = np.array([[5.1, 5.2, 5.3], [25.4, 6.1, 7.2], [8.3, 27.5, 20.6], [24.0, 26.0, 9.0]])
    t = np.array([[0, 1, 2], [1, 3, 2]], dtype=np.uint32)
    same(v, t, [32, 32, 32], 19)
    e = voxelize_static(np.zeros((0, 3)), np.zeros((0, 3), dtype=np.uint32), [16, 16, 16], 19, device=True)
    assert len(e.solid) == 0 and len(e.walls) == 0


@pytest.mark.parametrize("lattice", [19, 27])
def test_propeller_thin_blades(lattice):
    v, t = shapes.propeller(radius=30.0)
    v = np.asarray(v) + np.array([40.31, 40.23, 40.17])
    same(v, t, [80, 80, 80], lattice)


def test_bench_arm_512x256x256():
    from simlab_b200.shapes import arm

    v, t = arm(center=(128.0, 128.0, 128.0))
    a = same(v, t, [512, 256, 256], 19)
    st, vox = arm_les()
    assert np.array_equal(a.solid, vox.solid) and len(a.walls) == len(vox.walls)

"""The multi-level D3Q27 oracle against the reference's known answers for the
refined solver (crates/cfd/tests/refined.rs): Poiseuille flow between off-grid
Bouzidi plates with second-order convergence and force balance (34-81),
momentum lost by the fluid equal to the impulse on a sphere (83-98) and a
uniform stream crossing two refinement levels unchanged (100-119)."""
import numpy as np

from oracle import OracleMulti
from simlab_b200.lbm import FaceBc, voxelize_static
from simlab_b200.mlattice import LevelBox, MultiSetup
from simlab_b200.shapes import cuboid, merge, sphere

from helpers import poiseuille_error


def multi_setup(dims0, faces, nu0, u):
    """refined.rs:13-31."""
    return MultiSetup(dims0=list(dims0), faces=list(faces), nu0=nu0, u_inf=[u, 0.0, 0.0], u_init=[u, 0.0, 0.0], sponge_tau=1.0,
                      debug_dump=True)


def poiseuille27(h, lat_cls):
    """refined.rs:34-65: plates with edges off the lattice diagonals."""
    ya = 1.37
    yb = ya + h
    ny = int(np.ceil(yb)) + 2
    nx = nz = 3
    v, t = merge(cuboid([-5.3, -10.0, -4.1], [nx + 4.6, ya, nz + 5.7]), cuboid([-5.3, yb, -4.1], [nx + 4.6, ny + 10.0, nz + 5.7]))
    vox = voxelize_static(v, t, [nx, ny, nz], 27)
    nu = 0.1
    g = 0.02 * 8.0 * nu / (h * h)
    s = multi_setup([nx, ny, nz], [FaceBc.PERIODIC] * 6, nu, 0.0)
    s.body_force0 = [g, 0.0, 0.0]
    lat = lat_cls(s, vox)
    hist = lat.run(int(3.0 * h * h / nu))
    return poiseuille_error(lat.macros(0), hist, (ya, yb, nu, g, nx, ny))


def momentum27(lat_cls, steps=600):
    """refined.rs:83-98."""
    n, c = 40, 20.0
    v, t = sphere([c + 0.3, c - 0.6, c + 0.17], 6.0, 5)
    vox = voxelize_static(v, t, [n, n, n], 27)
    lat = lat_cls(multi_setup([n, n, n], [FaceBc.PERIODIC] * 6, 0.05, 0.05), vox)

    def mom():
        m = lat.macros(0)
        m = m[~np.isnan(m[:, 0])].astype(np.float64)
        return float((m[:, 0] * m[:, 1]).sum())

    p0 = mom()
    h = lat.run(steps)
    p1 = mom()
    imp = float(h[:, 0].sum())
    return (p0 - p1 - imp) / imp


def uniform_refined_setup():
    """refined.rs:100-109: velocity inlet, open elsewhere, two nested boxes."""
    s = multi_setup([64, 48, 48], [FaceBc.VELOCITY] + [FaceBc.OPEN] * 5, 0.01, 0.06)
    s.total_pressure_inlet = True
    for l in range(1, 3):
        d = s.dims(l - 1)
        s.boxes.append(LevelBox(lo=[d[0] // 4, d[1] // 4, d[2] // 4], n=[d[0] // 2, d[1] // 2, d[2] // 2]))
    return s


def check_uniform(lat):
    """refined.rs:110-118."""
    for l in range(3):
        m = lat.macros(l)
        m = m[~np.isnan(m[:, 0])]
        assert len(m) > 0
        assert np.all(np.abs(m[:, 0] - 1.0) < 1e-5), l
        assert np.all(np.abs(m[:, 1] - 0.06) < 1e-5), l
        assert np.all(np.abs(m[:, 2]) < 1e-6), l


def test_oracle_d3q27_poiseuille_second_order():
    e = []
    for h in (8.0, 16.0, 32.0):
        err, bal = poiseuille27(h, OracleMulti)
        assert abs(bal) < 1e-3
        e.append(err)
    order = np.log2(e[1] / e[2])
    assert order > 1.7 and e[2] < 1e-3


def test_oracle_d3q27_momentum_balance():
    assert abs(momentum27(OracleMulti)) < 1e-3


def test_oracle_uniform_stream_crosses_refinement_unchanged():
    s = uniform_refined_setup()
    lat = OracleMulti(s)
    assert lat.level_dims() == [(64, 48, 48), (63, 47, 47), (61, 45, 45)]
    lat.run(100 * lat.sub_steps())
    check_uniform(lat)


def test_oracle_multi_step_count_must_be_a_multiple():
    s = uniform_refined_setup()
    lat = OracleMulti(s)
    import pytest

    with pytest.raises(RuntimeError, match="multiple of 4"):
        lat.run(3)


def test_oracle_probes_uniform_stream_across_levels():
    """Probes on the refined lattice (mlattice.rs:243-305, 844-881;
    mshader.rs:563-602): in the uniform stream of refined.rs:100-119 every
    sampled pixel, whichever level it is taken from, and every surface vertex
    read the stream's state; pixels on the coarsest level's boundary nodes
    (outside its interior) have no level and stay NaN."""
    from simlab_b200.lbm import Probes, SliceDef, steps_array

    s = uniform_refined_setup()
    fd = s.dims(2)
    s.center = [0.5 * (fd[0] - 1) + 0.3, 0.5 * (fd[1] - 1) + 0.2, 0.5 * (fd[2] - 1) + 0.1]
    verts = [((2.0 * np.cos(a), 2.0 * np.sin(a), 0.5), (np.cos(a), np.sin(a), 0.0)) for a in np.linspace(0, 6.0, 7)]
    slices = [SliceDef(origin=[0, 0, 96], u=[4, 0, 0], v=[0, 4, 0], nu=64, nv=48),     # the whole coarse plane
              SliceDef(origin=[60, 44, 95], u=[1, 0, 0], v=[0, 1, 0], nu=120, nv=90)]  # across both refinement boxes
    o = OracleMulti(s, probes=Probes(verts=verts, slices=slices, vertex_offset=0.5))
    a = steps_array(8)
    a["sample"] = 1
    o.run(a)
    vm = o.vertex_means()
    assert vm.shape == (7,) and np.all(np.abs(vm - 1.0) < 1e-5)
    sm = o.slice_means()
    assert sm.shape == (64 * 48 + 120 * 90, 4)
    c = sm[:64 * 48].reshape(48, 64, 4)
    assert np.all(np.isnan(c[:, 0, 0])) and np.all(np.isnan(c[0, :, 0]))  # x = 0, y = 0 coarse boundary nodes
    ok = ~np.isnan(sm[:, 0])
    assert ok.sum() >= 62 * 46 + 120 * 90
    assert np.all(np.abs(sm[ok, 0] - 1.0) < 1e-5) and np.all(np.abs(sm[ok, 1] - 0.06) < 1e-5) and np.all(np.abs(sm[ok, 2:]) < 1e-6)
    o.reset_samples()
    assert np.all(np.isnan(o.vertex_means())) and np.all(np.isnan(o.slice_means()[:, 0]))

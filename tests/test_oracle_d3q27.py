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

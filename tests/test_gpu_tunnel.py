"""Wind-tunnel runs through the study layer on the GPU, against the
reference's validation bars (crates/cfd/tests/tunnel.rs): sphere drag at
Re 20, 100 and 300 on uniform D3Q19 and refined D3Q27 grids, the Stokes
torque on a sphere turning in still air, and (SIMLAB_LONG_VALIDATION=1, the
cases the reference runs only on request) sphere drag at Re 1000 and 1e4
and a thin disk at Re 1e4 on three D3Q27 levels."""
import math
import os

import pytest

from simlab_b200 import tunnel as T

from test_tunnel import SPHERE_D, SPHERE_U, rotating_sphere_case, sphere_case

pytestmark = pytest.mark.gpu


def sphere_cd_cgw(re):
    """Clift, Grace & Weber's standard drag curve (validation.rs:10-23)."""
    w = math.log10(re)
    if re <= 20.0:
        return 24.0 / re * (1.0 + 0.1315 * re ** (0.82 - 0.05 * w))
    if re <= 260.0:
        return 24.0 / re * (1.0 + 0.1935 * re ** 0.6305)
    if re <= 1500.0:
        return 10.0 ** (1.6435 - 1.1242 * w + 0.1558 * w * w)
    if re <= 1.2e4:
        return 10.0 ** (-2.4571 + 2.5558 * w - 0.9295 * w * w + 0.1049 * w ** 3)
    return 10.0 ** (-1.9181 + 0.6370 * w - 0.0636 * w * w)


def sphere_cd_sn(re):
    """Schiller & Naumann (validation.rs:26-28)."""
    return 24.0 / re * (1.0 + 0.15 * re ** 0.687)


def sphere_check(re, cells, passes, tol):
    """tunnel.rs tests sphere_check: Cd with the exact sphere area against the
    correlations, and the side force of a steady wake."""
    cfg, m = sphere_case(re, cells, duration=passes)
    r = T.run_with(cfg, m, 1e-3, T.SolverOptions())
    s = r.summary
    cd = s.drag_n / (0.5 * cfg.air.density * SPHERE_U ** 2 * math.pi * SPHERE_D ** 2 / 4.0)
    ref = sphere_cd_cgw(re) if re > 250.0 else 0.5 * (sphere_cd_cgw(re) + sphere_cd_sn(re))
    side = math.hypot(s.lift_n, s.side_n) / abs(s.drag_n)
    print(f"sphere Re={re} D={cells}: Cd {cd:.4f} vs {ref:.4f} ({(cd / ref - 1) * 100:+.2f} %), converged {s.converged}, "
          f"{s.simulated:.1f} passes, {s.mlups:.0f} MLUPS, side/drag {side:.4f}")
    assert abs(cd / ref - 1.0) < tol
    assert side < (0.05 if re < 500.0 else 0.15)
    assert s.cd == pytest.approx(s.drag_n / (0.5 * cfg.air.density * SPHERE_U ** 2 * s.ref_area_mm2 * 1e-6), rel=1e-12)
    return r


def test_sphere_re100_uniform_grid():
    """sphere_re100_quick: 16 cells across, 15 flow passes, within 5 %."""
    r = sphere_check(100.0, 16, 15.0, 0.05)
    assert r.summary.grid == [137, 113, 113]


def test_sphere_re100_refined_grid():
    """sphere_re100: 48 cells across on two D3Q27 levels, 30 passes, within 3 %."""
    r = sphere_check(100.0, 48, 30.0, 0.03)
    assert r.summary.cells < 137 * 113 * 113 * 27  # the nested levels, not a uniform 48-cell grid


def test_sphere_re20():
    """sphere_re20: 32 cells across on one D3Q19 level, 30 passes, within 5 %
    (the reference's own run reads 2.689 against 2.662, docs/VALIDATION.md:95)."""
    sphere_check(20.0, 32, 30.0, 0.05)


def test_sphere_re300_refined_grid():
    """sphere_re300: 48 cells across on two D3Q27 levels, 40 passes, within
    6 % of Clift, Grace & Weber (the reference reads 0.634 against 0.653)."""
    sphere_check(300.0, 48, 40.0, 0.06)


LONG = pytest.mark.skipif(os.environ.get("SIMLAB_LONG_VALIDATION") != "1",
                          reason="about a minute each on a B200; set SIMLAB_LONG_VALIDATION=1")


@LONG
@pytest.mark.parametrize("re,tol", [(1000.0, 0.05), (1e4, 0.08)])
def test_sphere_96_cells_three_levels(re, tol):
    """sphere_re1000 and sphere_re10000: 96 cells across on three D3Q27
    levels, 50 passes (the reference reads 0.474 and 0.392 against 0.471 and
    0.405)."""
    sphere_check(re, 96, 50.0, tol)


@LONG
def test_disk_normal_to_flow_re10000():
    """disk_normal_to_flow_re10000 (validation.rs:57-66): a disk of diameter
    50 mm, 5 % thick, square to the wind, 96 cells across, 50 passes, Cd on
    its face area within 15 % of Hoerner's 1.17 (the reference reads 1.111)."""
    from simlab_b200.shapes import cylinder

    cfg, _ = sphere_case(1e4, 96, duration=50.0)
    v, t = cylinder([0.0, 0.0, 0.0], SPHERE_D / 2.0, 0.05 * SPHERE_D, axis=0)
    r = T.run_with(cfg, T.Mesh(v, t), 1e-3, T.SolverOptions())
    cd = r.summary.drag_n / (0.5 * cfg.air.density * SPHERE_U ** 2 * math.pi * SPHERE_D ** 2 / 4.0)
    print(f"disk Re 1e4: Cd {cd:.4f} vs 1.17 ({(cd / 1.17 - 1) * 100:+.1f} %), converged {r.summary.converged}, {r.summary.cells} cells")
    assert abs(cd / 1.17 - 1.0) < 0.15


def test_rotating_sphere_stokes_torque():
    """rotating_sphere_stokes_torque: Re 1, 24 cells, 6 revolutions, the
    torque within 5 % of 8 pi mu R^3 omega."""
    cfg, m = rotating_sphere_case(1.0, 24, 6.0)
    o = T.SolverOptions()
    o.still_margins.side = 2.0
    r = T.run_with(cfg, m, 1e-3, o)
    omega = 600.0 * 2.0 * math.pi / 60.0
    stokes = 8.0 * math.pi * cfg.air.density * cfg.air.kinematic_viscosity * 0.025 ** 3 * omega
    t = r.summary.torque_nm
    print(f"rotating sphere: torque {t:.4e} vs {stokes:.4e} ({(-t / stokes - 1) * 100:+.2f} %), thrust {r.summary.thrust_n:.2e}")
    assert abs(-t / stokes - 1.0) < 0.05

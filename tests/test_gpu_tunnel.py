"""Wind-tunnel runs through the study layer on the GPU, against the
reference's validation bars (crates/cfd/tests/tunnel.rs): sphere drag at
Re 100 on the uniform D3Q19 grid and on the refined D3Q27 grid, and the
Stokes torque on a sphere turning in still air."""
import math

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

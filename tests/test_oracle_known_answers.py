"""The oracle against the reference's own known-answer tests (CPU).

These pin the CPU restatement of the reference update: the reference ships
no golden vectors, so its analytic and conservation tests are re-run here on
the oracle with the reference's tolerances.
"""
import numpy as np
import pytest

from oracle import OracleLattice
from simlab_b200.lbm import FaceBc, Storage

from helpers import ball, channel_case, momentum_setup, poiseuille_error


def _poiseuille(h, storage, umax, real64=False):
    st, vox, steps, params = channel_case(h, umax, storage)
    lat = OracleLattice(st, vox, real64=real64)
    hist = lat.run(steps)
    return poiseuille_error(lat.macros(), hist, params)


def test_poiseuille_second_order():
    """crates/cfd/tests/channel.rs:76-89: L2 < 2e-3 at H=32, order > 1.6, balance < 2e-3."""
    errs = []
    for h in (8.0, 16.0, 32.0):
        e, bal = _poiseuille(h, Storage.FP32, 0.02)
        assert abs(bal) < 2e-3, f"wall force does not balance the body force: {bal}"
        errs.append(e)
    o2 = np.log2(errs[1] / errs[2])
    assert errs[2] < 2e-3
    assert o2 > 1.6 or errs[2] < 1e-4


def test_poiseuille_fp16_stochastic_rounding():
    """channel.rs:91-101: FP16 storage with stochastic rounding stays < 3e-3."""
    for umax in (0.02, 0.06):
        e, bal = _poiseuille(16.0, Storage.FP16, umax)
        assert e < 3e-3, e


def test_poiseuille_fp64_oracle():
    e, bal = _poiseuille(16.0, Storage.FP64, 0.02, real64=True)
    assert e < 2e-3 and abs(bal) < 1e-9


def test_momentum_lost_by_fluid_equals_impulse():
    """crates/cfd/tests/momentum.rs:39-51 (600 steps, |mismatch| < 5e-3)."""
    n = 40
    lat = OracleLattice(momentum_setup(n, 0.05, 0.05, 0.0, [FaceBc.PERIODIC] * 6), ball(n, 6.0))

    def fluid_momentum():
        m = lat.macros()
        ok = ~np.isnan(m[:, 0])
        return float(np.sum(m[ok, 0] * m[ok, 1]))

    p0 = fluid_momentum()
    h = lat.run(600)
    p1 = fluid_momentum()
    impulse = float(h[:, 0].sum())
    err = (p0 - p1 - impulse) / impulse
    assert impulse > 0.0
    assert abs(err) < 5e-3, err


def test_uniform_state_feels_no_force():
    """momentum.rs:73-85: still air with open faces and a sphere: |F| < 1e-4."""
    n = 32
    lat = OracleLattice(momentum_setup(n, 0.05, 0.0, 0.0, [FaceBc.OPEN] * 6), ball(n, 5.0))
    h = lat.run(50)
    assert np.all(np.abs(h) < 1e-4)

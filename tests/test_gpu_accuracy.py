"""Force accuracy of reduced-precision storage against the FP64 engine on the
refined rotor case: thrust and torque within the 0.5 % force-coefficient bar.

The case is the three-level D3Q27 rotor (simlab_b200.cases.prop_refined:
coarse 256x128x128, two nested levels of 8.1 M and 16.0 M cells, a 2-blade
rotor of radius 60 finest cells spinning on the finest level, tip speed
0.08, axial inflow 0.02, half-revolution smoothstep spin-up as
crates/cfd/src/tunnel.rs:1085-1098), at a finest-level viscosity of 0.01
(tip Reynolds number 0.08 x 60 / 0.01 = 480 on the radius): a laminar wake,
so that two runs whose roundings differ stay close and the storage error is
measurable.  Two revolutions; thrust (force along the spin axis) and torque
(moment about it) averaged over the last one.  The FP64 engine started from
a perturbed state (1e-6 of the inflow speed) shows the flow's own noise
floor, which must be far below the storage errors for the comparison to
mean anything.  The reference's own rotating-body check is the Stokes torque
of a spinning sphere (crates/cfd/src/validation.rs:70-88,
crates/cfd/tests/tunnel.rs:77-85); this case carries the same moving-wall
links and momentum exchange on a rotor.
"""
import pytest

pytestmark = pytest.mark.gpu


def test_laminar_rotor_thrust_torque_vs_fp64():
    from simlab_b200.lbm import Storage
    from simlab_b200.validate import run_prop

    nu, revs = 0.01, 2.0
    ref = run_prop(Storage.FP64, revs, nu_finest=nu)
    assert ref["finite"]
    assert ref["thrust"] > 0.1 and ref["torque"] < -1.0  # the rotor pushes the flow and the flow resists its spin
    floor = run_prop(Storage.FP64, revs, nu_finest=nu, perturbed=1.0)
    for key in ("thrust", "torque"):
        assert abs(floor[key] / ref[key] - 1.0) < 1e-7, ("laminar floor", key, floor[key], ref[key])
    for s in (Storage.FP32, Storage.FP16, Storage.BF16):
        r = run_prop(s, revs, nu_finest=nu)
        assert r["finite"], s
        for key in ("thrust", "torque"):
            err = abs(r[key] / ref[key] - 1.0)
            assert err < 5e-3, (s, key, r[key], ref[key], err)

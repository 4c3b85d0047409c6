"""Gray-level lattice and discrete adjoint on the GPU (through the C ABI):
the FP64 engine against the FP64 oracle (forces, objective, gradient), the
checkpoint-and-recompute sweep against the sweep that keeps every step, the
FP32 adjoint against the FP64 one, and, on the full 192x96x96 design case,
the gradient against central finite differences (h = 1e-3) on 32 seeded
design cells through the torch.autograd.Function harness.  Tolerances: FP64
engine vs oracle 1e-10 relative; recompute vs keep-all bit-equal; FP32 vs
FP64 gradient 2e-3 relative L2 (small case), 1e-2 (full case); adjoint vs
finite differences 1e-4 relative to the largest component (FP64) and 2e-2
(FP32).  FP16-stored forward (FP32 arithmetic and adjoint) against FP32:
forces 2e-3 relative to the largest, gradient 2e-2 relative L2; its
recompute sweep against its keep-all sweep bit-equal (the stochastic
rounding repeats from the step's seed)."""
import numpy as np
import pytest

from oracle import OracleGray
from simlab_b200.cases import gray_design, splitmix64
from simlab_b200.gray import AdjointSpec, GrayLattice, GraySetup, gray_objective_function
from simlab_b200.lbm import Storage

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def small(storage=Storage.FP64):
    s = GraySetup(dims=[20, 10, 9], box_lo=[5, 2, 2], box_n=[6, 5, 4], nu=0.04, u_in=[0.05, 0.01, -0.005], alpha=0.8,
                  center=[8.0, 5.0, 4.5], storage=storage)
    return s, splitmix64(11, s.nbox())


def test_forward_matches_oracle():
    s, g = small()
    e, o = GrayLattice(s, g), OracleGray(s, g)
    fe, fo = e.run(60), o.run(60)
    assert np.max(np.abs(fe - fo)) <= 1e-12 * np.max(np.abs(fo))


@pytest.mark.parametrize("objective", [0, 1])
@pytest.mark.parametrize("recompute", [True, False])
def test_fp64_adjoint_matches_oracle(objective, recompute):
    s, g = small()
    spec = AdjointSpec(steps=45, t0=12, t1=40, checkpoint_every=10, objective=objective, dir=[1.0, -0.4, 0.25], recompute=recompute)
    e, o = GrayLattice(s, g), OracleGray(s, g)
    Je, ge = e.backward(spec)
    Jo, go = o.backward(spec)
    assert abs(Je / Jo - 1.0) < 1e-12
    assert np.max(np.abs(ge - go)) <= 1e-10 * np.max(np.abs(go))


def test_recompute_equals_keep_all():
    s, g = small(Storage.FP32)
    e = GrayLattice(s, g)
    J1, g1 = e.backward(AdjointSpec(steps=37, t0=5, t1=37, checkpoint_every=8, recompute=True))
    t1 = e.backward_times()
    J2, g2 = e.backward(AdjointSpec(steps=37, t0=5, t1=37, checkpoint_every=8, recompute=False))
    t2 = e.backward_times()
    assert J1 == J2 and np.array_equal(g1, g2)
    assert t1["recompute_ms"] > 0 and t2["recompute_ms"] == 0


def test_fp32_adjoint_close_to_fp64():
    s32, g = small(Storage.FP32)
    s64, _ = small(Storage.FP64)
    spec = AdjointSpec(steps=60, t0=30, t1=60, checkpoint_every=20)
    _, g32 = GrayLattice(s32, g).backward(spec)
    _, g64 = GrayLattice(s64, g).backward(spec)
    assert rel_l2(g32, g64) <= 2e-3


def test_design_case_gradient_against_central_differences():
    """The full design case (192x96x96, 64x48x48 box, drag over steps
    500-1000, checkpoint every 50): FP64 adjoint vs central differences with
    h = 1e-3 on 32 seeded design cells, through the autograd harness; FP32
    adjoint vs FP64 adjoint."""
    import torch

    st64, gam, spec = gray_design(Storage.FP64)
    st32, _, _ = gray_design(Storage.FP32)
    Fn = gray_objective_function()
    lat64 = GrayLattice(st64)
    x = torch.tensor(gam, dtype=torch.float64, requires_grad=True)
    J = Fn.apply(x, lat64, spec)
    J.backward()
    g64 = x.grad.numpy().copy()
    assert np.isfinite(J.item()) and J.item() > 0
    lat32 = GrayLattice(st32, gam)
    _, g32 = lat32.backward(spec)
    assert rel_l2(g32, g64) <= 1e-2
    rng = np.random.default_rng(2024)
    cells = rng.choice(st64.nbox(), 32, replace=False)
    h = 1e-3
    fd = np.zeros(32)
    for k, b in enumerate(cells):
        for sgn in (1, -1):
            gp = gam.copy()
            gp[b] = np.clip(gp[b] + sgn * h, 0.0, 1.0)
            lat64.set_field(gp)
            fd[k] += sgn * lat64.objective(spec) / (2 * h)
    scale = np.max(np.abs(fd))
    assert np.max(np.abs(fd - g64[cells])) <= 1e-4 * scale
    assert np.max(np.abs(fd - g32[cells])) <= 2e-2 * scale


def test_fp16_storage_forward_close_to_fp32():
    s16, g = small(Storage.FP16)
    s32, _ = small(Storage.FP32)
    f16, f32 = GrayLattice(s16, g).run(60), GrayLattice(s32, g).run(60)
    assert np.isfinite(f16).all()
    assert np.max(np.abs(f16 - f32)) <= 2e-3 * np.max(np.abs(f32))


def test_fp16_storage_recompute_equals_keep_all():
    s, g = small(Storage.FP16)
    e = GrayLattice(s, g)
    J1, g1 = e.backward(AdjointSpec(steps=37, t0=5, t1=37, checkpoint_every=8, objective=1, dir=[0.3, 1.0, 0.2], recompute=True))
    J2, g2 = e.backward(AdjointSpec(steps=37, t0=5, t1=37, checkpoint_every=8, objective=1, dir=[0.3, 1.0, 0.2], recompute=False))
    assert J1 == J2 and np.array_equal(g1, g2)


def test_fp16_storage_adjoint_close_to_fp32():
    s16, g = small(Storage.FP16)
    s32, _ = small(Storage.FP32)
    spec = AdjointSpec(steps=60, t0=30, t1=60, checkpoint_every=20)
    J16, g16 = GrayLattice(s16, g).backward(spec)
    J32, g32 = GrayLattice(s32, g).backward(spec)
    assert abs(J16 / J32 - 1.0) <= 2e-3
    assert rel_l2(g16, g32) <= 2e-2

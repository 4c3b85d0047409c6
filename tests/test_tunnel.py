"""The study layer (simlab_b200.tunnel, crates/cfd/src/tunnel.rs) on the host:
the plan of the reference's validation cases (validation.rs sphere_case,
rotating_sphere), the convergence test of the averaging window, and the whole
run loop over a stand-in lattice that returns a known force, so the SI
conversion, the sampling schedule and the run folder are checked without a
GPU."""
import json
import math

import numpy as np
import pytest

from simlab_b200 import lbm, tunnel as T
from simlab_b200.shapes import sphere

SPHERE_D, SPHERE_U = 0.05, 10.0


def sphere_case(re, cells, duration=15.0):
    """validation.rs:34-45: a 50 mm sphere in a 10 m/s wind along +x."""
    v, t = sphere([0.0, 0.0, 0.0], SPHERE_D / 2.0, 5)
    cfg = T.WindConfig(wind_dir=(1.0, 0.0, 0.0), speed_m_s=SPHERE_U, air=T.Air(1.2, SPHERE_U * SPHERE_D / re), quality=cells, duration=duration)
    return cfg, T.Mesh(v, t)


def rotating_sphere_case(re, cells, revs):
    """validation.rs:70-90: a 25 mm-radius sphere turning at 600 rpm in still air."""
    v, t = sphere([0.0, 0.0, 0.0], 0.025, 5)
    omega = 600.0 * 2.0 * math.pi / 60.0
    nu = omega * 0.025 ** 2 / re
    cfg = T.WindConfig(wind_dir=(0.0, 0.0, 1.0), speed_m_s=0.0, air=T.Air(1.2, nu), spin=T.Spin(600.0, (0.0, 0.0, 1.0)), quality=cells,
                       duration=revs)
    return cfg, T.Mesh(v, t)


def test_plan_sphere_uniform():
    cfg, m = sphere_case(100.0, 16)
    p = T.plan(cfg, m, 1e-3, T.SolverOptions())
    assert p.multi is None and not p.spin and not p.still
    assert p.cells_across == 16 and p.dx == pytest.approx(SPHERE_D / 16, rel=1e-3)
    assert p.u_lat == pytest.approx(0.075)  # the Mach limit sets the step
    assert 0.5 + 3 * p.nu_lat == pytest.approx(0.536, rel=1e-3)
    # margins: 2.5 D upstream, 5 D downstream, 3 D to each side
    assert p.dims[0] == pytest.approx(8.5 * 16 + 1, abs=1)
    assert p.dims[1] == p.dims[2] == pytest.approx(7 * 16 + 1, abs=1)
    assert p.center[0] == pytest.approx(3.0 * 16, abs=0.5)
    assert p.faces[0] == lbm.FaceBc.VELOCITY and p.faces[1] == lbm.FaceBc.OPEN
    assert p.steps_unit == pytest.approx(16 / 0.075, rel=1e-3)
    assert p.frontal_area == pytest.approx(math.pi * SPHERE_D ** 2 / 4, rel=0.01)
    assert p.blockage == pytest.approx(p.frontal_area / (7 * SPHERE_D) ** 2, rel=0.02)


@pytest.mark.parametrize("cells,levels", [(47, 1), (48, 2), (95, 2), (96, 3)])
def test_plan_refined_levels_nest(cells, levels):
    cfg, m = sphere_case(100.0, cells)
    p = T.plan(cfg, m, 1e-3, T.SolverOptions())
    nl = 1 if p.multi is None else len(p.multi.cells)
    assert nl == levels
    if p.multi is None:
        return
    mp = p.multi
    s0 = 1 << (nl - 1)
    assert [(d - 1) * s0 + 1 for d in mp.dims0] == p.dims
    pd = list(mp.dims0)
    org = [0.0, 0.0, 0.0]
    for l, (lo, n) in enumerate(mp.boxes, start=1):
        for k in range(3):
            assert lo[k] >= 3 and lo[k] + n[k] - 1 <= pd[k] - 4  # inside the parent, clear of its faces and sponges
            org[k] += lo[k] * (1 << (nl - l))
        pd = [2 * (n[k] - 1) + 1 for k in range(3)]
        assert int(np.prod(pd)) == mp.cells[l]
    assert org == pytest.approx(mp.org_f)
    # the finest box holds the part with room around it
    q = (m.positions - p.pref) @ p.r.T / p.dx + np.asarray(p.center) - np.asarray(mp.org_f)
    assert (q.min(axis=0) > 4).all() and (q.max(axis=0) < np.asarray(pd) - 5).all()


def test_plan_spinning_sphere_swept_box():
    cfg, m = rotating_sphere_case(1.0, 24, 6.0)
    o = T.SolverOptions()
    o.still_margins.side = 2.0
    p = T.plan(cfg, m, 1e-3, o)
    assert p.spin and p.still and p.multi is None
    assert p.axis_lat == pytest.approx([1.0, 0.0, 0.0])  # the spin axis is the lattice's x
    assert all(f == lbm.FaceBc.OPEN for f in p.faces)
    for k in range(3):
        assert p.box_lo[k] >= 1 and p.box_lo[k] + p.box_n[k] <= p.dims[k] - 1
        c = p.center[k]
        assert p.box_lo[k] <= c - 12 and p.box_lo[k] + p.box_n[k] - 1 >= c + 12  # the sphere (12 cells radius) is inside
    assert 0.5 + 3 * p.nu_lat <= 1.0 + 1e-12  # the relaxation-time limit caps the step
    assert p.steps_unit == pytest.approx(2 * math.pi / np.linalg.norm(p.omega_lat), rel=1e-9)


def test_plan_rejects_bad_configs():
    cfg, m = sphere_case(100.0, 16)
    cfg.speed_m_s = 0.0
    with pytest.raises(ValueError):
        T.plan(cfg, m, 1e-3, T.SolverOptions())
    cfg.speed_m_s = 10.0
    cfg.wind_dir = (0.0, 0.0, 0.0)
    with pytest.raises(ValueError):
        T.plan(cfg, m, 1e-3, T.SolverOptions())
    with pytest.raises(ValueError):
        T.plan(sphere_case(100.0, 16)[0], T.Mesh(np.zeros((0, 3)), np.zeros((0, 3))), 1e-3, T.SolverOptions())


def test_plan_fp16_when_fp32_does_not_fit():
    cfg, m = sphere_case(100.0, 16)
    p32 = T.plan(cfg, m, 1e-3, T.SolverOptions())
    p16 = T.plan(cfg, m, 1e-3, T.SolverOptions(memory_budget=p32.memory - 1))
    assert p32.storage == int(lbm.Storage.FP32) and p16.storage == int(lbm.Storage.FP16)
    assert p16.memory < p32.memory


def test_window_check_steady_and_drift():
    cfg, m = sphere_case(100.0, 16)
    p = T.plan(cfg, m, 1e-3, T.SolverOptions())
    ax = np.array([1.0, 0.0, 0.0])
    rng = np.random.default_rng(1)
    w = np.zeros((4000, 6))
    w[:, 0] = 1.0 + 1e-4 * rng.standard_normal(4000)
    worst, se_rel, trend, half = T._window_check(w, p, ax)
    assert worst < 1e-4 and se_rel < 1e-4 and not trend and half == 2000
    w[:, 0] = np.linspace(1.0, 1.2, 4000) + 1e-4 * rng.standard_normal(4000)
    worst, se_rel, trend, _ = T._window_check(w, p, ax)
    assert worst > 0.04 and trend
    # the trend is removed from the block scatter: a clean drift has a tiny standard error
    assert se_rel < 1e-3


class _FakeLattice:
    """A lattice that returns a fixed force and moment every step and records
    the schedule it was given."""

    made = []

    def __init__(self, setup, geometry=None, probes=None):
        self.setup, self.geometry, self.probes = setup, geometry, probes
        self.calls, self.resets = [], []
        self.steps = 0
        self.force = np.array([2e-3, 0.0, 1e-5, 0.0, 0.0, 0.0])
        _FakeLattice.made.append(self)

    def run(self, a):
        self.calls.append(a.copy())
        self.steps += len(a)
        return np.tile(self.force, (len(a), 1))

    def reset_samples(self):
        self.resets.append(self.steps)

    def vertex_means(self):
        return np.full(len(self.probes.verts), 1.001, dtype=np.float32)

    def slice_means(self):
        n = sum(s.nu * s.nv for s in self.probes.slices)
        out = np.zeros((n, 4), dtype=np.float32)
        out[:, 0] = 1.0
        out[:, 1] = 0.05
        return out

    @property
    def memory_bytes(self):
        return 123

    def close(self):
        pass


def test_run_loop_si_conversion_and_folder(monkeypatch, tmp_path):
    monkeypatch.setattr(lbm, "Lattice", _FakeLattice)
    _FakeLattice.made.clear()
    cfg, m = sphere_case(100.0, 16, duration=15.0)
    r = T.run_with(cfg, m, 1e-3, T.SolverOptions(gpu_voxelizer=False))
    lat = _FakeLattice.made[-1]
    p = T.plan(cfg, m, 1e-3, T.SolverOptions())
    s = r.summary
    # a constant force converges once the minimum window has passed
    assert s.converged
    fscale = 1.2 * p.dx ** 4 / p.dt ** 2
    assert s.drag_n == pytest.approx(2e-3 * fscale, rel=1e-12)
    assert s.lift_n == pytest.approx(1e-5 * fscale, rel=1e-12)
    assert s.cd == pytest.approx(s.drag_n / (0.5 * 1.2 * 100.0 * p.frontal_area), rel=1e-12)
    assert s.reynolds == pytest.approx(100.0, rel=1e-3)
    # the schedule: still steps, sampling from the window start every steps_unit/100 steps, one reset there
    a = np.concatenate(lat.calls)
    assert len(a) == s.steps
    assert np.all(a["rot"] == np.eye(3))
    unit = p.steps_unit
    w0 = max(int(0.35 * 15.0 * unit), int(0.5 * unit))
    every = max(int(unit // 100), 1)
    k = np.arange(len(a)) + 1
    assert np.array_equal(a["sample"] != 0, (k > w0) & ((k - w0) % every == 0))
    assert len(lat.resets) == 1 and lat.resets[0] <= w0 < lat.resets[0] + len(lat.calls[0])
    # probes and slices
    assert len(lat.probes.verts) == len(m.positions)
    pconv = 1.2 * (p.dx / p.dt) ** 2 / 3.0
    assert r.surface_pressure_pa[0] == pytest.approx(np.float32(0.001) * pconv, rel=1e-3)
    assert r.slices[0].name == "along" and r.slices[1].name == "across"
    sp = r.slices[0].fields[0]
    assert sp.name == "speed" and sp.data[0] == pytest.approx(0.05 * p.dx / p.dt, rel=1e-6)
    T.write_run(r, tmp_path)
    # the engine's run folder (crates/engine/src/wind.rs:463-497)
    assert (tmp_path / "field.pressure.f32").stat().st_size == 4 * len(m.positions)
    assert np.array_equal(np.fromfile(tmp_path / "field.cp.f32", dtype="<f4"), r.surface_cp)
    hdr = json.loads((tmp_path / "slice.along.json").read_text())
    assert hdr["nu"] * hdr["nv"] * 4 == (tmp_path / "slice.along.speed.f32").stat().st_size
    assert [f["name"] for f in hdr["fields"]] == ["speed", "pressure", "u", "v"]
    run = json.loads((tmp_path / "run.json").read_text())
    assert run["kind"] == "wind" and run["summary"]["converged"] and run["summary"]["storage"] == "Fp32"
    assert [f["name"] for f in run["fields"]] == ["pressure", "cp"] and run["fields"][0]["min"] == -run["fields"][0]["max"]
    assert [s["name"] for s in run["slices"]] == ["along", "across"]
    assert (tmp_path / "history.csv").read_text().splitlines()[0] == "t,fx,fy,fz,mx,my,mz"


def test_run_loop_spin_schedule(monkeypatch):
    monkeypatch.setattr(lbm, "Lattice", _FakeLattice)
    _FakeLattice.made.clear()
    cfg, m = rotating_sphere_case(1.0, 12, 2.0)
    r = T.run_with(cfg, m, 1e-3, T.SolverOptions(gpu_voxelizer=False))
    lat = _FakeLattice.made[-1]
    p = T.plan(cfg, m, 1e-3, T.SolverOptions())
    a = np.concatenate(lat.calls)
    w = np.linalg.norm(p.omega_lat)
    ramp = math.ceil(0.5 * 2 * math.pi / w)
    # smoothstep spin-up, then full speed; each step's previous rotation is the last step's
    f = np.linalg.norm(a["omega"], axis=1) / w
    x = (np.arange(ramp) + 0.5) / ramp
    assert f[:ramp] == pytest.approx(x * x * (3 - 2 * x), rel=1e-12)
    assert np.all(f[ramp:] == pytest.approx(1.0))
    assert np.array_equal(a["rot_prev"][1:], a["rot"][:-1])
    assert np.array_equal(a["rot_prev"][0], np.eye(3))
    th = np.cumsum(f * w)
    assert a["rot"][-1] == pytest.approx(T.rotation([1.0, 0.0, 0.0], th[-1]), abs=1e-9)
    assert r.summary.thrust_n is not None and r.summary.cd is None and r.summary.time_unit == "revolutions"

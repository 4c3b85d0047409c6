"""The study layer over the engine: a wind-tunnel run of a part, from a
configuration in SI units to SI results (crates/cfd/src/tunnel.rs).

`plan` sizes the tunnel (frame along the wind, cells across the part, domain
margins, refinement boxes for still parts, time step from the Mach and
relaxation-time limits, sponges, storage); `run_with` voxelizes the part,
builds the lattice (one D3Q19 level, nested D3Q27 levels, or a spinning part),
steps it in batches with the spin-up schedule and the convergence window,
and converts the window's mean force and moment, the surface pressure and the
flow slices to SI.  `write_run` stores a result in the run-folder layout
(docs/ARCHITECTURE.md "Storage"; crates/cfd/examples/run_stl.rs:125-140).

Geometry is a triangle mesh in metres: `Mesh(positions (n, 3), triangles
(m, 3))`.  All lattice work goes through simlab_b200.lbm and
simlab_b200.mlattice (the C ABI).
"""
from __future__ import annotations

import json
import math
import time
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

# ---------------------------------------------------------------- configuration (simlab_core::config, tunnel.rs:150-234)


@dataclass
class Mesh:
    """A closed triangle surface, positions in metres."""

    positions: np.ndarray
    triangles: np.ndarray

    def __post_init__(self):
        self.positions = np.asarray(self.positions, dtype=np.float64).reshape(-1, 3)
        self.triangles = np.asarray(self.triangles, dtype=np.uint32).reshape(-1, 3)

    def bounds(self):
        return self.positions.min(axis=0), self.positions.max(axis=0)

    def triangle_areas(self) -> np.ndarray:
        p = self.positions[self.triangles]
        return 0.5 * np.linalg.norm(np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), axis=1)

    def volume(self) -> float:
        p = self.positions[self.triangles]
        return float(np.einsum("ij,ij->i", p[:, 0], np.cross(p[:, 1], p[:, 2])).sum() / 6.0)


@dataclass
class Air:
    density: float = 1.204              # kg/m^3
    kinematic_viscosity: float = 1.516e-5  # m^2/s


@dataclass
class Spin:
    rpm: float
    axis: Sequence[float]
    center_mm: Sequence[float] = (0.0, 0.0, 0.0)


@dataclass
class WindConfig:
    """simlab_core::WindConfig: `quality` is "draft", "normal", "fine" or an
    int (cells across the part's largest size); `duration` in flow passes
    (still air: revolutions), None for the quality's default."""

    wind_dir: Sequence[float] = (1.0, 0.0, 0.0)
    speed_m_s: float = 10.0
    air: Air = field(default_factory=Air)
    spin: Optional[Spin] = None
    quality: object = "normal"
    duration: Optional[float] = None


@dataclass
class Margins:
    upstream: float
    downstream: float
    side: float


@dataclass
class SolverOptions:
    """tunnel.rs:160-234 with the reference's defaults."""

    cells_across: Optional[int] = None
    storage: Optional[int] = None          # lbm Storage; None: FP32 when it fits memory_budget, else FP16
    memory_budget: Optional[int] = None
    max_lattice_speed: float = 0.075
    max_tip_speed: float = 0.10
    max_tau: float = 1.0
    wind_margins: Margins = field(default_factory=lambda: Margins(2.5, 5.0, 3.0))
    still_margins: Margins = field(default_factory=lambda: Margins(2.5, 2.5, 1.0))
    smagorinsky: float = 0.10
    tolerance: float = 0.005
    spin_ramp_revs: float = 0.5
    vertex_offset: float = 1.0
    side_bc: str = "open"                   # or "velocity"
    sponge_sigma: float = 0.1
    sponge_widths: Sequence[float] = (0.4, 1.0, 0.4)
    absorb_velocity: bool = False
    total_pressure_inlet: bool = True
    wall_model: bool = False
    refine: bool = True
    gpu_voxelizer: bool = True             # static parts: voxelize on the device (the host voxelizer's result, bit for bit)


def cells_across(q) -> int:
    if isinstance(q, (int, np.integer)):
        return int(min(max(int(q), 8), 4096))
    return {"draft": 64, "normal": 128, "fine": 192}[q]


def default_duration(q, still_spin: bool) -> float:
    d, n, f = (8.0, 12.0, 16.0) if still_spin else (20.0, 40.0, 60.0)
    return d if q == "draft" else (f if q == "fine" else n)


def thin_cells_target(q) -> int:
    return 0 if isinstance(q, (int, np.integer)) else {"draft": 16, "normal": 24, "fine": 32}[q]


THIN_MAX_BOOST = 8
SIDE_MIN_FRONT = 1.5
REFINE_THIN = 2.0
# refinement-box extents per level (upstream, downstream, side) in wake sizes
REFINE_EXT = ((1.2, 3.0, 1.0), (0.8, 1.6, 0.75), (0.65, 1.0, 0.65))


def cells_for_thin(n_q: int, n_thin: int, l_ref: float, thin: float) -> int:
    if thin <= 0.0 or l_ref <= 0.0:
        return n_q
    want = int(math.ceil(n_thin * l_ref / thin))
    return min(max(want, n_q), n_q * THIN_MAX_BOOST)


def thin_cost_cap(q) -> float:
    return {"draft": 4.0e11, "normal": 4.0e12}.get(q, 2.0e13) if not isinstance(q, (int, np.integer)) else 2.0e13


def still_levels(n_across: int) -> int:
    nl = 1
    while nl < 4 and n_across / float(1 << nl) >= 24.0:
        nl += 1
    return nl


def frame(main) -> np.ndarray:
    """Rows ex (along `main`), ey, ez (up, unless `main` is nearly vertical)."""
    ex = np.asarray(main, dtype=np.float64)
    ex = ex / np.linalg.norm(ex)
    up = np.array([1.0, 0.0, 0.0]) if abs(ex[2]) > 0.95 else np.array([0.0, 0.0, 1.0])
    ez = up - ex * np.dot(up, ex)
    ez /= np.linalg.norm(ez)
    return np.array([ex, np.cross(ez, ex), ez])


def rotation(a, t: float) -> np.ndarray:
    """Rotation by t about the unit axis a (tunnel.rs rotation)."""
    a = np.asarray(a, dtype=np.float64)
    c, s, k = math.cos(t), math.sin(t), 1.0 - math.cos(t)
    return np.array([[c + a[0] * a[0] * k, a[0] * a[1] * k - a[2] * s, a[0] * a[2] * k + a[1] * s],
                     [a[1] * a[0] * k + a[2] * s, c + a[1] * a[1] * k, a[1] * a[2] * k - a[0] * s],
                     [a[2] * a[0] * k - a[1] * s, a[2] * a[1] * k + a[0] * s, c + a[2] * a[2] * k]])


def frontal_area(m: Mesh, r: np.ndarray, res: int = 1024) -> float:
    """The part's shadow on the plane across the wind, rasterized on a grid
    of `res` pixels across its larger side (tunnel.rs frontal_area)."""
    pts = m.positions @ r[1:3].T
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    size = float(max(hi - lo))
    if size <= 0.0:
        return 0.0
    h = size / res
    nu, nv = int(math.ceil((hi[0] - lo[0]) / h)) + 1, int(math.ceil((hi[1] - lo[1]) / h)) + 1
    img = np.zeros((nv, nu), dtype=bool)
    for t in m.triangles:
        a, b, c = pts[t[0]], pts[t[1]], pts[t[2]]
        i0 = max(int(math.floor((min(a[0], b[0], c[0]) - lo[0]) / h)), 0)
        i1 = min(int(math.ceil((max(a[0], b[0], c[0]) - lo[0]) / h)), nu - 1)
        j0 = max(int(math.floor((min(a[1], b[1], c[1]) - lo[1]) / h)), 0)
        j1 = min(int(math.ceil((max(a[1], b[1], c[1]) - lo[1]) / h)), nv - 1)
        if i1 < i0 or j1 < j0:
            continue
        xs = lo[0] + (np.arange(i0, i1 + 1) + 0.5) * h
        ys = lo[1] + (np.arange(j0, j1 + 1) + 0.5) * h
        X, Y = np.meshgrid(xs, ys)

        def e(p, q):
            return (q[0] - p[0]) * (Y - p[1]) - (q[1] - p[1]) * (X - p[0])

        e0, e1, e2 = e(a, b), e(b, c), e(c, a)
        inside = ((e0 >= 0) & (e1 >= 0) & (e2 >= 0)) | ((e0 <= 0) & (e1 <= 0) & (e2 <= 0))
        img[j0:j1 + 1, i0:i1 + 1] |= inside
    return float(img.sum()) * h * h


# ---------------------------------------------------------------- plan (tunnel.rs:541-811)
@dataclass
class MultiPlan:
    dims0: list
    boxes: list            # (lo[3], n[3]) per finer level, in its parent's nodes
    org_f: list            # finest-level node of the coarsest level's node 0
    cells: list


@dataclass
class Plan:
    r: np.ndarray          # rows: the lattice axes in model axes (x along the wind or the spin axis)
    pref: np.ndarray       # model point at the lattice's `center` (m)
    dx: float
    dt: float
    dims: list
    center: list
    u_lat: float
    omega_lat: np.ndarray
    nu_lat: float
    spin: bool
    still: bool
    cells_across: int
    d_front: float
    frontal_area: float
    steps_unit: float      # steps per flow pass (still air: per revolution)
    duration: float
    storage: int
    memory: int
    blockage: float
    sponge: list
    faces: list
    rotor_radius: float
    axis_lat: np.ndarray
    axis_model: np.ndarray
    box_lo: list
    box_n: list
    est_records: int
    updates_per_step: float
    d_thin: float
    multi: Optional[MultiPlan] = None
    thin: Optional[tuple] = None   # (target, wanted) cells across the thin size when raised for it

    def cost(self) -> float:
        return self.updates_per_step * math.ceil(self.duration * self.steps_unit)

    def cells_thin(self) -> float:
        return self.d_thin / self.dx


def _pop_bytes(storage: int) -> int:
    return {0: 4, 1: 2, 2: 2, 3: 8}[int(storage)]


def plan(cfg: WindConfig, m: Mesh, unit_m: float, opt: SolverOptions, budget: Optional[int] = None) -> Plan:
    from .lbm import FaceBc, Storage

    if len(m.triangles) == 0:
        raise ValueError("the part has no surface")
    speed = float(cfg.speed_m_s)
    if not (speed >= 0.0) or not math.isfinite(speed):
        raise ValueError("wind speed must be zero or positive")
    spin = cfg.spin if (cfg.spin is not None and cfg.spin.rpm != 0.0 and np.linalg.norm(cfg.spin.axis) > 0.0) else None
    if speed == 0.0 and spin is None:
        raise ValueError("still air needs a spinning part; set a wind speed or a spin")
    if speed > 0.0 and np.linalg.norm(cfg.wind_dir) == 0.0:
        raise ValueError("the wind direction is zero")
    still = speed == 0.0
    r = frame(spin.axis if still else cfg.wind_dir)
    blo, bhi = m.bounds()
    pref = np.asarray(spin.center_mm, dtype=np.float64) * unit_m if spin is not None else 0.5 * (blo + bhi)
    v = m.positions - pref
    q = v @ r.T
    lo, hi = q.min(axis=0), q.max(axis=0)
    axis_model = np.asarray(spin.axis, dtype=np.float64) / np.linalg.norm(spin.axis) if spin is not None else np.array([1.0, 0.0, 0.0])
    a = v @ axis_model
    rotor_radius = float(np.sqrt(np.maximum(np.einsum("ij,ij->i", v, v) - a * a, 0.0)).max())
    alo, ahi = float(a.min()), float(a.max())
    axis_lat = r @ axis_model
    if spin is not None:  # the swept cylinder's box
        for k in range(3):
            e = rotor_radius * math.sqrt(max(1.0 - axis_lat[k] ** 2, 0.0))
            p0, p1 = alo * axis_lat[k], ahi * axis_lat[k]
            lo[k], hi[k] = min(p0, p1) - e, max(p0, p1) + e
    ext = hi - lo
    l_ref = float(ext.max())
    if l_ref <= 0.0:
        raise ValueError("the part has no size")
    d_thin = max(min(ext[1], ext[2]), l_ref * 1e-3) if spin is None else l_ref
    if opt.cells_across is not None:
        n_across = int(opt.cells_across)
    else:
        n_q = cells_across(cfg.quality)
        n_t = thin_cells_target(cfg.quality)
        want = cells_for_thin(n_q, n_t, l_ref, d_thin)
        n_across = n_q
        if want > n_q:
            # the finest grid up to `want` that fits the budget and the time cap, ~8 % coarser a try
            bud = budget if budget is not None else opt.memory_budget
            base = plan(cfg, m, unit_m, _with(opt, cells_across=n_q), bud)
            t_cap = max(thin_cost_cap(cfg.quality), base.cost())
            n = want
            while True:
                p = plan(cfg, m, unit_m, _with(opt, cells_across=n), bud)
                fits = (bud is None or p.memory <= bud) and p.cost() <= t_cap
                if fits or n <= n_q:
                    p = p if fits else base
                    p.thin = (n_t, want)
                    return p
                n = max(int(n * 0.92), n_q)
    dx = l_ref / n_across
    d_front = max(2.0 * rotor_radius if still else max(ext[1], ext[2]), l_ref * 1e-3)
    d_box = min(d_front, REFINE_THIN * d_thin) if spin is None else d_front
    mg = opt.still_margins if still else opt.wind_margins
    side = mg.side * d_front if still else max(mg.side * d_box, SIDE_MIN_FRONT * d_front)
    dom_lo = np.array([lo[0] - mg.upstream * d_front, lo[1] - side, lo[2] - side])
    dom_hi = np.array([hi[0] + mg.downstream * d_front, hi[1] + side, hi[2] + side])
    dims = [int(math.ceil((dom_hi[k] - dom_lo[k]) / dx)) + 1 for k in range(3)]
    center = [-dom_lo[k] / dx for k in range(3)]
    multi = None
    if spin is None and opt.refine:
        nl = still_levels(n_across)
        if nl > 1:
            s0 = float(1 << (nl - 1))
            dx0 = dx * s0
            dims0 = [int(math.ceil((dom_hi[k] - dom_lo[k]) / dx0)) + 1 for k in range(3)]
            dims = [int((dims0[k] - 1) * s0) + 1 for k in range(3)]
            center = [-dom_lo[k] / dx for k in range(3)]
            lo_c = [(center[k] + lo[k] / dx) / s0 for k in range(3)]
            hi_c = [(center[k] + hi[k] / dx) / s0 for k in range(3)]
            pd = list(dims0)
            boxes, org = [], [0.0, 0.0, 0.0]
            cells = [int(np.prod(dims0, dtype=np.int64))]
            for l in range(1, nl):
                sc = float(1 << (nl - l))  # finest cells per level (l-1) cell
                df = d_box / dx / sc
                eu, ed, es = REFINE_EXT[l - 1]
                e_lo, e_hi = [eu * df, es * df, es * df], [ed * df, es * df, es * df]
                b_lo, b_n = [0, 0, 0], [0, 0, 0]
                for k in range(3):
                    aa = max(int(math.floor(lo_c[k] - e_lo[k])), 3)
                    bb = min(int(math.ceil(hi_c[k] + e_hi[k])), pd[k] - 4)
                    b_lo[k], b_n[k] = aa, max(bb - aa + 1, 8)
                for k in range(3):
                    org[k] += b_lo[k] * sc
                    lo_c[k] = 2.0 * (lo_c[k] - b_lo[k])
                    hi_c[k] = 2.0 * (hi_c[k] - b_lo[k])
                    pd[k] = 2 * (b_n[k] - 1) + 1
                cells.append(int(np.prod(pd, dtype=np.int64)))
                boxes.append((b_lo, b_n))
            multi = MultiPlan(dims0=dims0, boxes=boxes, org_f=org, cells=cells)
    # time step from the Mach limit, then the viscosity limit
    omega = spin.rpm * 2.0 * math.pi / 60.0 if spin is not None else 0.0
    umax_phys = speed + abs(omega) * rotor_radius
    ulat_max = opt.max_tip_speed if spin is not None else opt.max_lattice_speed
    dt = ulat_max * dx / umax_phys
    nu = cfg.air.kinematic_viscosity
    nu_max = (opt.max_tau - 0.5) / 3.0
    if nu * dt / (dx * dx) > nu_max:
        dt = nu_max * dx * dx / nu
    nu_lat = nu * dt / (dx * dx)
    u_lat = speed * dt / dx
    omega_lat = axis_lat * (omega * dt)
    steps_unit = 2.0 * math.pi / (abs(omega) * dt) if still else l_ref / speed / dt
    duration = max(cfg.duration if cfg.duration is not None else default_duration(cfg.quality, still), 1.0)
    n = int(np.prod(dims, dtype=np.int64))
    if spin is not None:  # the swept box in cells
        box_lo, box_n = [0, 0, 0], [0, 0, 0]
        for k in range(3):
            aa = int(math.floor(center[k] + lo[k] / dx - 3.0))
            bb = int(math.ceil(center[k] + hi[k] / dx + 3.0))
            box_lo[k] = max(aa, 1)
            box_n[k] = max(min(bb, dims[k] - 2) - box_lo[k] + 1, 1)
    else:
        box_lo, box_n = [0, 0, 0], [0, 0, 0]
    area_m2 = float(m.triangle_areas().sum())
    est_records = int(np.prod(box_n)) if spin is not None else int(2.0 * area_m2 / (dx * dx)) + 1000
    faces_cells = 2 * (dims[0] * dims[1] + dims[1] * dims[2] + dims[0] * dims[2])

    def mem_for(s: int) -> int:
        if multi is not None:
            pops = sum(c * (2 * 27 * _pop_bytes(s) + 4 + 8) for c in multi.cells)
            return pops + est_records * 24 * 4 * 2 + 64 * 1024 * 1024
        return n * (19 * _pop_bytes(s) + 4) + est_records * 40 * 4 + faces_cells * 44 + 64 * 1024 * 1024

    n_max = max(multi.cells) if multi is not None else n

    def fits_layout(s: int) -> bool:
        # this engine's limits: 32-bit cell indices per level (refined), the
        # single lattice's own bound per storage (lbm_max_cells)
        if multi is not None:
            return n_max < (1 << 32) - 1
        from .lbm import library
        return n <= int(library().lbm_max_cells(int(s)))

    bud = budget if budget is not None else opt.memory_budget
    if opt.storage is not None:
        storage = int(opt.storage)
    elif (bud is not None and mem_for(int(Storage.FP32)) > bud) or not fits_layout(int(Storage.FP32)):
        storage = int(Storage.FP16)
    else:
        storage = int(Storage.FP32)
    memory = mem_for(storage) if fits_layout(storage) else (1 << 62)
    frontal = math.pi * rotor_radius ** 2 if still else frontal_area(m, r)
    blockage = frontal / ((dom_hi[1] - dom_lo[1]) * (dom_hi[2] - dom_lo[2]))
    dxs = dx * ((dims[0] - 1) / (multi.dims0[0] - 1)) if multi is not None else dx  # sponge widths in coarsest cells

    def cl(x, lo_):
        return int(max(_round_away(x / dxs), lo_))

    if still:
        sp = cl(opt.sponge_widths[2] * d_front, 8)
        sponge, faces = [sp] * 6, [FaceBc.OPEN] * 6
    else:
        sd = FaceBc.VELOCITY if opt.side_bc == "velocity" else FaceBc.OPEN
        s_side = cl(opt.sponge_widths[2] * d_front, 6)
        sponge = [cl(opt.sponge_widths[0] * d_front, 6), cl(opt.sponge_widths[1] * d_front, 8)] + [s_side] * 4
        faces = [FaceBc.VELOCITY, FaceBc.OPEN] + [sd] * 4
    if multi is not None:
        nl = len(multi.cells)
        ups = sum(c * float(1 << l) for l, c in enumerate(multi.cells)) / float(1 << (nl - 1))
    else:
        ups = float(n)
    return Plan(r=r, pref=pref, dx=dx, dt=dt, dims=dims, center=center, u_lat=u_lat, omega_lat=omega_lat, nu_lat=nu_lat,
                spin=spin is not None, still=still, cells_across=n_across, d_front=d_front, frontal_area=frontal, steps_unit=steps_unit,
                duration=duration, storage=storage, memory=memory, blockage=blockage, sponge=sponge, faces=faces, rotor_radius=rotor_radius,
                axis_lat=axis_lat, axis_model=axis_model, box_lo=box_lo, box_n=box_n, est_records=est_records, updates_per_step=ups,
                d_thin=d_thin, multi=multi)


def _with(opt: SolverOptions, **kw) -> SolverOptions:
    d = dict(opt.__dict__)
    d.update(kw)
    return SolverOptions(**d)


# ---------------------------------------------------------------- results (tunnel.rs:236-330)
@dataclass
class SliceField:
    name: str
    label: str
    unit: str
    min: float
    max: float
    data: np.ndarray = field(repr=False)   # f32, index iv * nu + iu; NaN inside the part


@dataclass
class FlowSlice:
    name: str
    label: str
    origin_mm: list        # corner of the first pixel, model units
    u_mm: list             # the whole slice's extent along u
    v_mm: list
    nu: int
    nv: int
    fields: list


@dataclass
class WindSummary:
    kind: str
    headline: str
    force_n: list
    moment_nm: list
    drag_n: float
    lift_n: float
    side_n: float
    cd: Optional[float]
    ref_area_mm2: float
    thrust_n: Optional[float]
    torque_nm: Optional[float]
    power_w: Optional[float]
    reynolds: float
    cells: int
    steps: int
    mlups: float
    seconds: float
    converged: bool
    warnings: list
    grid: list
    cells_across: int
    dx_mm: float
    dt_s: float
    mach_lattice: float
    tau: float
    blockage: float
    storage: str
    memory_bytes: int
    averaged_over: float
    simulated: float
    time_unit: str
    q_ref_pa: float
    thin_mm: float
    cells_thin: float


@dataclass
class WindResult:
    summary: WindSummary
    surface_pressure_pa: np.ndarray   # f32 per mesh vertex
    surface_cp: np.ndarray
    slices: list
    history: list                     # (flow passes or revolutions, force (3), moment (3)) per batch, model axes, SI


class Cancelled(RuntimeError):
    pass


def sig(x: float, n: int) -> str:
    """x with n significant figures in plain decimal notation."""
    if x == 0.0 or not math.isfinite(x):
        return f"{x}"
    mag = math.floor(math.log10(abs(x)))
    dec = max(n - 1 - mag, 0)
    f = 10.0 ** (n - 1 - mag)
    return f"{_round_away(x * f) / f:.{dec}f}"


def _round_away(x: float) -> float:
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _normalize(v: np.ndarray) -> np.ndarray:
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return np.divide(v, n, out=np.zeros_like(v), where=n > 0)


def _rotations(a: np.ndarray, th: np.ndarray) -> np.ndarray:
    """rotation(a, t) for every t of th: (n, 3, 3)."""
    c, s = np.cos(th), np.sin(th)
    k = 1.0 - c
    R = np.empty((len(th), 3, 3))
    R[:, 0, 0] = c + a[0] * a[0] * k
    R[:, 0, 1] = a[0] * a[1] * k - a[2] * s
    R[:, 0, 2] = a[0] * a[2] * k + a[1] * s
    R[:, 1, 0] = a[1] * a[0] * k + a[2] * s
    R[:, 1, 1] = c + a[1] * a[1] * k
    R[:, 1, 2] = a[1] * a[2] * k - a[0] * s
    R[:, 2, 0] = a[2] * a[0] * k - a[1] * s
    R[:, 2, 1] = a[2] * a[1] * k + a[0] * s
    R[:, 2, 2] = c + a[2] * a[2] * k
    return R


def _thin_check(warnings: list, solid_cells: float, m: Mesh, dx: float) -> None:
    vol = abs(m.volume())
    if vol > 0.0:
        ratio = solid_cells * dx ** 3 / vol
        if ratio < 0.6:
            warnings.append(f"only {ratio * 100:.0f} % of the model's volume became solid cells: parts of it are thinner than a "
                            "cell; they still block the air, but a finer grid gives better forces")
    else:
        warnings.append("the surface is open; inside and outside were decided by votes along three axes")


def _thin_warning(p: Plan) -> Optional[str]:
    if p.spin:
        return None
    have = p.cells_thin()
    if p.thin is not None and have + 0.5 < p.thin[0]:
        return (f"the part is {sig(p.d_thin * 1e3, 2)} mm thin across the wind and has {have:.0f} cells across that size, not the "
                f"{p.thin[0]} asked for (that needs {p.thin[1]} across the whole part; memory and run time allow {p.cells_across}), "
                "so its drag is less certain")
    if p.thin is None and have < 8.0:
        return f"the part is {sig(p.d_thin * 1e3, 2)} mm thin across the wind with {have:.0f} cells across it: its drag is rough"
    return None


MLUPS_PACE = 2800.0  # the update rate that sizes a batch (tunnel.rs:145): a batch is ~1/4 s of it


def _slices_for(p: Plan) -> tuple[int, list]:
    """Two slices through the part's centre in global finest cells, one pixel
    every `pitch` cells, the pitch doubled until a slice has at most ~4 M
    pixels on a refined grid (tunnel.rs:978-1000)."""
    nx, ny, nz = p.dims
    pitch = 1
    if p.multi is not None:
        while max((nx // pitch) * (nz // pitch), (ny // pitch) * (nz // pitch)) > 4_000_000:
            pitch *= 2

    def snap(x):
        return max(int(_round_away(x / pitch)) * pitch, pitch)

    def span(n):
        return max(int((n - 1 - pitch) / pitch), 1)

    xc = snap(min(max(p.center[0], 1.0), nx - 2.0))
    yc = snap(min(max(p.center[1], 1.0), ny - 2.0))
    return pitch, [((pitch, yc, pitch), (pitch, 0, 0), (0, 0, pitch), span(nx), span(nz)),
                   ((xc, pitch, pitch), (0, pitch, 0), (0, 0, pitch), span(ny), span(nz))]


def run_with(cfg: WindConfig, m: Mesh, unit_m: float, opt: Optional[SolverOptions] = None, progress=None) -> WindResult:
    """A wind-tunnel run through the C ABI (tunnel.rs:903-1390): `m` in
    metres, `unit_m` metres per model unit (Spin.center_mm and the slices'
    coordinates).  `progress(fraction, message, metrics)` is called after
    every batch; it returns True to cancel."""
    from .lbm import Lattice, LatticeSetup, Probes, SliceDef, SpinGeometry, StepIn, Storage, steps_array, voxelize_spin, voxelize_static
    from .lbm import STEP_DTYPE
    from .mlattice import LevelBox, MultiLattice, MultiSetup

    opt = opt or SolverOptions()
    t_start = time.perf_counter()
    p = plan(cfg, m, unit_m, opt)
    warnings: list = []
    R = p.r

    def to_body(x):
        return ((x - p.pref) @ R.T) / p.dx

    def to_lat(x):
        return to_body(x) + np.asarray(p.center)

    if p.spin:
        s = to_body(m.positions)
        blo, bhi = s.min(axis=0), s.max(axis=0)
        vol = float(np.prod(bhi - blo + 2.0))
        h = max((vol / 64e6) ** (1.0 / 3.0), 0.125)  # occupancy 8x finer than the lattice, at most ~64 M samples
        vox = voxelize_spin(s, m.triangles, p.axis_lat, h)
        solid = sum(int(w).bit_count() for w in np.asarray(vox.occ_bits, dtype=np.uint32)) * vox.occ_h ** 3
        _thin_check(warnings, solid, m, p.dx)
        geom = SpinGeometry(vox=vox, box_lo=p.box_lo, box_n=p.box_n)
    elif p.multi is not None:
        b = p.multi.boxes[-1]
        fd = [2 * (b[1][k] - 1) + 1 for k in range(3)]
        vox = voxelize_static(to_lat(m.positions) - np.asarray(p.multi.org_f), m.triangles, fd, lattice=27, device=opt.gpu_voxelizer)
        _thin_check(warnings, float(len(vox.solid)), m, p.dx)
        geom = vox
    else:
        vox = voxelize_static(to_lat(m.positions), m.triangles, p.dims, device=opt.gpu_voxelizer)
        _thin_check(warnings, float(len(vox.solid)), m, p.dx)
        geom = vox

    # surface probes: vertices with area-weighted normals, pointing out of the part
    flip = -1.0 if m.volume() < 0.0 else 1.0
    P = m.positions[m.triangles]
    tn = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    vn = np.zeros_like(m.positions)
    for c in range(3):
        np.add.at(vn, m.triangles[:, c], tn)
    vn = (_normalize(vn) * flip) @ R.T
    vb = to_body(m.positions)
    verts = [(vb[i], vn[i]) for i in range(len(vb))]
    pitch, slices = _slices_for(p)
    probes = Probes(verts=verts, slices=[SliceDef(origin=s[0], u=s[1], v=s[2], nu=s[3], nv=s[4]) for s in slices],
                    vertex_offset=opt.vertex_offset)
    u_inf = (p.u_lat, 0.0, 0.0)
    if p.multi is None:
        setup = LatticeSetup(dims=p.dims, faces=p.faces, nu=p.nu_lat, smagorinsky=opt.smagorinsky, u_inf=u_inf, u_init=u_inf, sponge=p.sponge,
                             sponge_tau=1.0, sponge_sigma=opt.sponge_sigma, absorb_velocity=opt.absorb_velocity and not p.still,
                             total_pressure_inlet=opt.total_pressure_inlet, storage=Storage(p.storage), center=p.center, wall_model=opt.wall_model)
        lat = Lattice(setup, geom, probes)
        sub_steps = 1
    else:
        mp = p.multi
        nl = len(mp.cells)
        setup = MultiSetup(dims0=mp.dims0, boxes=[LevelBox(lo=b[0], n=b[1]) for b in mp.boxes], faces=p.faces, nu0=p.nu_lat / float(1 << (nl - 1)),
                           smagorinsky=0.0, u_inf=u_inf, u_init=u_inf, sponge=p.sponge, sponge_tau=1.0, sponge_sigma=opt.sponge_sigma,
                           absorb_velocity=opt.absorb_velocity, total_pressure_inlet=opt.total_pressure_inlet, storage=Storage(p.storage),
                           center=[p.center[k] - mp.org_f[k] for k in range(3)])
        lat = MultiLattice(setup, geom, probes)
        sub_steps = lat.sub_steps()
    try:
        return _solve(cfg, m, unit_m, opt, p, lat, sub_steps, slices, warnings, t_start, progress, STEP_DTYPE)
    finally:
        lat.close()


def _window_check(w: np.ndarray, p: Plan, axis_l: np.ndarray):
    """Convergence of the window's mean (tunnel.rs:1154-1185): the halves'
    disagreement, the standard error from 8 block means about their linear
    trend, and whether the halves differ by a real drift."""
    sigs = [w[:, :3] @ axis_l, w[:, 3:] @ axis_l] if p.spin else [w[:, 0]]
    half = len(w) // 2
    worst = se_rel = 0.0
    trend = False
    nbk = 8
    bl = len(w) // nbk
    xs = np.arange(nbk) - (nbk - 1) / 2.0
    if bl == 0:  # fewer samples than blocks: no block statistics (the reference's 0/0 gives no trend and no error)
        for s in sigs:
            m1, m2 = s[:half].mean(), s[half:].mean()
            sc = 0.5 * (abs(m1) + abs(m2))
            if sc > 0.0:
                worst = max(worst, abs(m2 - m1) / 2.0 / sc)
        return worst, se_rel, trend, half
    for s in sigs:
        m1, m2 = s[:half].mean(), s[half:].mean()
        sc = 0.5 * (abs(m1) + abs(m2))
        bm = s[:nbk * bl].reshape(nbk, bl).mean(axis=1)
        mm = bm.mean()
        slope = float((xs * (bm - mm)).sum() / (xs * xs).sum())
        sd = math.sqrt(float(((bm - mm - slope * xs) ** 2).sum()) / (nbk - 2))
        se = sd / math.sqrt(nbk)
        if sc > 0.0:
            worst = max(worst, abs(m2 - m1) / 2.0 / sc)
            se_rel = max(se_rel, se / sc)
            trend |= abs(m2 - m1) > 6.0 * se
    return worst, se_rel, trend, half


def _solve(cfg, m, unit_m, opt, p, lat, ss, slices, warnings, t_start, progress, STEP_DTYPE) -> WindResult:
    total = int(math.ceil(math.ceil(p.duration * p.steps_unit) / ss)) * ss
    om_mag = float(np.linalg.norm(p.omega_lat))
    ramp = int(math.ceil(opt.spin_ramp_revs * 2.0 * math.pi / om_mag)) if p.spin else 0
    unit = p.steps_unit
    # wind: skip the first 35 % of the run and average at least 10 passes;
    # still air: skip 3 revolutions, average at least 2
    tr_units, min_units = (3.0, 2.0) if p.still else (0.35 * p.duration, 10.0)
    w0 = max(int(min(tr_units, 0.35 * p.duration) * unit), ramp + int(0.5 * unit))
    min_win = int(min(min_units, 0.3 * p.duration) * unit)
    w0 = min(w0, total // 2)
    every = max(int(math.floor(unit / 100.0)), 1)
    batch = int(math.ceil(min(max(int(0.25 * MLUPS_PACE * 1e6 / p.updates_per_step), 16), 4096) / ss)) * ss
    axis_l = p.axis_lat / np.linalg.norm(p.axis_lat)
    w_spin = float(np.dot(p.omega_lat, axis_l))
    fscale = cfg.air.density * p.dx ** 4 / (p.dt * p.dt)
    mscale = fscale * p.dx
    R = p.r
    hist = np.zeros((total, 6))
    history = []
    theta, rot_prev = 0.0, np.eye(3)
    step, converged, sampling = 0, False, False
    t_loop = time.perf_counter()
    while step < total:
        nb = min(batch, total - step)
        s = np.arange(step, step + nb)
        a = np.zeros(nb, dtype=STEP_DTYPE)
        if p.spin:
            x = (s + 0.5) / max(ramp, 1)
            f = np.where(s < ramp, x * x * (3.0 - 2.0 * x), 1.0)
            th = np.cumsum(np.concatenate(([theta], f * w_spin)))[1:]  # signed: negative rpm turns the other way
            rots = _rotations(axis_l, th)
            a["rot"] = rots
            a["rot_prev"][0] = rot_prev
            a["rot_prev"][1:] = rots[:-1]
            a["omega"] = f[:, None] * p.omega_lat[None, :]
            theta, rot_prev = float(th[-1]), rots[-1]
        else:
            a["rot"] = np.eye(3)
            a["rot_prev"] = np.eye(3)
        a["sample"] = ((s + 1 > w0) & ((s + 1 - w0) % every == 0)).astype(a["sample"].dtype)
        if not sampling and step + nb > w0:
            lat.reset_samples()
            sampling = True
        h = lat.run(a)
        hist[step:step + nb] = h
        step += nb
        fm = h.mean(axis=0)
        f_model, m_model = (R.T @ fm[:3]) * fscale, (R.T @ fm[3:]) * mscale
        tu = step / unit
        history.append((tu, f_model, m_model))
        if progress is not None:
            el = time.perf_counter() - t_loop
            mets = {}
            if p.spin:
                mets.update(thrust_n=float(f_model @ p.axis_model), torque_nm=float(m_model @ p.axis_model))
            if not p.still:
                mets.update(drag_n=float(f_model @ R[0]), lift_n=float(f_model @ R[2]))
            msg = (f"Solving: {step} of {total} steps ({tu:.1f} {'revolutions' if p.still else 'flow passes'}, "
                   f"{step * p.updates_per_step / max(el, 1e-9) / 1e6:.0f} MLUPs)")
            if progress(0.02 + 0.96 * step / total, msg, mets):
                raise Cancelled("cancelled")
        if not np.isfinite(h).all():
            raise RuntimeError("the flow solution blew up (unstable); try a finer grid or a lower speed")
        if step > w0 + min_win:
            worst, se_rel, trend, half = _window_check(hist[w0:step], p, axis_l)
            if worst < opt.tolerance and se_rel < opt.tolerance:
                converged = True
                break
            # a drifting window drops its first half (surface and slice sums
            # restart), never in the last 30 % of the run
            if worst > 3.0 * opt.tolerance and trend and step - w0 >= min_win and step < 0.7 * total:
                w0 += half
                lat.reset_samples()
    loop_s = time.perf_counter() - t_loop
    mlups = step * p.updates_per_step / loop_s / 1e6
    hist = hist[:step]
    avg = hist[min(w0, len(hist) - 1):].mean(axis=0)
    force, moment = (R.T @ avg[:3]) * fscale, (R.T @ avg[3:]) * mscale
    rho, vel = cfg.air.density, p.dx / p.dt
    drag, lift, side = float(force @ R[0]), float(force @ R[2]), float(force @ R[1])
    speed = float(cfg.speed_m_s)
    q_ref = 0.5 * rho * speed * speed if speed > 0.0 else 0.5 * rho * (om_mag / p.dt * p.rotor_radius) ** 2
    cd = drag / (q_ref * p.frontal_area) if speed > 0.0 and not p.spin and p.frontal_area > 0.0 else None
    thrust = torque = power = None
    if p.spin:
        om = cfg.spin.rpm * 2.0 * math.pi / 60.0
        torque = float(moment @ p.axis_model)
        thrust, power = float(force @ p.axis_model), -torque * om
    if p.spin:  # blade Reynolds number at 75 % radius, the chord from the area of both faces of two blades
        chord = float(m.triangle_areas().sum()) / (4.0 * p.rotor_radius)
        reynolds = (0.75 * om_mag / p.dt * p.rotor_radius + speed) * chord / cfg.air.kinematic_viscosity
    else:
        reynolds = speed * p.d_front / cfg.air.kinematic_viscosity
    pconv = rho * vel * vel / 3.0
    ppa = ((lat.vertex_means().astype(np.float64) - 1.0) * pconv).astype(np.float32)
    cp = (ppa.astype(np.float64) / q_ref).astype(np.float32)
    out_slices = _slice_results(p, lat.slice_means(), slices, unit_m, vel, pconv)
    if not converged:
        warnings.append(f"the forces had not settled to within {opt.tolerance * 100:.1f} % by the end of the run; "
                        "the numbers are averages over its last part")
    if p.blockage > 0.06:
        warnings.append(f"the part fills {p.blockage * 100:.1f} % of the tunnel's cross-section; drag may read a little high")
    tw = _thin_warning(p)
    if tw:
        warnings.append(tw)
    tau0 = 0.5 + 3.0 * p.nu_lat
    wall_re = reynolds if p.spin else speed * p.dx / cfg.air.kinematic_viscosity
    if tau0 < 0.502 and wall_re > 300.0:
        warnings.append(f"the boundary layer is thinner than a cell (cell Reynolds number {wall_re:.0f}): surface friction and "
                        "separation are approximate")
    if thrust is not None:
        headline = (f"Thrust {sig(abs(thrust), 3)} N ({sig(abs(thrust) / 9.80665e-3, 3)} g), torque {sig(abs(torque) * 1e3, 3)} mN·m, "
                    f"{sig(abs(power), 3)} W at {sig(abs(cfg.spin.rpm), 4)} rpm")
    elif cd is not None:
        headline = f"Drag {sig(drag, 3)} N at {sig(speed, 3)} m/s (Cd {sig(cd, 3)})"
    else:
        headline = f"Drag {sig(drag, 3)} N at {sig(speed, 3)} m/s"
    cells = sum(p.multi.cells) if p.multi is not None else int(np.prod(p.dims, dtype=np.int64))
    summ = WindSummary(kind="wind", headline=headline, force_n=force.tolist(), moment_nm=moment.tolist(), drag_n=drag, lift_n=lift, side_n=side,
                       cd=cd, ref_area_mm2=p.frontal_area * 1e6, thrust_n=thrust, torque_nm=torque, power_w=power, reynolds=reynolds,
                       cells=int(cells), steps=int(step), mlups=mlups, seconds=time.perf_counter() - t_start, converged=converged,
                       warnings=warnings, grid=list(p.dims), cells_across=p.cells_across, dx_mm=p.dx * 1e3, dt_s=p.dt,
                       mach_lattice=(p.u_lat + om_mag * p.rotor_radius / p.dx) * math.sqrt(3.0), tau=tau0, blockage=p.blockage,
                       storage={0: "Fp32", 1: "Fp16", 2: "Bf16", 3: "Fp64"}[p.storage], memory_bytes=int(lat.memory_bytes),
                       averaged_over=max(step - w0, 0) / unit, simulated=step / unit, time_unit="revolutions" if p.still else "passes",
                       q_ref_pa=q_ref, thin_mm=0.0 if p.spin else p.d_thin * 1e3, cells_thin=0.0 if p.spin else p.cells_thin())
    return WindResult(summary=summ, surface_pressure_pa=ppa, surface_cp=cp, slices=out_slices, history=history)


def _slice_results(p: Plan, sm: np.ndarray, slices: list, unit_m: float, vel: float, pconv: float) -> list:
    """Slice pixels to SI fields in model coordinates (tunnel.rs:1262-1318)."""
    R = p.r
    out, off = [], 0

    def lat_to_model(x):
        return p.pref + R.T @ ((np.asarray(x, dtype=np.float64) - np.asarray(p.center)) * p.dx)

    for si, (o, u, v, nu, nv) in enumerate(slices):
        n = nu * nv
        px = np.asarray(sm[off:off + n], dtype=np.float64)
        off += n
        su, sv = np.asarray(u, dtype=np.float64), np.asarray(v, dtype=np.float64)
        ua, va = su / np.linalg.norm(su), sv / np.linalg.norm(sv)
        corner = np.asarray(o, dtype=np.float64) - 0.5 * (su + sv)
        uvec = px[:, 1:4]

        def mk(name, label, unit, data):
            d = data.astype(np.float32)
            fin = d[np.isfinite(d)]
            return SliceField(name=name, label=label, unit=unit, min=float(fin.min()) if fin.size else math.inf,
                              max=float(fin.max()) if fin.size else -math.inf, data=d)

        if si == 0:
            name, label = "along", ("Along the spin axis" if p.still else "Along the wind")
            ul = "axial" if p.still else "streamwise"
        else:
            name, label = "across", ("Across the axis, through the rotor" if p.still else "Across the wind, through the part")
            ul = "sideways"
        out.append(FlowSlice(name=name, label=label, origin_mm=(lat_to_model(corner) / unit_m).tolist(),
                             u_mm=((R.T @ su) * nu * p.dx / unit_m).tolist(), v_mm=((R.T @ sv) * nv * p.dx / unit_m).tolist(), nu=int(nu),
                             nv=int(nv), fields=[mk("speed", "Air speed", "m/s", np.linalg.norm(uvec, axis=1) * vel),
                                                 mk("pressure", "Pressure (relative to far field)", "Pa", (px[:, 0] - 1.0) * pconv),
                                                 mk("u", f"In-plane velocity, {ul}", "m/s", (uvec @ ua) * vel),
                                                 mk("v", "In-plane velocity, up", "m/s", (uvec @ va) * vel)]))
    return out


def run(cfg: WindConfig, m: Mesh, unit_m: float, progress=None) -> WindResult:
    return run_with(cfg, m, unit_m, SolverOptions(), progress)


def _finite_range(a: np.ndarray) -> tuple[float, float]:
    f = np.asarray(a, dtype=np.float32)
    f = f[np.isfinite(f)]
    return (0.0, 0.0) if f.size == 0 else (float(f.min()), float(f.max()))


def write_run(r: WindResult, folder) -> None:
    """A wind run's folder as the engine stores it (docs/ARCHITECTURE.md
    "Storage"; crates/engine/src/wind.rs:463-497): surface pressure and Cp
    per mesh vertex as field.pressure.f32 / field.cp.f32 (little-endian f32),
    each slice's header as slice.<name>.json and its fields as
    slice.<name>.<field>.f32 (row-major in v then u), plus run.json (the
    summary and the field and slice lists) and the force history as CSV."""
    d = Path(folder)
    d.mkdir(parents=True, exist_ok=True)
    fields = []
    if np.isfinite(r.surface_pressure_pa).any():
        lo, hi = _finite_range(r.surface_pressure_pa)
        np.asarray(r.surface_pressure_pa, dtype="<f4").tofile(d / "field.pressure.f32")
        m = max(abs(lo), abs(hi))  # symmetric about zero: white is ambient
        fields.append({"name": "pressure", "label": "Air pressure", "unit": "Pa", "min": -m, "max": m, "data_min": lo, "data_max": hi,
                       "scale": "linear", "diverging": True})
    if np.isfinite(r.surface_cp).any():
        lo, hi = _finite_range(r.surface_cp)
        np.asarray(r.surface_cp, dtype="<f4").tofile(d / "field.cp.f32")
        fields.append({"name": "cp", "label": "Pressure coefficient", "unit": "", "min": lo, "max": hi, "scale": "linear", "diverging": True})
    slices = []
    for s in r.slices:
        if not s.fields:
            continue
        hdr = {k: getattr(s, k) for k in ("name", "label", "origin_mm", "u_mm", "v_mm", "nu", "nv")}
        infos = []
        for f in s.fields:
            lo, hi = _finite_range(f.data)
            np.asarray(f.data, dtype="<f4").tofile(d / f"slice.{s.name}.{f.name}.f32")
            infos.append({"name": f.name, "label": f.label, "unit": f.unit, "min": lo, "max": hi})
        hdr["fields"] = infos
        (d / f"slice.{s.name}.json").write_text(json.dumps(hdr))
        slices.append({"name": s.name, "label": s.label})
    with open(d / "history.csv", "w") as fh:
        fh.write("t,fx,fy,fz,mx,my,mz\n")
        for t, fv, mv in r.history:
            fh.write(",".join(repr(float(x)) for x in (t, *fv, *mv)) + "\n")
    run = {"kind": "wind", "summary": asdict(r.summary), "fields": fields, "slices": slices}
    (d / "run.json").write_text(json.dumps(run, indent=2))

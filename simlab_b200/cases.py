"""Frozen workloads (synthetic inputs with the benchmark configurations'
shapes): geometry generators and lattice setups shared by the tests, the
smoke check and the bench.

* `sphere_re40`: 96x48x48, sphere r=6 at (24,24,24), velocity inlet u=0.04,
  open (zero-gradient pressure) outlet, free-slip sides, Re 40 on the
  diameter (nu = 0.012, tau = 0.536), halfway bounce-back, plain BGK.
* `arm_les`: 512x256x256 D3Q19 with the reference's regularized collision
  and Smagorinsky LES (Cs = 0.17), a 200x12x8-cell box beam with a cylinder
  (r = 10, h = 14, axis z) at its +y end centred at (128,128,128), inlet
  u = 0.05, Re = 1e5 on the 12-cell width (nu = 6e-6, tau0 = 0.500018), the
  reference's wind-tunnel faces (velocity inlet holding the total pressure,
  open outlet and sides; tunnel.rs:764-771) with sponges 16/32/16 cells,
  sponge tau 1.0 and absorbing strength 0.1 (tunnel.rs:206-234, 1006-1007).
  `scale=2` gives the 1024x512x512 arm.
* `prop_refined`: D3Q27 cumulant on three nested levels (coarse 256x128x128,
  each finer box 0.63 of its parent per axis, about a quarter of its volume)
  with a 2-blade rotor of radius 60 finest cells spinning on the finest level
  (chord 0.15R -> 0.08R, twist 25 -> 8 degrees, 5 % elliptic section), tip
  speed 0.08, axial inflow 0.02, spin-up over half a revolution.
* `gray_design`: the gray-level adjoint case, 192x96x96 D3Q19 BGK with a
  64x48x48 design box of smoothed random solid fraction, drag averaged over
  steps 500-1000, a checkpoint every 50 steps.
"""
from __future__ import annotations

import numpy as np

from .lbm import Collision, FaceBc, LatticeSetup, Storage, halfway, voxelize_static
from .shapes import arm, sphere


def sphere_re40(storage=Storage.FP32, collision=Collision.BGK, debug_dump=True):
    dims = (96, 48, 48)
    center = (24.0, 24.0, 24.0)
    r, u, re = 6.0, 0.04, 40.0
    v, t = sphere(list(center), r, 5)
    vox = halfway(voxelize_static(v, t, list(dims)))
    F = FaceBc
    st = LatticeSetup(dims=list(dims), faces=[F.VELOCITY, F.OPEN, F.FREE_SLIP, F.FREE_SLIP, F.FREE_SLIP, F.FREE_SLIP], nu=u * 2 * r / re,
                      u_inf=[u, 0.0, 0.0], u_init=[u, 0.0, 0.0], collision=collision, storage=storage, center=list(center),
                      debug_dump=debug_dump)
    return st, vox


def sphere_cd(fx, u=0.04, r=6.0):
    return np.asarray(fx) / (0.5 * u * u * np.pi * r * r)


def arm_les(storage=Storage.FP16, scale: int = 1, debug_dump=False, dims=None):
    dims = tuple(dims) if dims is not None else (512 * scale, 256 * scale, 256 * scale)
    c = (dims[0] / 4.0, dims[1] / 2.0, dims[2] / 2.0)
    v, t = arm(center=c, scale=scale)
    vox = voxelize_static(v, t, list(dims))
    u = 0.05
    nu = u * 12.0 / 1e5
    F = FaceBc
    sp = [16 * scale, 32 * scale] + [16 * scale] * 4
    st = LatticeSetup(dims=list(dims), faces=[F.VELOCITY, F.OPEN, F.OPEN, F.OPEN, F.OPEN, F.OPEN], nu=nu, smagorinsky=0.17,
                      u_inf=[u, 0.0, 0.0], u_init=[u, 0.0, 0.0], sponge=sp, sponge_tau=1.0, sponge_sigma=0.1, absorb_velocity=False,
                      total_pressure_inlet=True, storage=storage, center=list(c), debug_dump=debug_dump,
                      collision=Collision.REGULARIZED)
    return st, vox


def arm_reference_area(scale: int = 1) -> float:
    """Frontal area of the arm seen from +x (beam 200x8 plus the cylinder's 20x14 above/below it is inside)."""
    return float((200 * 8 + 0) * scale * scale)


# algorithmic bytes per lattice update: 19 populations read and written once plus the u32 flag word
BYTES_PER_LUP = {Storage.FP32: 156, Storage.FP16: 80, Storage.BF16: 80, Storage.FP64: 308}


# ------------------------------------------------------------------ gray-level design case
def splitmix64(seed: int, n: int) -> np.ndarray:
    """n uniform doubles in [0, 1) from SplitMix64 (Steele, Lea & Flood 2014),
    the top 53 bits of each output."""
    M = (1 << 64) - 1
    out = np.empty(n, dtype=np.float64)
    s = seed & M
    for k in range(n):
        s = (s + 0x9E3779B97F4A7C15) & M
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z ^= z >> 31
        out[k] = (z >> 11) * (1.0 / (1 << 53))
    return out


def gaussian_smooth(a: np.ndarray, sigma: float = 3.0, radius: int = 9) -> np.ndarray:
    """Separable Gaussian filter with mirrored edges (the edge sample repeated)."""
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    k /= k.sum()
    out = np.asarray(a, dtype=np.float64)
    for ax in range(out.ndim):
        pad = [(0, 0)] * out.ndim
        pad[ax] = (radius, radius)
        p = np.pad(out, pad, mode="symmetric")
        out = np.apply_along_axis(lambda r: np.convolve(r, k, mode="valid"), ax, p)
    return out


def gray_design(storage=Storage.FP32, dims=(192, 96, 96), box_lo=(48, 24, 24), box_n=(64, 48, 48), u=0.04, re=100.0, seed=20240601):
    """The gray-level adjoint case: D3Q19 BGK on 192x96x96, a 64x48x48 design
    box of solid fraction seeded uniform in [0, 1] (SplitMix64, fixed seed) and
    smoothed by a Gaussian of sigma 3 cells (radius 9, mirrored edges); inlet
    u = 0.04, Re = 100 on the box height (nu = u * 48 / 100).  Returns the
    setup, gamma (box order, x fastest) and the adjoint spec of the mean drag
    over steps 500-1000 with a checkpoint every 50 steps."""
    from .gray import AdjointSpec, GraySetup

    nb = int(np.prod(box_n))
    g = splitmix64(seed, nb).reshape(box_n[2], box_n[1], box_n[0])
    g = np.clip(gaussian_smooth(g, 3.0, 9), 0.0, 1.0).reshape(-1)
    nu = u * box_n[1] / re
    center = [box_lo[k] + 0.5 * (box_n[k] - 1) for k in range(3)]
    st = GraySetup(dims=list(dims), box_lo=list(box_lo), box_n=list(box_n), nu=nu, u_in=[u, 0.0, 0.0], alpha=1.0, center=center, storage=storage)
    spec = AdjointSpec(steps=1000, t0=500, t1=1000, checkpoint_every=50, objective=0, dir=[1.0, 0.0, 0.0], recompute=True)
    return st, g, spec


# ------------------------------------------------------------------ refined rotor case
def rotation(axis, theta):
    """Rotation by theta about a unit axis (Rodrigues)."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(theta) * K + (1 - np.cos(theta)) * (K @ K)


# body frame -> lattice: the rotor's spin axis (body z) along the tunnel flow (lattice x)
BODY_TO_LATTICE = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])


def spin_schedule(n, omega, ramp_steps, axis=(1.0, 0.0, 0.0), body=BODY_TO_LATTICE, start=0):
    """StepIn records of a part spinning about the lattice `axis` at `omega`
    rad per finest step, spun up with the smoothstep of tunnel.rs:1085-1098
    over `ramp_steps`: rot is the body->lattice rotation after each step,
    rot_prev the one before, omega the step's angular velocity."""
    from .lbm import steps_array

    a = steps_array(n)
    ax = np.asarray(axis, dtype=np.float64)
    theta = 0.0
    prev = body.copy()
    for s in range(start + n):
        x = (s + 0.5) / ramp_steps if s < ramp_steps else 1.0
        f = x * x * (3.0 - 2.0 * x) if s < ramp_steps else 1.0
        theta += f * omega
        rot = rotation(ax, theta) @ body
        if s >= start:
            k = s - start
            a[k]["rot"] = rot
            a[k]["rot_prev"] = prev
            a[k]["omega"] = ax * (f * omega)
        prev = rot
    return a


def prop_refined(storage=Storage.FP32, radius=60.0, tip_speed=0.08, u=0.02, nu_finest=4e-5, dims0=(256, 128, 128), sponge=True):
    """The refined rotor case: returns (MultiSetup, SpinGeometry, omega).
    The rotor sits at the centre of the finest level (plus sub-cell offsets
    so no symmetry plane falls on a lattice plane), its axis along the flow."""
    from .lbm import SpinGeometry, voxelize_spin
    from .mlattice import LevelBox, MultiSetup
    from .shapes import propeller

    F = FaceBc
    nl = 3
    s = MultiSetup(dims0=list(dims0), faces=[F.VELOCITY] + [F.OPEN] * 5, nu0=nu_finest / 2 ** (nl - 1), u_inf=[u, 0.0, 0.0],
                   u_init=[u, 0.0, 0.0], sponge=[0, 16, 8, 8, 8, 8] if sponge else [0] * 6, sponge_tau=1.0, sponge_sigma=0.1 if sponge else 0.0,
                   total_pressure_inlet=True, storage=storage, debug_dump=False)
    for l in range(1, nl):
        d = s.dims(l - 1)
        n = [int(d[k] * 0.63) for k in range(3)]
        s.boxes.append(LevelBox(lo=[(d[k] - n[k]) // 2 for k in range(3)], n=n))
    fd = s.dims(nl - 1)
    c = [0.5 * (fd[0] - 1) + 0.31, 0.5 * (fd[1] - 1) + 0.23, 0.5 * (fd[2] - 1) + 0.17]
    s.center = c
    v, t = propeller(radius=radius)
    sv = voxelize_spin(v, t, [0.0, 0.0, 1.0], 0.125)
    r = int(np.ceil(sv.radius)) + 3
    ax_lo, ax_hi = int(np.floor(c[0] + sv.axial[0])) - 3, int(np.ceil(c[0] + sv.axial[1])) + 3
    geo = SpinGeometry(vox=sv, box_lo=[ax_lo, int(c[1]) - r, int(c[2]) - r], box_n=[ax_hi - ax_lo + 1, 2 * r + 2, 2 * r + 2])
    return s, geo, tip_speed / radius


# ------------------------------------------------------------------ at-scale adjoint case
def prop_gray_band(storage=Storage.FP16, dims=(384, 192, 192), radius=60.0, band=3.0, u=0.04, nu=0.02, steps=600, checkpoint_every=50):
    """The at-scale adjoint case: the two-blade rotor of the refined case
    (radius 60 cells, axis along the flow) held still on one 384x192x192
    D3Q19 level as a gray body: its cells at solid fraction 1, the fluid cells
    within `band` cells of it design cells at 0.5; the objective is the mean
    torque about the rotor axis over the second half of `steps`, with the
    moments kept where they fit in device memory and the other segments
    recomputed from checkpoints every `checkpoint_every` steps.  Returns the
    setup, gamma (design-box order, x fastest), the band mask in that order
    and the adjoint spec."""
    from .gray import AdjointSpec, GraySetup
    from .lbm import inside_grid
    from .shapes import propeller
    from scipy.ndimage import distance_transform_edt

    c = np.array([0.5 * (dims[0] - 1) - 64.0 + 0.31, 0.5 * (dims[1] - 1) + 0.23, 0.5 * (dims[2] - 1) + 0.17])
    v, t = propeller(radius=radius)
    vl = np.asarray(v, dtype=np.float64) @ BODY_TO_LATTICE.T + c
    m = int(np.ceil(band)) + 2
    lo = np.maximum(np.floor(vl.min(axis=0)).astype(int) - m, 1)
    hi = np.minimum(np.ceil(vl.max(axis=0)).astype(int) + m, np.array(dims) - 2)
    n = hi - lo + 1
    solid = inside_grid(vl, t, lo.astype(float), 1.0, n).reshape(n[2], n[1], n[0])
    dist = distance_transform_edt(~solid)
    near = (~solid) & (dist <= band)
    gam = np.where(solid, 1.0, np.where(near, 0.5, 0.0)).reshape(-1)
    st = GraySetup(dims=list(dims), box_lo=[int(x) for x in lo], box_n=[int(x) for x in n], nu=nu, u_in=[u, 0.0, 0.0], alpha=1.0,
                   center=[float(x) for x in c], storage=storage)
    spec = AdjointSpec(steps=steps, t0=steps // 2 + 1, t1=steps, checkpoint_every=checkpoint_every, objective=1, dir=[1.0, 0.0, 0.0],
                       recompute=False)
    return st, gam, near.reshape(-1), spec


# ------------------------------------------------------------------ spinning-part overhead case
def rotor_tunnel(storage=Storage.FP16, spinning: bool = True, dims=(256, 128, 128), radius=40.0, tip_speed=0.08, u=0.03, nu=4e-4):
    """One D3Q19 level with the refined case's two-blade rotor (radius 40
    cells here), axis along the flow, in the reference's wind-tunnel faces:
    spinning (`Geometry::Spin`: every cell of the swept box a record,
    re-voxelized each step) or held still (`Geometry::Static` of the same
    surface at angle zero).  Returns (setup, geometry, omega)."""
    from .lbm import SpinGeometry, voxelize_spin
    from .shapes import propeller

    c = [0.5 * (dims[0] - 1) - 32.0 + 0.31, 0.5 * (dims[1] - 1) + 0.23, 0.5 * (dims[2] - 1) + 0.17]
    F = FaceBc
    st = LatticeSetup(dims=list(dims), faces=[F.VELOCITY] + [F.OPEN] * 5, nu=nu, u_inf=[u, 0.0, 0.0], u_init=[u, 0.0, 0.0],
                      storage=storage, center=c, collision=Collision.REGULARIZED, total_pressure_inlet=True)
    v, t = propeller(radius=radius)
    if spinning:
        sv = voxelize_spin(v, t, [0.0, 0.0, 1.0], 0.125)
        r = int(np.ceil(sv.radius)) + 3
        lo, hi = int(np.floor(c[0] + sv.axial[0])) - 3, int(np.ceil(c[0] + sv.axial[1])) + 3
        geo = SpinGeometry(vox=sv, box_lo=[lo, int(c[1]) - r, int(c[2]) - r], box_n=[hi - lo + 1, 2 * r + 2, 2 * r + 2])
    else:
        geo = voxelize_static(np.asarray(v, dtype=np.float64) @ BODY_TO_LATTICE.T + np.asarray(c), t, list(dims))
    return st, geo, tip_speed / radius

"""Shared case builders for the tests (reference test setups restated)."""
from __future__ import annotations

import numpy as np

from simlab_b200.lbm import Collision, FaceBc, LatticeSetup, Storage, halfway, voxelize_static
from simlab_b200.shapes import cuboid, merge, sphere


def channel_setup(dims, nu, g, storage=Storage.FP32):
    """crates/cfd/tests/channel.rs:22-37."""
    return LatticeSetup(dims=list(dims), faces=[FaceBc.PERIODIC] * 6, nu=nu, body_force=[g, 0.0, 0.0], storage=storage,
                        center=[0.0, 0.0, 0.0], debug_dump=True)


def channel_case(h: float, umax: float, storage=Storage.FP32):
    """Plane Poiseuille between plates placed off the grid (channel.rs:39-53)."""
    ya = 1.37
    yb = ya + h
    ny = int(np.ceil(yb)) + 2
    nx = nz = 3
    v, t = merge(cuboid([-5.0, -10.0, -5.0], [nx + 5.0, ya, nz + 5.0]), cuboid([-5.0, yb, -5.0], [nx + 5.0, ny + 10.0, nz + 5.0]))
    vox = voxelize_static(v, t, [nx, ny, nz])
    nu = 0.1
    g = umax * 8.0 * nu / (h * h)
    steps = int(3.0 * h * h / nu)
    return channel_setup([nx, ny, nz], nu, g, storage), vox, steps, (ya, yb, nu, g, nx, ny)


def poiseuille_error(mac, hist, params):
    """L2 error against the exact parabola and the force balance (channel.rs:54-74)."""
    ya, yb, nu, g, nx, ny = params
    e2 = r2 = 0.0
    for y in range(ny):
        if y <= ya or y >= yb:
            continue
        exact = g / (2.0 * nu) * (y - ya) * (yb - y)
        c = (1 * ny + y) * nx + 1
        e2 += (float(mac[c, 1]) - exact) ** 2
        r2 += exact * exact
    fluid = float(np.nansum(mac[:, 0].astype(np.float64)))
    bal = (hist[-1, 0] - g * fluid) / (g * fluid)
    return float(np.sqrt(e2 / r2)), float(bal)


def ball(n: int, r: float, lattice: int = 19):
    """crates/cfd/tests/momentum.rs:28-32."""
    c = n / 2.0
    v, t = sphere([c + 0.3, c - 0.6, c + 0.17], r, 5)
    return voxelize_static(v, t, [n, n, n], lattice)


def momentum_setup(n, nu, u0, g, faces, storage=Storage.FP32):
    """crates/cfd/tests/momentum.rs:9-26."""
    return LatticeSetup(dims=[n, n, n], faces=list(faces), nu=nu, u_inf=[u0, 0.0, 0.0], u_init=[u0, 0.0, 0.0], body_force=[g, 0.0, 0.0],
                        storage=storage, center=[n / 2.0] * 3, debug_dump=True)


def sphere_case(storage=Storage.FP32, collision=Collision.BGK, dims=(96, 48, 48), center=(24.0, 24.0, 24.0), r=6.0, u=0.04, re=40.0):
    """The 96x48x48 sphere case: sphere r=6 at (24,24,24), velocity inlet
    u=0.04, open outlet, free-slip sides, Re 40 on the diameter, halfway
    bounce-back, plain BGK."""
    v, t = sphere(list(center), r, 5)
    vox = halfway(voxelize_static(v, t, list(dims)))
    nu = u * 2.0 * r / re
    F = FaceBc
    st = LatticeSetup(dims=list(dims), faces=[F.VELOCITY, F.OPEN, F.FREE_SLIP, F.FREE_SLIP, F.FREE_SLIP, F.FREE_SLIP], nu=nu,
                      u_inf=[u, 0.0, 0.0], u_init=[u, 0.0, 0.0], collision=collision, storage=storage, center=list(center),
                      debug_dump=True)
    return st, vox


def cd_sphere(fx, u=0.04, r=6.0):
    return np.asarray(fx) / (0.5 * u * u * np.pi * r * r)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    m = np.isfinite(a) & np.isfinite(b)
    return float(np.sqrt(np.sum((a[m] - b[m]) ** 2) / np.sum(b[m] ** 2)))

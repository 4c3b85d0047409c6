"""Analytic test geometry as triangle meshes (fixture generators).

`cuboid` and `sphere` follow crates/cfd/src/shapes.rs:8-21 and 47-99 (axis-
aligned box with outward triangles; geodesic sphere from a subdivided
icosahedron).  `arm` builds the quadcopter-arm stand-in of the 512x256x256
LES case: a box beam with a cylinder at one end.  `propeller` builds the
parametric rotor of the refined D3Q27 case (linear chord and twist, elliptic
section, cylindrical hub).
"""
from __future__ import annotations

import math

import numpy as np


def cuboid(lo, hi):
    """Axis-aligned box, outward-facing triangles (shapes.rs:8-21)."""
    lo = [float(v) for v in lo]
    hi = [float(v) for v in hi]
    pts = np.array([[hi[0] if i & 1 else lo[0], hi[1] if i & 2 else lo[1], hi[2] if i & 4 else lo[2]] for i in range(8)])
    quads = [[0, 2, 3, 1], [4, 5, 7, 6], [0, 1, 5, 4], [2, 6, 7, 3], [0, 4, 6, 2], [1, 3, 7, 5]]
    tris = []
    for q in quads:
        tris.append([q[0], q[1], q[2]])
        tris.append([q[0], q[2], q[3]])
    return pts, np.array(tris, dtype=np.uint32)


def sphere(center, radius, subdiv):
    """Geodesic sphere, outward-facing (shapes.rs:47-99): the icosahedron's
    12 vertices and 20 faces, each face split in four per level at edge
    midpoints pushed out to the unit sphere."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1],
         [-t, 0, -1], [-t, 0, 1]]
    f = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
         [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]

    def norm(p):
        n = math.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
        return [p[0] / n, p[1] / n, p[2] / n]

    v = [norm([float(c) for c in p]) for p in v]
    for _ in range(subdiv):
        mid: dict = {}

        def get(a, b):
            k = (min(a, b), max(a, b))
            if k not in mid:
                m = norm([v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]])
                v.append(m)
                mid[k] = len(v) - 1
            return mid[k]

        nf = []
        for a, b, c in f:
            ab, bc, ca = get(a, b), get(b, c), get(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        f = nf
    pts = np.array([[center[0] + radius * p[0], center[1] + radius * p[1], center[2] + radius * p[2]] for p in v])
    return pts, np.array(f, dtype=np.uint32)


def cylinder(center, radius, height, axis=2, n=96):
    """Closed cylinder, outward-facing, axis along `axis` (0, 1 or 2)."""
    verts = []
    tris = []
    a1, a2 = [(1, 2), (2, 0), (0, 1)][axis]
    for side in (-0.5, 0.5):
        for k in range(n):
            ang = 2.0 * math.pi * k / n
            p = [0.0, 0.0, 0.0]
            p[axis] = center[axis] + side * height
            p[a1] = center[a1] + radius * math.cos(ang)
            p[a2] = center[a2] + radius * math.sin(ang)
            verts.append(p)
        c = list(center)
        c[axis] = center[axis] + side * height
        verts.append(c)
    c0, c1 = n, 2 * n + 1
    for k in range(n):
        k1 = (k + 1) % n
        a2_, b2 = k + n + 1, k1 + n + 1
        tris += [[c0, k1, k], [c1, a2_, b2], [k, k1, b2], [k, b2, a2_]]
    return np.array(verts, dtype=np.float64), np.array(tris, dtype=np.uint32)


def merge(*meshes):
    """One surface from several (indices shifted)."""
    vs, ts, off = [], [], 0
    for v, t in meshes:
        vs.append(np.asarray(v, dtype=np.float64))
        ts.append(np.asarray(t, dtype=np.uint32) + off)
        off += len(v)
    return np.concatenate(vs), np.concatenate(ts)


def arm(center=(128.0, 128.0, 128.0), length=200.0, width=12.0, thick=8.0, cyl_r=10.0, cyl_h=14.0, scale=1.0):
    """Quadcopter-arm stand-in: a box beam `length` (y) x `width` (x) x
    `thick` (z) cells centred at `center`, with a cylinder of radius `cyl_r`
    and height `cyl_h` (axis z) centred on the beam's +y end.  Frozen
    orientation: the flow runs along +x, so the beam is broadside to it.
    `scale` multiplies every length (the 1024x512x512 case uses 2)."""
    cx, cy, cz = center
    L, W, T = length * scale, width * scale, thick * scale
    box = cuboid([cx - W / 2 + 0.013, cy - L / 2 + 0.017, cz - T / 2 + 0.011], [cx + W / 2 + 0.013, cy + L / 2 + 0.017, cz + T / 2 + 0.011])
    cyl = cylinder([cx + 0.013, cy + L / 2 + 0.017, cz + 0.011], cyl_r * scale, cyl_h * scale, axis=2)
    return merge(box, cyl)


def blade(radius=60.0, r_root=7.0, chord_root=0.15, chord_tip=0.08, twist_root=25.0, twist_tip=8.0, thick=0.05, nr=48, ns=32):
    """One blade along +x in body coordinates (spin axis z): stations from
    r_root to `radius`, chord falling linearly from chord_root * radius to
    chord_tip * radius, twist (the section's angle to the rotation plane) from
    twist_root to twist_tip degrees, an elliptic section of thickness
    `thick` x chord centred on the mid-chord line; outward-facing, capped
    at both ends.  The blade moves toward +y when the part spins about +z."""
    verts, tris = [], []
    for k in range(nr + 1):
        r = r_root + (radius - r_root) * k / nr
        f = (r - r_root) / (radius - r_root)
        c = (chord_root + (chord_tip - chord_root) * f) * radius
        th = math.radians(twist_root + (twist_tip - twist_root) * f)
        for j in range(ns):
            ph = 2.0 * math.pi * j / ns
            s = 0.5 * c * math.cos(ph)  # chordwise, leading edge at +s
            t = 0.5 * thick * c * math.sin(ph)
            # chord along (0, cos th, -sin th), thickness normal (0, sin th, cos th)
            verts.append([r, s * math.cos(th) + t * math.sin(th), -s * math.sin(th) + t * math.cos(th)])
    for k in range(nr):
        for j in range(ns):
            j1 = (j + 1) % ns
            a, b = k * ns + j, k * ns + j1
            c_, d = (k + 1) * ns + j, (k + 1) * ns + j1
            tris += [[a, b, d], [a, d, c_]]
    c0 = len(verts)
    verts.append([r_root, 0.0, 0.0])
    c1 = len(verts)
    verts.append([radius, 0.0, 0.0])
    for j in range(ns):
        j1 = (j + 1) % ns
        tris.append([c0, j1, j])
        tris.append([c1, nr * ns + j, nr * ns + j1])
    return np.array(verts, dtype=np.float64), np.array(tris, dtype=np.uint32)


def propeller(radius=60.0, blades=2, hub_radius=None, hub_height=None, **kw):
    """A rotor in body coordinates (origin at the centre, spin axis z):
    `blades` copies of `blade` spaced evenly about z and a cylindrical hub.
    Defaults: hub radius 0.12 R and height 0.15 R."""
    hr = 0.12 * radius if hub_radius is None else hub_radius
    hh = 0.15 * radius if hub_height is None else hub_height
    bv, bt = blade(radius=radius, r_root=0.8 * hr, **kw)
    parts = [cylinder([0.0, 0.0, 0.0], hr, hh, axis=2, n=48)]
    for b in range(blades):
        a = 2.0 * math.pi * b / blades
        c, s = math.cos(a), math.sin(a)
        v = bv.copy()
        v[:, 0], v[:, 1] = c * bv[:, 0] - s * bv[:, 1], s * bv[:, 0] + c * bv[:, 1]
        parts.append((v, bt))
    return merge(*parts)

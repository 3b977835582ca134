"""Synthetic triangle meshes for the solver's test and benchmark cases.

The reference builds its specimens with three.js generators, which are not part of
this project; these generators produce meshes of the same kinds (spheres, boxes,
cylinders) plus the benchmark bodies (seeded spherical-harmonic-perturbed ellipsoid,
NACA 0012 wing).  Every function returns (positions float32 [V, 3], indices int32
[T, 3]) in world units.
"""
from __future__ import annotations

import math

import numpy as np

Mesh = tuple[np.ndarray, np.ndarray]


def _finish(pos, idx) -> Mesh:
    return (np.ascontiguousarray(np.asarray(pos, dtype=np.float64).astype(np.float32)),
            np.ascontiguousarray(np.asarray(idx, dtype=np.int32)))


def icosphere_unit(subdivisions: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: icosahedron with edge-midpoint subdivision, projected to |p| = 1.
    20 * 4**subdivisions triangles, float64 vertices."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
         (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdivisions):
        cache: dict[tuple[int, int], int] = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, dtype=np.int32)


def icosphere(radius: float, center=(0.0, 0.0, 0.0), subdivisions: int = 3) -> Mesh:
    p, f = icosphere_unit(subdivisions)
    return _finish(p * radius + np.asarray(center, dtype=np.float64), f)


def uv_sphere(radius: float, width_segments: int, height_segments: int, center=(0.0, 0.0, 0.0)) -> Mesh:
    """Latitude-longitude sphere (poles on the y axis), degenerate pole triangles dropped."""
    u = np.arange(width_segments + 1) / width_segments
    v = np.arange(height_segments + 1) / height_segments
    U, V = np.meshgrid(u, v)
    pos = np.stack([-radius * np.cos(U * 2 * np.pi) * np.sin(V * np.pi),
                    radius * np.cos(V * np.pi) + 0 * U,
                    radius * np.sin(U * 2 * np.pi) * np.sin(V * np.pi)], axis=-1).reshape(-1, 3)
    row = width_segments + 1
    iy, ix = np.meshgrid(np.arange(height_segments), np.arange(width_segments), indexing="ij")
    a = iy * row + ix + 1
    b = iy * row + ix
    c = (iy + 1) * row + ix
    d = (iy + 1) * row + ix + 1
    t1 = np.stack([a, b, d], -1)[1:].reshape(-1, 3)
    t2 = np.stack([b, c, d], -1)[:-1].reshape(-1, 3)
    return _finish(pos + np.asarray(center, dtype=np.float64), np.concatenate([t1, t2]))


def lathe(points: np.ndarray, segments: int, center=(0.0, 0.0, 0.0)) -> Mesh:
    """Surface of revolution of (radius, y) profile points about the y axis."""
    pts = np.asarray(points, dtype=np.float64)
    P = len(pts)
    ang = 2 * np.pi * np.arange(segments + 1) / segments
    pos = np.stack([pts[None, :, 0] * np.sin(ang)[:, None], np.broadcast_to(pts[None, :, 1], (segments + 1, P)),
                    pts[None, :, 0] * np.cos(ang)[:, None]], -1).reshape(-1, 3)
    idx = []
    for i in range(segments):
        for j in range(P - 1):
            a, b = i * P + j, (i + 1) * P + j
            idx += [(a, b, a + 1), (b, b + 1, a + 1)]
    return _finish(pos + np.asarray(center, dtype=np.float64), idx)


def ogive_nose(length: float = 1.0, body: float = 0.4, radius: float = 0.25, axial_steps: int = 60,
               segments: int = 72) -> Mesh:
    """Tangent-ogive nose cone on a body tube, the shape of the reference's 'rocket_nose'
    preset (presets.ts:82-111): the profile revolved about y, turned -90 degrees about z
    so the tip points to -x, and centred on its bounding box."""
    rho = (radius * radius + length * length) / (2 * radius)
    pts = [(max(0.0, math.sqrt(max(0.0, rho * rho - (length - x) ** 2)) + radius - rho), x)
           for x in np.linspace(0, length, axial_steps + 1)]
    pts += [(radius, length + body), (0.0, length + body)]
    pos, idx = lathe(np.array(pts), segments)
    p = pos.astype(np.float64)
    p = np.stack([p[:, 1], -p[:, 0], p[:, 2]], 1)
    p -= (p.max(0) + p.min(0)) / 2
    return p.astype(np.float32), idx


def box(sx: float, sy: float, sz: float, segments: int = 4, center=(0.0, 0.0, 0.0)) -> Mesh:
    """Axis-aligned box with each face split into segments x segments quads, wound
    counter-clockwise seen from outside."""
    pos, idx = [], []
    half = np.array([sx, sy, sz]) * 0.5
    for axis in range(3):
        for sign in (-1.0, 1.0):
            u_ax, v_ax = [a for a in range(3) if a != axis]
            base = len(pos)
            for j in range(segments + 1):
                for i in range(segments + 1):
                    p = np.zeros(3)
                    p[axis] = sign * half[axis]
                    p[u_ax] = -half[u_ax] + 2 * half[u_ax] * i / segments
                    p[v_ax] = -half[v_ax] + 2 * half[v_ax] * j / segments
                    pos.append(p)
            for j in range(segments):
                for i in range(segments):
                    a = base + j * (segments + 1) + i
                    b, c, d = a + 1, a + segments + 2, a + segments + 1
                    # (a, b, c) turns from u to v: outward when e_u x e_v = sign * e_axis
                    outward = (sign > 0) != (axis == 1)
                    idx += [(a, b, c), (a, c, d)] if outward else [(a, c, b), (a, d, c)]
    return _finish(np.array(pos) + np.asarray(center, dtype=np.float64), idx)


def cylinder(radius: float, height: float, radial_segments: int, height_segments: int = 1,
             axis: int = 1, center=(0.0, 0.0, 0.0)) -> Mesh:
    """Closed circular cylinder along `axis` (0 = x, 1 = y, 2 = z)."""
    pos, idx = [], []
    for j in range(height_segments + 1):
        h = -height / 2 + height * j / height_segments
        for i in range(radial_segments):
            t = 2 * math.pi * i / radial_segments
            pos.append((radius * math.cos(t), h, radius * math.sin(t)))
    for j in range(height_segments):
        for i in range(radial_segments):
            a = j * radial_segments + i
            b = j * radial_segments + (i + 1) % radial_segments
            idx += [(a, b + radial_segments, b), (a, a + radial_segments, b + radial_segments)]
    for cap, h in ((0, -height / 2), (height_segments, height / 2)):
        c = len(pos)
        pos.append((0.0, h, 0.0))
        for i in range(radial_segments):
            a = cap * radial_segments + i
            b = cap * radial_segments + (i + 1) % radial_segments
            idx.append((c, b, a) if cap else (c, a, b))
    p = np.array(pos)
    if axis == 0:
        p = p[:, [1, 0, 2]]
    elif axis == 2:
        p = p[:, [0, 2, 1]]
    return _finish(p + np.asarray(center, dtype=np.float64), idx)


def real_sph_harmonics(p: np.ndarray) -> np.ndarray:
    """The 8 real spherical harmonics of degree 1 and 2 (unnormalised) at unit vectors p."""
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    return np.stack([x, y, z, x * y, y * z, 3 * z * z - 1, x * z, x * x - y * y], axis=1)


def perturbed_ellipsoid(semi_axes=(40.0, 16.0, 12.0), amplitude: float = 1.5, seed: int = 0,
                        subdivisions: int = 5, center=(0.0, 0.0, 0.0), scale: float = 1.0) -> Mesh:
    """Ellipsoid (semi-axes in lattice cells) with a seeded radial perturbation made of
    the 8 degree-1/2 real spherical harmonics, normalised to a maximum of `amplitude`
    cells.  subdivisions=5 gives 20480 triangles.  `scale` converts cells to metres."""
    p, f = icosphere_unit(subdivisions)
    coeff = np.random.default_rng(seed).standard_normal(8)
    noise = real_sph_harmonics(p) @ coeff
    noise *= amplitude / np.max(np.abs(noise))
    r = p * np.asarray(semi_axes, dtype=np.float64)
    radial = r / np.linalg.norm(r, axis=1, keepdims=True)
    r = r + noise[:, None] * radial
    return _finish(r * scale + np.asarray(center, dtype=np.float64), f)


def naca0012_profile(n: int) -> np.ndarray:
    """Closed-trailing-edge NACA 0012 section, unit chord, LE at x = 0.  Cosine spacing;
    returns the 2n-2 perimeter points counter-clockwise from the trailing edge."""
    beta = np.linspace(0.0, math.pi, n)
    x = 0.5 * (1.0 - np.cos(beta))
    t = 0.12
    yt = 5 * t * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)
    upper = np.stack([x[::-1], yt[::-1]], axis=1)          # TE -> LE along the upper side
    lower = np.stack([x[1:-1], -yt[1:-1]], axis=1)         # LE -> TE along the lower side
    return np.concatenate([upper, lower], axis=0)


def naca0012_wing(chord: float, span: float, aoa_deg: float, center=(0.0, 0.0, 0.0),
                  n_chord: int = 64, n_span: int = 16) -> Mesh:
    """Extruded NACA 0012 wing along z, rotated by the angle of attack about z around the
    quarter chord (trailing edge down for positive angles), centred on `center`."""
    prof = naca0012_profile(n_chord) * chord
    prof[:, 0] -= 0.25 * chord
    a = math.radians(aoa_deg)
    rot = np.array([[math.cos(a), math.sin(a)], [-math.sin(a), math.cos(a)]])
    prof = prof @ rot.T
    P = len(prof)
    pos, idx = [], []
    for j in range(n_span + 1):
        z = -span / 2 + span * j / n_span
        for x, y in prof:
            pos.append((x, y, z))
    for j in range(n_span):
        for i in range(P):
            a0, a1 = j * P + i, j * P + (i + 1) % P
            b0, b1 = a0 + P, a1 + P
            idx += [(a0, a1, b1), (a0, b1, b0)]
    for cap, z in ((0, -span / 2), (n_span, span / 2)):
        c = len(pos)
        cx, cy = prof.mean(axis=0)
        pos.append((cx, cy, z))
        for i in range(P):
            a0, a1 = cap * P + i, cap * P + (i + 1) % P
            idx.append((c, a0, a1) if cap else (c, a1, a0))
    return _finish(np.array(pos) + np.asarray(center, dtype=np.float64), idx)


def lattice_center(nx: int, ny: int, nz: int, h: float, cell=(0.0, 0.0, 0.0)) -> tuple[float, float, float]:
    """World coordinates of the centre of lattice cell `cell` (fractional allowed) for the
    voxelizer's lattice, which is centred on the world origin (voxelizer.ts:107-109)."""
    return tuple(-n * h * 0.5 + (c + 0.5) * h for n, c in zip((nx, ny, nz), cell))


def as_soup(mesh: Mesh) -> np.ndarray:
    """Non-indexed triangle soup float32 [T*3, 3] (BufferGeometry.toNonIndexed)."""
    pos, idx = mesh
    return np.ascontiguousarray(pos[idx.reshape(-1)])

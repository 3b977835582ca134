"""Python restatement of the reference's STL reader and mesh statistics
(src/geometry/stlLoader.ts) -- TEST INFRASTRUCTURE ONLY.

The tests compare libaerosim's aerosim_parse_stl / aerosim_normalize_and_center /
aerosim_compute_mesh_stats with these functions bit for bit.  The ASCII reader runs
the reference's own vertex regular expression (stlLoader.ts:79) through Python's `re`,
with JavaScript's `\\s` and `\\d` spelled out as character classes, so it is an
independent check of the library's hand-written matcher.  The three.js 0.170.0 pieces
that decide the numbers (Vector3.applyMatrix4, Box3, BufferGeometry.translate/scale,
Quaternion.setFromEuler 'XYZ', Matrix4.compose) are restated from that library's
published source; it is not part of the reference tree.  The frontal area comes from
the C oracle's computeProjectedFrontalArea restatement.

Parity pins: the reference's known answers (src/validation/phase1.test.ts:38-97: cube
watertight with volume 1 and A_ref 1, the ASCII right tetrahedron with 4 triangles,
volume 1/6 and A_ref 0.5) are re-run in tests/test_mesh_stats.py.
"""
from __future__ import annotations

import math
import re
import struct

import numpy as np

# JavaScript's \s: WhiteSpace and LineTerminator code points.
_JS_SPACE = "[\t\n\v\f\r \u00a0\u1680\u2000-\u200a\u2028\u2029\u202f\u205f\u3000\ufeff]"
_NUM = r"([+-]?[0-9]*\.?[0-9]+(?:[eE][+-]?[0-9]+)?)"
# stlLoader.ts:79
VERTEX_RE = re.compile(rf"vertex{_JS_SPACE}+{_NUM}{_JS_SPACE}+{_NUM}{_JS_SPACE}+{_NUM}")


class STLFormatError(ValueError):
    pass


def _ascii(text: str) -> np.ndarray:
    """parseAsciiSTL, stlLoader.ts:77-95."""
    vals = []
    for m in VERTEX_RE.finditer(text):
        vals.extend(float(g) for g in m.groups())
    if len(vals) < 9 or len(vals) % 9 != 0:
        raise STLFormatError("ASCII STL file contains no valid triangles.")
    with np.errstate(over="ignore"):  # out-of-range values become +-Infinity, as in a Float32Array
        return np.asarray(vals, dtype=np.float64).astype(np.float32).reshape(-1, 3)


def _binary(buf: bytes, faces: int) -> np.ndarray:
    """parseBinarySTL, stlLoader.ts:40-75 (positions only)."""
    out = np.empty((faces * 3, 3), dtype=np.float32)
    for i in range(faces):
        v = struct.unpack_from("<9f", buf, 84 + 50 * i + 12)
        out[i * 3:i * 3 + 3] = np.asarray(v, dtype=np.float32).reshape(3, 3)
    return out


def _decode(b: bytes) -> str:
    text = b.decode("utf-8", errors="replace")
    return text[1:] if text.startswith("\ufeff") else text  # TextDecoder drops the BOM


def parse_stl(buf: bytes) -> tuple[np.ndarray, str]:
    """parseSTL, stlLoader.ts:9-38: (positions float32 [V, 3], "binary" | "ascii")."""
    n = len(buf)
    if n < 84:
        return _ascii(_decode(buf)), "ascii"
    faces = struct.unpack_from("<I", buf, 80)[0]
    expected = 84 + faces * 50
    if expected == n:
        return _binary(buf, faces), "binary"
    header = _decode(buf[:min(256, n)])
    if re.sub(f"^{_JS_SPACE}+", "", header).lower().startswith("solid"):
        full = _decode(buf)
        if "facet" in full and "vertex" in full:
            return _ascii(full), "ascii"
    if expected <= n and faces > 0:
        return _binary(buf, faces), "binary"
    raise STLFormatError("Invalid or corrupted STL file.")


def _apply(e, x, y, z):
    """Vector3.applyMatrix4 on float64 arrays (element order as three.js evaluates it)."""
    w = 1.0 / (e[3] * x + e[7] * y + e[11] * z + e[15])
    return ((e[0] * x + e[4] * y + e[8] * z + e[12]) * w,
            (e[1] * x + e[5] * y + e[9] * z + e[13]) * w,
            (e[2] * x + e[6] * y + e[10] * z + e[14]) * w)


def _apply_f32(e, pos: np.ndarray) -> np.ndarray:
    p = pos.astype(np.float64)
    x, y, z = _apply(e, p[:, 0], p[:, 1], p[:, 2])
    return np.stack([x, y, z], axis=1).astype(np.float32)


def normalize_and_center(pos: np.ndarray) -> tuple[np.ndarray, bool]:
    """normalizeAndCenterGeometry, stlLoader.ts:101-127."""
    pos = np.asarray(pos, dtype=np.float32).reshape(-1, 3)
    if pos.shape[0] == 0:
        return pos.copy(), False
    p = pos.astype(np.float64)
    c = (p.min(axis=0) + p.max(axis=0)) * 0.5
    t = [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, -c[0], -c[1], -c[2], 1.0]
    pos = _apply_f32(t, pos)
    # translate() recomputes the geometry's Box3 in place: the size is the centred box's
    q = pos.astype(np.float64)
    size = q.max(axis=0) - q.min(axis=0)
    max_dim = max(size[0], size[1], size[2])
    if max_dim > 10.0:
        s = 0.001 if max_dim > 50 else 1.0 / max_dim
        pos = _apply_f32([s, 0, 0, 0, 0, s, 0, 0, 0, 0, s, 0, 0, 0, 0, 1.0], pos)
        return pos, True
    return pos, False


def model_matrix(position, rotation_deg, scale) -> list[float]:
    """Matrix4.compose(position, Quaternion.setFromEuler(XYZ), scale) as computeMeshStats
    builds it (stlLoader.ts:142-153); column-major."""
    d2r = math.pi / 180.0
    rx, ry, rz = (a * d2r for a in rotation_deg)
    c1, c2, c3 = math.cos(rx / 2), math.cos(ry / 2), math.cos(rz / 2)
    s1, s2, s3 = math.sin(rx / 2), math.sin(ry / 2), math.sin(rz / 2)
    qx = s1 * c2 * c3 + c1 * s2 * s3
    qy = c1 * s2 * c3 - s1 * c2 * s3
    qz = c1 * c2 * s3 + s1 * s2 * c3
    qw = c1 * c2 * c3 - s1 * s2 * s3
    x2, y2, z2 = qx + qx, qy + qy, qz + qz
    xx, xy, xz = qx * x2, qx * y2, qx * z2
    yy, yz, zz = qy * y2, qy * z2, qz * z2
    wx, wy, wz = qw * x2, qw * y2, qw * z2
    sx, sy, sz = scale
    return [(1 - (yy + zz)) * sx, (xy + wz) * sx, (xz - wy) * sx, 0.0,
            (xy - wz) * sy, (1 - (xx + zz)) * sy, (yz + wx) * sy, 0.0,
            (xz + wy) * sz, (yz - wx) * sz, (1 - (xx + yy)) * sz, 0.0,
            float(position[0]), float(position[1]), float(position[2]), 1.0]


def _js_round(v: float) -> float:
    r = math.floor(v)
    if v - r >= 0.5:
        r += 1
    return float(r) + 0.0


def mesh_stats(pos, idx, position=(0, 0, 0), rotation_deg=(0, 0, 0), scale=(1, 1, 1), res: int = 512) -> dict:
    """computeMeshStats, stlLoader.ts:133-244 (MeshStats without the name)."""
    from . import frontal_area
    pos = np.asarray(pos, dtype=np.float32).reshape(-1, 3)
    flat = None if idx is None else np.asarray(idx, dtype=np.int64).reshape(-1)
    T = (flat.size if flat is not None else pos.shape[0]) // 3
    m = model_matrix(position, rotation_deg, scale)
    P = pos.astype(np.float64).tolist()
    mn = [math.inf] * 3
    mx = [-math.inf] * 3
    s6 = 0.0
    edges: dict = {}
    keyed = T <= 100000

    def key(v):
        return tuple(_js_round(c * 1e5) for c in v)

    def add(a, b):
        if a == b:
            return
        k = (a, b) if a < b else (b, a)
        edges[k] = edges.get(k, 0) + 1

    for t in range(T):
        ii = [int(flat[t * 3 + k]) if flat is not None else t * 3 + k for k in range(3)]
        v = [P[i] for i in ii]
        if keyed:
            k0, k1, k2 = key(v[0]), key(v[1]), key(v[2])
            add(k0, k1)
            add(k1, k2)
            add(k2, k0)
        w = [_apply(m, *vi) for vi in v]
        for p in w:
            for c in range(3):
                mn[c] = min(mn[c], p[c])
                mx[c] = max(mx[c], p[c])
        (x0, y0, z0), (x1, y1, z1), (x2, y2, z2) = w
        s6 += x0 * (y1 * z2 - z1 * y2) + y0 * (z1 * x2 - x1 * z2) + z0 * (x1 * y2 - y1 * x2)
    open_edges = sum(1 for c in edges.values() if c != 2)
    size = [max(0.0, mx[c] - mn[c]) for c in range(3)]
    world = np.asarray(m, dtype=np.float64)
    return {"triangleCount": T, "vertexCount": pos.shape[0], "isWatertight": open_edges == 0 and T > 0,
            "openEdgeCount": open_edges, "boundingBoxSize": {"x": size[0], "y": size[1], "z": size[2]},
            "characteristicLength": max(1e-4, size[0]),
            "frontalArea": frontal_area((pos, None if flat is None else flat.astype(np.int32)), world, res),
            "volume": abs(s6) / 6.0}

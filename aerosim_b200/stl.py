"""STL reader, millimetre auto-scale and mesh statistics (src/geometry/stlLoader.ts)
over libaerosim.so.  computeMeshStats' frontal area (A_ref) is rasterised on the GPU
(aerosim_frontal_area_cuda) unless `device` is negative.

Geometries are (positions float32 [V, 3], indices int32 or None), the form every
other entry point of this package takes; a transform is the reference's
ModelTransform ({"position": {x, y, z}, "rotationDeg": {x, y, z}, "scale": {x, y, z}})
or a (position, rotation_deg, scale) triple of 3-sequences.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .engine import _geometry, _matrix


def _vec(v) -> list[float]:
    if isinstance(v, dict):
        return [float(v["x"]), float(v["y"]), float(v["z"])]
    return [float(c) for c in v]


def _transform(t) -> N.ModelTransform:
    if t is None:
        t = ((0, 0, 0), (0, 0, 0), (1, 1, 1))
    if isinstance(t, dict):
        p, r, s = t.get("position", (0, 0, 0)), t.get("rotationDeg", (0, 0, 0)), t.get("scale", (1, 1, 1))
    else:
        p, r, s = t
    out = N.ModelTransform()
    for name, v in (("position", p), ("rotation_deg", r), ("scale", s)):
        getattr(out, name)[:] = _vec(v)
    return out


def parse_stl(buffer: bytes | bytearray | memoryview) -> tuple[np.ndarray, None]:
    """parseSTL(buffer), stlLoader.ts:9-38: binary when the size is 84 + 50 x facets,
    ASCII when the text starts with "solid" and names facets and vertices, binary when
    the facets fit; raises AerosimError (code ERR_FORMAT) with the reference's message
    otherwise."""
    raw = np.frombuffer(bytes(buffer), dtype=np.uint8)
    lib = N.load()
    n = C.c_int64()
    fmt = C.c_int32()
    src = N.ptr(raw, C.c_uint8) if raw.size else None
    N.check(lib.aerosim_parse_stl(src, raw.size, None, 0, C.byref(n), C.byref(fmt)))
    pos = np.empty((n.value, 3), dtype=np.float32)
    N.check(lib.aerosim_parse_stl(src, raw.size, N.ptr(pos, C.c_float), n.value, C.byref(n), C.byref(fmt)))
    return pos, None


def stl_format(buffer) -> str:
    """"binary" or "ascii": the branch parseSTL takes for this buffer."""
    raw = np.frombuffer(bytes(buffer), dtype=np.uint8)
    n, fmt = C.c_int64(), C.c_int32()
    N.check(N.load().aerosim_parse_stl(N.ptr(raw, C.c_uint8) if raw.size else None, raw.size, None, 0,
                                       C.byref(n), C.byref(fmt)))
    return "binary" if fmt.value == N.STL_BINARY else "ascii"


def normalize_and_center_geometry(geometry) -> tuple[tuple[np.ndarray, np.ndarray | None], bool]:
    """normalizeAndCenterGeometry(geometry), stlLoader.ts:101-127: a centred copy, and
    whether it was scaled (by 0.001 above 50 units, to unit size above 10)."""
    pos, idx = _geometry(geometry)
    pos = pos.copy()
    flag = C.c_int32()
    N.check(N.load().aerosim_normalize_and_center(N.ptr(pos, C.c_float), pos.shape[0], C.byref(flag)))
    return (pos, idx), bool(flag.value)


def model_matrix(transform) -> np.ndarray:
    """World matrix of a ModelTransform (Matrix4.compose with XYZ Euler degrees,
    stlLoader.ts:142-153), column-major float64 [16]."""
    t = _transform(transform)
    m = np.empty(16, dtype=np.float64)
    N.check(N.load().aerosim_model_matrix(C.byref(t), N.ptr(m, C.c_double)))
    return m


def frontal_area_cuda(geometry, world_matrix=None, grid_resolution: int = 512, device: int = 0) -> float:
    """computeProjectedFrontalArea on the GPU; equal bit for bit to frontal_area()."""
    pos, idx = _geometry(geometry)
    m = _matrix(world_matrix)
    out = C.c_double()
    N.check(N.load().aerosim_frontal_area_cuda(int(device), N.ptr(pos, C.c_float), pos.shape[0],
                                               N.ptr(idx, C.c_int32), 0 if idx is None else idx.size,
                                               N.ptr(m, C.c_double), int(grid_resolution), C.byref(out)))
    return out.value


def compute_mesh_stats(geometry, name: str = "", transform=None, device: int = 0) -> dict:
    """computeMeshStats(geometry, name, transform), stlLoader.ts:133-244, as the
    reference's MeshStats dictionary."""
    pos, idx = _geometry(geometry)
    t = _transform(transform)
    s = N.MeshStats()
    N.check(N.load().aerosim_compute_mesh_stats(N.ptr(pos, C.c_float), pos.shape[0], N.ptr(idx, C.c_int32),
                                                0 if idx is None else idx.size, C.byref(t), int(device),
                                                C.byref(s)))
    b = s.bounding_box_size
    return {"name": name, "triangleCount": s.triangle_count, "vertexCount": s.vertex_count,
            "isWatertight": bool(s.is_watertight), "openEdgeCount": s.open_edge_count,
            "boundingBoxSize": {"x": b[0], "y": b[1], "z": b[2]},
            "characteristicLength": s.characteristic_length, "frontalArea": s.frontal_area, "volume": s.volume}


parseSTL = parse_stl
normalizeAndCenterGeometry = normalize_and_center_geometry
computeMeshStats = compute_mesh_stats

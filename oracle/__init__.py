"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, the smoke check and the benchmark's CPU-baseline leg as the checker
and the timed CPU restatement of the reference's TypeScript CPU path.  The product
(aerosim_b200/) never imports it.

Parity pinning: the reference cannot be executed here (no JavaScript runtime), so
the oracle is pinned by the reference's own known-answer tests, re-run in
tests/test_oracle_known_answers.py.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_P = C.c_void_p
_F32P = C.POINTER(C.c_float)
_F64P = C.POINTER(C.c_double)
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
_U8P = C.POINTER(C.c_uint8)

_SIG = {
    "orc_bvh_create": ([_F32P, C.c_int64, _I32P, C.c_int64, _F64P], _P),
    "orc_bvh_free": ([_P], None),
    "orc_bvh_bounds": ([_P, _F64P], None),
    "orc_bvh_nodes": ([_P, _F64P, _I32P, _I32P, _I32P], C.c_int),
    "orc_bvh_intersect_segment": ([_P] + [C.c_double] * 7, C.c_double),
    "orc_bvh_is_point_inside": ([_P, C.c_double, C.c_double, C.c_double], C.c_int),
    "orc_bvh_scanline": ([_P, C.c_double, C.c_double, _F64P, C.c_int], C.c_int),
    "orc_voxelize": ([_F32P, C.c_int64, _I32P, C.c_int64, _F64P, C.c_double, C.c_int, C.c_int, C.c_int], _P),
    "orc_voxel_free": ([_P], None),
    "orc_voxel_info": ([_P, _I64P, _F64P, _I32P], None),
    "orc_voxel_get": ([_P, _U8P, _I32P, _I32P, _F32P, _F32P], None),
    "orc_solver_create": ([C.c_int, C.c_int, C.c_int, _U8P, _I32P, _F32P, C.c_int64, C.c_double,
                           C.c_double, C.c_double, C.c_int], _P),
    "orc_solver_free": ([_P], None),
    "orc_solver_set_params": ([_P, C.c_double, C.c_double, C.c_double, C.c_int], None),
    "orc_solver_reset": ([_P], None),
    "orc_solver_step": ([_P, C.c_int, C.c_int], None),
    "orc_solver_step_index": ([_P], C.c_int64),
    "orc_solver_rescale_count": ([_P], C.c_int64),
    "orc_solver_get_f": ([_P, _F32P, C.c_int], None),
    "orc_solver_set_f": ([_P, _F32P], None),
    "orc_solver_get_macro": ([_P, _F32P, _F32P, _F32P, _F32P], None),
    "orc_solver_mass_stats": ([_P, _F64P], None),
    "orc_momentum_exchange": ([C.c_int, C.c_int, C.c_int, _U8P, _I32P, _F32P, C.c_int64, _F32P, _F64P], None),
    "orc_force_coefficients": ([C.c_double] * 9 + [_F64P], None),
    "orc_frontal_area": ([_F32P, C.c_int64, _I32P, C.c_int64, _F64P, C.c_int], C.c_double),
    "orc_surface_area": ([_F32P, C.c_int64, _I32P, C.c_int64, _F64P], C.c_double),
    "orc_max_threads": ([], C.c_int),
}

_lib = None


def build() -> str:
    """Compiles the oracle with its Makefile (g++ -O2 -ffp-contract=off -fopenmp)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for k, (a, r) in _SIG.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = r
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _geom(mesh):
    pos, idx = mesh
    pos = np.ascontiguousarray(np.asarray(pos, np.float32).reshape(-1, 3))
    idx = None if idx is None else np.ascontiguousarray(np.asarray(idx, np.int32).reshape(-1))
    return pos, idx


def _mat(m):
    return None if m is None else np.ascontiguousarray(np.asarray(m, np.float64).reshape(16))


class BVH:
    """MeshBVH (bvh.ts)."""

    def __init__(self, mesh, world=None):
        pos, idx = _geom(mesh)
        m = _mat(world)
        self._keep = (pos, idx, m)
        self.h = lib().orc_bvh_create(_p(pos, C.c_float), pos.shape[0], _p(idx, C.c_int32),
                                      0 if idx is None else idx.size, _p(m, C.c_double))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_bvh_free(self.h)

    def bounds(self):
        b = np.empty(6)
        lib().orc_bvh_bounds(self.h, _p(b, C.c_double))
        return b[:3], b[3:]

    def intersect_segment(self, ox, oy, oz, dx, dy, dz, max_t=1.0):
        return lib().orc_bvh_intersect_segment(self.h, ox, oy, oz, dx, dy, dz, max_t)

    def is_point_inside(self, x, y, z) -> bool:
        return bool(lib().orc_bvh_is_point_inside(self.h, x, y, z))

    def scanline(self, y, z):
        buf = np.empty(1024)
        n = lib().orc_bvh_scanline(self.h, y, z, _p(buf, C.c_double), 1024)
        return buf[:min(n, 1024)].copy()


@dataclass
class Voxel:
    nx: int
    ny: int
    nz: int
    dx: float
    origin: tuple
    flags: np.ndarray
    bmap: np.ndarray
    bcells: np.ndarray
    q: np.ndarray
    minq: np.ndarray
    solid: int
    window: tuple
    ms: float

    @property
    def boundary_count(self) -> int:
        return int(self.bcells.size)


def voxelize(mesh, world, tunnel_height: float, nx: int, ny: int, nz: int) -> Voxel:
    """voxelizeMeshToLattice (voxelizer.ts:86-281)."""
    pos, idx = _geom(mesh)
    m = _mat(world)
    L = lib()
    h = L.orc_voxelize(_p(pos, C.c_float), pos.shape[0], _p(idx, C.c_int32), 0 if idx is None else idx.size,
                       _p(m, C.c_double), float(tunnel_height), nx, ny, nz)
    try:
        counts = np.empty(2, np.int64)
        geom = np.empty(5)
        win = np.empty(6, np.int32)
        L.orc_voxel_info(h, _p(counts, C.c_int64), _p(geom, C.c_double), _p(win, C.c_int32))
        n = nx * ny * nz
        b = int(counts[1])
        flags = np.empty(n, np.uint8)
        bmap = np.empty(n, np.int32)
        bcells = np.empty(b, np.int32)
        q = np.empty(b * 18, np.float32)
        minq = np.empty(b, np.float32)
        L.orc_voxel_get(h, _p(flags, C.c_uint8), _p(bmap, C.c_int32), _p(bcells, C.c_int32),
                        _p(q, C.c_float), _p(minq, C.c_float))
        return Voxel(nx, ny, nz, float(geom[0]), (float(geom[1]), float(geom[2]), float(geom[3])), flags,
                     bmap, bcells, q, minq, int(counts[0]), tuple(int(v) for v in win), float(geom[4]))
    finally:
        L.orc_voxel_free(h)


class Solver:
    """LBMCpuReferenceSolver (lbmCpuReference.ts:55-495)."""

    def __init__(self, vox: Voxel, u_inlet=0.08, nu=0.0005, cs=0.12, ground_no_slip=False):
        self.nx, self.ny, self.nz = vox.nx, vox.ny, vox.nz
        self.N = vox.nx * vox.ny * vox.nz
        self.vox = vox
        self.h = lib().orc_solver_create(vox.nx, vox.ny, vox.nz, _p(vox.flags, C.c_uint8),
                                         _p(vox.bmap, C.c_int32), _p(vox.q, C.c_float), vox.boundary_count,
                                         u_inlet, nu, cs, 1 if ground_no_slip else 0)
        self.params = [u_inlet, nu, cs, ground_no_slip]

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_solver_free(self.h)

    def set_params(self, u_inlet=None, nu=None, cs=None, ground_no_slip=None):
        p = self.params
        for i, v in enumerate((u_inlet, nu, cs, ground_no_slip)):
            if v is not None:
                p[i] = v
        lib().orc_solver_set_params(self.h, p[0], p[1], p[2], 1 if p[3] else 0)

    def reset(self):
        lib().orc_solver_reset(self.h)

    def step(self, n=1, threads=1):
        lib().orc_solver_step(self.h, int(n), int(threads))

    @property
    def step_index(self) -> int:
        return int(lib().orc_solver_step_index(self.h))

    @property
    def rescale_count(self) -> int:
        return int(lib().orc_solver_rescale_count(self.h))

    def f(self, which=0) -> np.ndarray:
        """which=0: fSrc (latest populations after the swap), 1: fDst."""
        out = np.empty(19 * self.N, np.float32)
        lib().orc_solver_get_f(self.h, _p(out, C.c_float), which)
        return out

    def set_f(self, f: np.ndarray):
        f = np.ascontiguousarray(f, np.float32)
        lib().orc_solver_set_f(self.h, _p(f, C.c_float))

    def macro(self):
        ux, uy, uz, rho = (np.empty(self.N, np.float32) for _ in range(4))
        lib().orc_solver_get_macro(self.h, _p(ux, C.c_float), _p(uy, C.c_float), _p(uz, C.c_float),
                                   _p(rho, C.c_float))
        return {"ux": ux, "uy": uy, "uz": uz, "rho": rho}

    def mass_stats(self):
        o = np.empty(4)
        lib().orc_solver_mass_stats(self.h, _p(o, C.c_double))
        return {"totalMass": o[0], "meanRho": o[1], "maxSpeed": o[2], "hasNaN": bool(o[3])}


def colormap(t: float) -> tuple[float, float, float]:
    """sampleCFDColormap (lbmCpuReference.ts:23-46)."""
    o = np.empty(3)
    lib().orc_colormap(C.c_double(t), _p(o, C.c_double))
    return float(o[0]), float(o[1]), float(o[2])


def extract_slice(solver: "Solver", axis: str, fraction: float, mode: str) -> np.ndarray:
    """extractSliceRGBA (lbmCpuReference.ts:499-596): uint8 [height][width][4]."""
    a = {"x": 0, "y": 1, "z": 2}[axis]
    m = {"velocity": 0, "vorticity": 1, "pressure": 2}[mode]
    w, h = C.c_int(), C.c_int()
    lib().orc_extract_slice(solver.h, a, C.c_double(fraction), m, None, C.byref(w), C.byref(h))
    out = np.zeros((h.value, w.value, 4), np.uint8)
    lib().orc_extract_slice(solver.h, a, C.c_double(fraction), m, out.ctypes.data_as(C.POINTER(C.c_uint8)),
                            C.byref(w), C.byref(h))
    return out


def q_criterion(nx, ny, nz, dx, ux, uy, uz, flags=None) -> dict:
    """computeQCriterion (vortexIso.ts:22-122)."""
    n = nx * ny * nz
    ux, uy, uz = (np.ascontiguousarray(a, np.float32) for a in (ux, uy, uz))
    fl = None if flags is None else np.ascontiguousarray(flags, np.uint8)
    q, om, omv = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(3 * n, np.float32)
    mq, mo = C.c_double(), C.c_double()
    lib().orc_q_criterion(nx, ny, nz, C.c_double(dx), _p(ux, C.c_float), _p(uy, C.c_float), _p(uz, C.c_float),
                          None if fl is None else fl.ctypes.data_as(C.POINTER(C.c_uint8)), _p(q, C.c_float),
                          _p(om, C.c_float), _p(omv, C.c_float), C.byref(mq), C.byref(mo))
    return {"qValues": q, "omegaMag": om, "omegaVec": omv, "maxQ": mq.value, "maxOmega": mo.value}


def momentum_exchange(vox: Voxel, f: np.ndarray) -> dict:
    """integrateLatticeMomentumExchange raw sums (forceIntegrator.ts:159-216)."""
    o = np.empty(7)
    f = np.ascontiguousarray(f, np.float32)
    lib().orc_momentum_exchange(vox.nx, vox.ny, vox.nz, _p(vox.flags, C.c_uint8), _p(vox.bcells, C.c_int32),
                                _p(vox.q, C.c_float), vox.boundary_count, _p(f, C.c_float), _p(o, C.c_double))
    return {"fx": o[0], "fy": o[1], "fz": o[2], "mx": o[3], "my": o[4], "mz": o[5], "cut": int(o[6])}


def force_coefficients(fx, fy, mz, dx, u_inlet, frontal_area, char_len, tunnel_w, tunnel_h) -> dict:
    o = np.empty(5)
    lib().orc_force_coefficients(fx, fy, mz, dx, u_inlet, frontal_area, char_len, tunnel_w, tunnel_h,
                                 _p(o, C.c_double))
    return {"cdRaw": o[0], "cd": o[1], "cl": o[2], "cm": o[3], "xcp": o[4]}


def frontal_area(mesh, world=None, res=512) -> float:
    pos, idx = _geom(mesh)
    m = _mat(world)
    return float(lib().orc_frontal_area(_p(pos, C.c_float), pos.shape[0], _p(idx, C.c_int32),
                                        0 if idx is None else idx.size, _p(m, C.c_double), res))


def surface_area(mesh, world=None) -> float:
    pos, idx = _geom(mesh)
    m = _mat(world)
    return float(lib().orc_surface_area(_p(pos, C.c_float), pos.shape[0], _p(idx, C.c_int32),
                                        0 if idx is None else idx.size, _p(m, C.c_double)))


def max_threads() -> int:
    return int(lib().orc_max_threads())

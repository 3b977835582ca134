"""Host mirror of the reference's solver interface over libaerosim.so.

  voxelize_mesh_to_lattice(geometry, world_matrix, tunnel, grid) -> VoxelGridResult
      src/geometry/voxelizer.ts:86-281 (runs on the GPU)
  LBMEngine(device)                                         src/solver/lbmEngine.ts:39
      .set_voxel_grid(voxel, config, reset_flow=True)       :142-287
      .update_config(config)                                :289-300
      .step_and_extract_slice(substeps=4, read_macro_field) :404-675 (forces, macro field)
      .reset_flow()                                         :677-688
      .get_step_count()                                     :690
The reference's camelCase names are available as aliases.  Geometry is a
(positions float32 [V, 3], indices int32 [T, 3] or None) pair, the world matrix a
column-major 16-element sequence (THREE.Matrix4.elements) or None, the tunnel a
mapping with length / width / height, the grid a mapping with nx / ny / nz.

Every method raises AerosimError on a library error; step_and_extract_slice returns
None when no voxel grid is set, like the reference.  The slice RGBA image of the
reference's viewport is not produced (visualisation is outside this library).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .forces import AIR_20C, ForceConvergenceTracker


@dataclass
class VoxelGridResult:
    """VoxelGridResult, src/geometry/voxelizer.ts:19-59."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    originX: float
    originY: float
    originZ: float
    cellFlags: np.ndarray
    boundaryIndexMap: np.ndarray
    boundaryCellIndices: np.ndarray
    boundaryQValues: np.ndarray
    boundaryMinQ: np.ndarray
    solidCellCount: int
    boundaryCellCount: int
    fluidCellCount: int
    voxelizationTimeMs: float


def _geometry(geometry):
    pos, idx = geometry
    pos = np.ascontiguousarray(np.asarray(pos, dtype=np.float32).reshape(-1, 3))
    if idx is not None:
        idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int32).reshape(-1))
    return pos, idx


def _matrix(world_matrix):
    if world_matrix is None:
        return None
    m = np.ascontiguousarray(np.asarray(world_matrix, dtype=np.float64).reshape(16))
    return m


def _tunnel(t) -> N.Tunnel:
    if isinstance(t, dict):
        return N.Tunnel(float(t["length"]), float(t["width"]), float(t["height"]))
    return N.Tunnel(*[float(v) for v in t])


class _Handle:
    def __init__(self, device: int = 0):
        lib = N.load()
        h = C.c_void_p()
        rc = lib.aerosim_create(int(device), C.byref(h))
        if rc != N.OK:
            raise N.AerosimError(rc, lib.aerosim_last_error(None).decode())
        self.lib = lib
        self.h = h

    def call(self, name: str, *args):
        rc = getattr(self.lib, name)(self.h, *args)
        N.check(rc, self.h)

    def close(self) -> None:
        if self.h:
            self.lib.aerosim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def voxelize_into(handle: _Handle, geometry, world_matrix, tunnel, grid, reset_flow: bool = True) -> N.VoxelInfo:
    pos, idx = _geometry(geometry)
    m = _matrix(world_matrix)
    info = N.VoxelInfo()
    handle.call("aerosim_voxelize", N.ptr(pos, C.c_float), pos.shape[0], N.ptr(idx, C.c_int32),
                0 if idx is None else idx.size, N.ptr(m, C.c_double), _tunnel(tunnel),
                int(grid["nx"]), int(grid["ny"]), int(grid["nz"]), 1 if reset_flow else 0, C.byref(info))
    return info


def read_voxel_grid(handle: _Handle) -> VoxelGridResult:
    info = N.VoxelInfo()
    handle.call("aerosim_get_voxel_info", C.byref(info))
    n = info.nx * info.ny * info.nz
    b = info.boundary_cell_count
    flags = np.empty(n, np.uint8)
    bmap = np.empty(n, np.int32)
    bcells = np.empty(b, np.int32)
    q = np.empty(b * 18, np.float32)
    minq = np.empty(b, np.float32)
    handle.call("aerosim_read_voxel_grid", N.ptr(flags, C.c_uint8), N.ptr(bmap, C.c_int32),
                N.ptr(bcells, C.c_int32), N.ptr(q, C.c_float), N.ptr(minq, C.c_float))
    return VoxelGridResult(info.nx, info.ny, info.nz, info.dx, info.dy, info.dz, info.origin_x,
                           info.origin_y, info.origin_z, flags, bmap, bcells, q, minq,
                           int(info.solid_cell_count), int(b), int(info.fluid_cell_count),
                           round(info.voxelization_time_ms, 2))


_shared_voxelizer: _Handle | None = None


def voxelize_mesh_to_lattice(geometry, world_matrix, tunnel, grid, device: int = 0) -> VoxelGridResult:
    """voxelizeMeshToLattice (voxelizer.ts:86-281) on the GPU; returns host arrays."""
    global _shared_voxelizer
    if _shared_voxelizer is None:
        _shared_voxelizer = _Handle(device)
    voxelize_into(_shared_voxelizer, geometry, world_matrix, tunnel, grid)
    return read_voxel_grid(_shared_voxelizer)


voxelizeMeshToLattice = voxelize_mesh_to_lattice


def frontal_area(geometry, world_matrix=None, grid_resolution: int = 512) -> float:
    """computeProjectedFrontalArea, src/geometry/frontalArea.ts:22-179 (A_ref)."""
    pos, idx = _geometry(geometry)
    m = _matrix(world_matrix)
    out = C.c_double()
    lib = N.load()
    rc = lib.aerosim_frontal_area(N.ptr(pos, C.c_float), pos.shape[0], N.ptr(idx, C.c_int32),
                                  0 if idx is None else idx.size, N.ptr(m, C.c_double),
                                  int(grid_resolution), C.byref(out))
    N.check(rc, None)
    return out.value


def _default_config() -> dict:
    """LBMEngine defaults, lbmEngine.ts:42-57 (visualisation keys omitted)."""
    return {"uInletLattice": 0.085, "nuLattice": 0.0005, "smagorinskyCs": 0.12, "groundNoSlip": False,
            "windSpeedMps": 25.0, "fluid": dict(AIR_20C), "trueSurfaceAreaM2": math.pi,
            "frontalAreaM2": math.pi * 0.25, "characteristicLengthM": 1.0,
            "boundingBoxSize": {"x": 1, "y": 1, "z": 1},
            "tunnel": {"length": 6.0, "width": 2.8, "height": 2.4}, "precision": "f32"}


class LBMEngine:
    """LBMEngine (lbmEngine.ts:39-710) with the WebGPU pipelines replaced by
    libaerosim.so.  `device` is a CUDA ordinal; there is no CPU fallback."""

    def __init__(self, device: int = 0):
        self._h = _Handle(device)
        self.config = _default_config()
        self.voxel: VoxelGridResult | None = None
        self._has_grid = False
        self._slice_dims: dict = {}  # axis -> (width, height) of the current grid's slices
        self.force_tracker = ForceConvergenceTracker()

    # -- configuration ----------------------------------------------------
    def _push_config(self) -> None:
        c = self.config
        t = c["tunnel"]
        prec = c.get("precision", "f32")
        prec = N.PRECISIONS[prec] if isinstance(prec, str) else int(prec)
        cfg = N.Config(float(c["uInletLattice"]), float(c["nuLattice"]), float(c["smagorinskyCs"]),
                       1 if c["groundNoSlip"] else 0, prec, float(c["frontalAreaM2"]),
                       float(c["characteristicLengthM"]),
                       N.Tunnel(float(t["length"]), float(t["width"]), float(t["height"])))
        self._h.call("aerosim_set_config", C.byref(cfg))

    def update_config(self, config: dict) -> None:
        """updateConfig (lbmEngine.ts:289-300): applies without resetting the flow
        (a precision change re-initialises it)."""
        self.config.update(config)
        self._push_config()

    def set_voxel_grid(self, voxel: VoxelGridResult, config: dict | None = None, reset_flow: bool = True) -> None:
        """setVoxelGrid (lbmEngine.ts:142-287): uploads a host VoxelGridResult."""
        self.voxel = voxel
        self.config.update(config or {})
        self.force_tracker.reset(60)
        self._push_config()
        origin = np.array([voxel.originX, voxel.originY, voxel.originZ], np.float64)
        flags = np.ascontiguousarray(voxel.cellFlags, dtype=np.uint8)
        bmap = np.ascontiguousarray(voxel.boundaryIndexMap, dtype=np.int32)
        bcells = np.ascontiguousarray(voxel.boundaryCellIndices, dtype=np.int32)
        q = np.ascontiguousarray(voxel.boundaryQValues, dtype=np.float32)
        self._h.call("aerosim_set_voxel_grid", voxel.nx, voxel.ny, voxel.nz, float(voxel.dx),
                     N.ptr(origin, C.c_double), N.ptr(flags, C.c_uint8), N.ptr(bmap, C.c_int32),
                     N.ptr(bcells, C.c_int32), N.ptr(q, C.c_float), int(bcells.size), 1 if reset_flow else 0)
        self._has_grid = True
        self._slice_dims = {}

    def voxelize(self, geometry, world_matrix, tunnel, grid, config: dict | None = None,
                 reset_flow: bool = True) -> N.VoxelInfo:
        """voxelizeMeshToLattice + setVoxelGrid without a host round trip."""
        self.config.update(config or {})
        self.config["tunnel"] = dict(tunnel) if isinstance(tunnel, dict) else \
            {"length": tunnel[0], "width": tunnel[1], "height": tunnel[2]}
        self.force_tracker.reset(60)
        self._push_config()
        info = voxelize_into(self._h, geometry, world_matrix, tunnel, grid, reset_flow)
        self.voxel = None
        self._has_grid = True
        self._slice_dims = {}
        return info

    def read_voxel_grid(self) -> VoxelGridResult:
        return read_voxel_grid(self._h)

    def reset_flow(self) -> None:
        """resetFlow (lbmEngine.ts:677-688)."""
        self.force_tracker.reset(60)
        if self._has_grid:
            self._h.call("aerosim_reset_flow")

    def get_step_count(self) -> int:
        v = C.c_int64()
        self._h.call("aerosim_get_step_count", C.byref(v))
        return v.value

    # -- stepping and readback ----------------------------------------------
    def step(self, n: int) -> None:
        self._h.call("aerosim_step", int(n))

    def read_forces(self) -> N.Forces:
        f = N.Forces()
        self._h.call("aerosim_read_forces", C.byref(f))
        return f

    def read_macro(self):
        info = N.VoxelInfo()
        self._h.call("aerosim_get_voxel_info", C.byref(info))
        n = info.nx * info.ny * info.nz
        ux, uy, uz, rho = (np.empty(n, np.float32) for _ in range(4))
        self._h.call("aerosim_read_macro", N.ptr(ux, C.c_float), N.ptr(uy, C.c_float),
                     N.ptr(uz, C.c_float), N.ptr(rho, C.c_float))
        return {"ux": ux, "uy": uy, "uz": uz, "rho": rho}

    def read_populations(self, dtype=np.float32) -> np.ndarray:
        info = N.VoxelInfo()
        self._h.call("aerosim_get_voxel_info", C.byref(info))
        n = info.nx * info.ny * info.nz
        out = np.empty(19 * n, dtype)
        self._h.call("aerosim_read_populations", N.vptr(out),
                     N.DTYPE_F32 if out.dtype == np.float32 else N.DTYPE_F64)
        return out

    def write_populations(self, f: np.ndarray) -> None:
        f = np.ascontiguousarray(f)
        if f.dtype not in (np.float32, np.float64):
            raise ValueError("populations must be float32 or float64")
        self._h.call("aerosim_write_populations", N.vptr(f),
                     N.DTYPE_F32 if f.dtype == np.float32 else N.DTYPE_F64)

    def mass_stats(self) -> dict:
        """computeFluidMassStats (lbmCpuReference.ts:461-495) plus rescale totals."""
        m = N.Mass()
        self._h.call("aerosim_mass_stats", C.byref(m))
        return {"totalMass": m.total_mass, "meanRho": m.mean_rho, "maxSpeed": m.max_speed,
                "hasNaN": bool(m.has_nan), "cumulativeRescale": m.cumulative_rescale,
                "rescaleCount": m.rescale_count}

    def last_step_timing(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        self._h.call("aerosim_last_step_timing", C.byref(ms), C.byref(n))
        return ms.value, n.value

    def set_pipeline_wait_limit(self, polls: int) -> None:
        """Polls of a step kernel's ring wait before the step gives up and reports
        AerosimError(ERR_DEVICE) (negative: the default; 0: give up at once, which runs
        the failure path on purpose).  reset_flow() clears the error."""
        self._h.call("aerosim_set_pipeline_wait_limit", int(polls))

    def extract_slice_rgba(self, axis: str = "z", fraction: float = 0.5, mode: str = "velocity") -> dict:
        """extractSliceRGBA (lbmCpuReference.ts:499-596) of the last step's macro fields:
        {'width', 'height', 'rgba'} with rgba uint8 [height * width * 4]."""
        a = {"x": 0, "y": 1, "z": 2}[axis]
        m = {"velocity": 0, "vorticity": 1, "pressure": 2}[mode]
        w, h = C.c_int32(), C.c_int32()
        self._h.call("aerosim_extract_slice", a, float(fraction), m, None, C.byref(w), C.byref(h))
        rgba = np.empty(w.value * h.value * 4, np.uint8)
        self._h.call("aerosim_extract_slice", a, float(fraction), m, N.ptr(rgba, C.c_uint8), C.byref(w), C.byref(h))
        return {"width": w.value, "height": h.value, "rgba": rgba}

    def step_and_extract_slice(self, substeps: int = 4, read_macro_field: bool = False, slice: dict | None = None):
        """stepAndExtractSlice (lbmEngine.ts:404-675): runs `substeps` steps, integrates
        the forces on the device and feeds the tracker; with `slice` ({'axis',
        'fraction', 'mode'}) also the slice image (width, height, rgba)."""
        if not self._has_grid:
            return None
        f = N.Forces()
        w, h = C.c_int32(), C.c_int32()
        if slice is None:
            self._h.call("aerosim_step_and_extract_slice", int(substeps), 2, 0.5, 0, None, None, None, C.byref(f))
        else:
            a = {"x": 0, "y": 1, "z": 2}[slice.get("axis", "z")]
            m = {"velocity": 0, "vorticity": 1, "pressure": 2}[slice.get("mode", "velocity")]
            frac = float(slice.get("fraction", 0.5))
            dims = self._slice_dims.get(a)
            if dims is None:  # the image size of this axis, asked once per grid
                self._h.call("aerosim_extract_slice", a, frac, m, None, C.byref(w), C.byref(h))
                dims = self._slice_dims[a] = (w.value, h.value)
            rgba = np.empty(dims[0] * dims[1] * 4, np.uint8)
            self._h.call("aerosim_step_and_extract_slice", int(substeps), a, frac, m, N.ptr(rgba, C.c_uint8),
                         C.byref(w), C.byref(h), C.byref(f))
        c = self.config
        readout = self.force_tracker.push_sample(f.step, f.cd, f.cl, f.cm, f.xcp, c["windSpeedMps"],
                                                 c["fluid"], c["frontalAreaM2"])
        out = {"stepCount": int(f.step), "forceReadout": readout, "forces": f}
        if slice is not None:
            out.update({"width": w.value, "height": h.value, "rgba": rgba})
        if read_macro_field:
            out["macroField"] = self.read_macro()
        return out

    def q_criterion(self, fields: dict | None = None, dx: float | None = None) -> dict:
        """computeQCriterion (vortexIso.ts:22-122) on the GPU: of the last step's macro
        velocity, or of caller fields {'nx','ny','nz','ux','uy','uz'[, 'flags']} with
        spacing dx.  Returns qValues, omegaMag, omegaVec, maxQ, maxOmega."""
        mq, mo = C.c_double(), C.c_double()
        if fields is None:
            info = self.voxel_info()
            n = info.nx * info.ny * info.nz
            q, om, omv = np.empty(n, np.float32), np.empty(n, np.float32), np.empty(3 * n, np.float32)
            self._h.call("aerosim_q_criterion", N.ptr(q, C.c_float), N.ptr(om, C.c_float), N.ptr(omv, C.c_float),
                         C.byref(mq), C.byref(mo))
        else:
            nx, ny, nz = int(fields["nx"]), int(fields["ny"]), int(fields["nz"])
            n = nx * ny * nz
            u = [np.ascontiguousarray(fields[k], np.float32) for k in ("ux", "uy", "uz")]
            fl = fields.get("flags")
            fl = None if fl is None else np.ascontiguousarray(fl, np.uint8)
            q, om, omv = np.empty(n, np.float32), np.empty(n, np.float32), np.empty(3 * n, np.float32)
            self._h.call("aerosim_q_criterion_fields", nx, ny, nz, float(dx), *[N.ptr(a, C.c_float) for a in u],
                         N.ptr(fl, C.c_uint8), N.ptr(q, C.c_float), N.ptr(om, C.c_float), N.ptr(omv, C.c_float),
                         C.byref(mq), C.byref(mo))
        return {"qValues": q, "omegaMag": om, "omegaVec": omv, "maxQ": mq.value, "maxOmega": mo.value}

    def set_sgs_mlp(self, params, tensor_cores: str | None = None) -> None:
        """Learned SGS closure (aerosim_b200.sgs parameters) for the following steps;
        None restores Smagorinsky.  tensor_cores selects the in-kernel evaluation:
        "mma_sync" (warp-level tiles), "tcgen05" (128-cell tiles, TMEM accumulators) or
        None to keep the current choice."""
        if params is None:
            self._h.call("aerosim_set_sgs_mlp", None)
        else:
            p = np.ascontiguousarray(params, dtype=np.float32)
            self._h.call("aerosim_set_sgs_mlp", N.ptr(p, C.c_float))
        if tensor_cores is not None:
            self.set_sgs_path(tensor_cores)

    def set_sgs_path(self, tensor_cores: str) -> str:
        """Chooses the closure's tensor-core path ("default", "mma_sync", "tcgen05");
        returns the path the next step runs ("mma_sync", "tcgen05", or "default" when
        no closure is set)."""
        used = C.c_int32()
        self._h.call("aerosim_set_sgs_mlp_path", N.SGS_PATHS[tensor_cores], C.byref(used))
        return {v: k for k, v in N.SGS_PATHS.items()}[used.value]

    def read_wall_distance(self) -> np.ndarray:
        info = self.voxel_info()
        out = np.empty(info.nx * info.ny * info.nz, np.float32)
        self._h.call("aerosim_read_wall_distance", N.ptr(out, C.c_float))
        return out

    def voxel_info(self) -> N.VoxelInfo:
        info = N.VoxelInfo()
        self._h.call("aerosim_get_voxel_info", C.byref(info))
        return info

    def close(self) -> None:
        self._h.close()

    # reference spellings
    setVoxelGrid = set_voxel_grid
    updateConfig = update_config
    stepAndExtractSlice = step_and_extract_slice
    resetFlow = reset_flow
    getStepCount = get_step_count


class LBMBatch:
    """Many wind-tunnel instances stepped together: one persistent kernel launch per
    step over the rows of all instances, runs of steps replayed from a CUDA graph
    (aerosim_batch_*).  `engines` are LBMEngine objects with voxel grids and the same
    FP32-arithmetic precision; creating the batch resets their flows.  Each engine's
    readouts (forces, macro field, populations, mass stats) follow the batch's steps."""

    def __init__(self, engines: list[LBMEngine]):
        self.lib = N.load()
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h.h for e in self.engines])
        h = C.c_void_p()
        N.check(self.lib.aerosim_batch_create(arr, len(self.engines), C.byref(h)))
        self.h = h

    def step(self, n: int = 1) -> None:
        N.check(self.lib.aerosim_batch_step(self.h, int(n)))

    def autotune(self, steps_per_trial: int = 20) -> dict:
        """Times every launch configuration that fits, keeps the fastest and resets
        the flows."""
        t = N.BatchTuning()
        N.check(self.lib.aerosim_batch_autotune(self.h, int(steps_per_trial), C.byref(t)))
        return self._tuning_dict(t)

    def set_tuning(self, stages: int, ctas_per_sm: int, graph_steps: int = 20, item_cells: int = 0) -> None:
        """Launch configuration by hand; item_cells sets the cells per work item (x-rows
        per item = item_cells / row span, 1..8; 0: 256 cells)."""
        t = N.BatchTuning(int(stages), int(ctas_per_sm), int(graph_steps), int(item_cells), 0.0)
        N.check(self.lib.aerosim_batch_set_tuning(self.h, C.byref(t)))

    def tuning(self) -> dict:
        t = N.BatchTuning()
        N.check(self.lib.aerosim_batch_get_tuning(self.h, C.byref(t)))
        return self._tuning_dict(t)

    @staticmethod
    def _tuning_dict(t) -> dict:
        return {"stages": t.stages, "ctasPerSm": t.ctas_per_sm, "graphSteps": t.graph_steps,
                "itemCells": t.item_cells, "msPerStep": t.ms_per_step}

    def last_step_timing(self) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        N.check(self.lib.aerosim_batch_last_timing(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def set_pipeline_wait_limit(self, polls: int) -> None:
        """As LBMEngine.set_pipeline_wait_limit for the batched step; autotune() resets
        a batch whose step failed."""
        N.check(self.lib.aerosim_batch_set_pipeline_wait_limit(self.h, int(polls)))

    @property
    def cells(self) -> int:
        v = C.c_int64()
        N.check(self.lib.aerosim_batch_cells(self.h, C.byref(v)))
        return v.value

    def close(self) -> None:
        if self.h:
            self.lib.aerosim_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

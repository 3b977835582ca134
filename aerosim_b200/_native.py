"""ctypes bindings of libaerosim.so (include/aerosim.h).

The library is the only compute path: importing this module fails loudly when the
built library is missing, and every call that returns a non-zero status raises
AerosimError with the library's message.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("AEROSIM_LIB", os.path.join(_HERE, "lib", "libaerosim.so"))

OK = 0
ERR_ARG, ERR_STATE, ERR_CUDA, ERR_DEVICE, ERR_NOMEM, ERR_FORMAT = -1, -2, -3, -4, -5, -6

STL_BINARY, STL_ASCII = 0, 1

CELL_FLUID, CELL_SOLID, CELL_BOUNDARY = 0, 1, 2

PREC_F32, PREC_F32_MIRROR, PREC_F16S, PREC_BF16S, PREC_F64, PREC_F16C = 0, 1, 2, 3, 4, 5
PRECISIONS = {"f32": PREC_F32, "f32_mirror": PREC_F32_MIRROR, "f16s": PREC_F16S,
              "bf16s": PREC_BF16S, "f64": PREC_F64, "f16c": PREC_F16C}
# bytes of population storage per cell and step (19 reads + 19 writes)
BYTES_PER_CELL = {PREC_F32: 152, PREC_F32_MIRROR: 152, PREC_F16S: 76, PREC_BF16S: 76, PREC_F64: 304,
                  PREC_F16C: 76}

DTYPE_F32, DTYPE_F64 = 0, 1

SGS_PATH_DEFAULT, SGS_PATH_WARP, SGS_PATH_TCGEN05 = 0, 1, 2
SGS_PATHS = {"default": SGS_PATH_DEFAULT, "mma_sync": SGS_PATH_WARP, "tcgen05": SGS_PATH_TCGEN05}


class AerosimError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"aerosim error {code}: {msg}")
        self.code = code


class Tunnel(C.Structure):
    _fields_ = [("length", C.c_double), ("width", C.c_double), ("height", C.c_double)]


class VoxelInfo(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("origin_x", C.c_double), ("origin_y", C.c_double), ("origin_z", C.c_double),
                ("solid_cell_count", C.c_int64), ("boundary_cell_count", C.c_int64),
                ("fluid_cell_count", C.c_int64), ("voxelization_time_ms", C.c_double)]


class Config(C.Structure):
    _fields_ = [("u_inlet_lattice", C.c_double), ("nu_lattice", C.c_double),
                ("smagorinsky_cs", C.c_double), ("ground_no_slip", C.c_int32),
                ("precision", C.c_int32), ("frontal_area_m2", C.c_double),
                ("characteristic_length_m", C.c_double), ("tunnel", Tunnel)]


class Forces(C.Structure):
    _fields_ = [("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double),
                ("mx", C.c_double), ("my", C.c_double), ("mz", C.c_double),
                ("cd_raw", C.c_double), ("cd", C.c_double), ("cl", C.c_double),
                ("cm", C.c_double), ("xcp", C.c_double),
                ("cut_face_links", C.c_int64), ("step", C.c_int64)]


class Mass(C.Structure):
    _fields_ = [("total_mass", C.c_double), ("mean_rho", C.c_double), ("max_speed", C.c_double),
                ("has_nan", C.c_int32), ("reserved", C.c_int32),
                ("cumulative_rescale", C.c_double), ("rescale_count", C.c_int64)]


class BatchTuning(C.Structure):
    _fields_ = [("stages", C.c_int32), ("ctas_per_sm", C.c_int32), ("graph_steps", C.c_int32),
                ("item_cells", C.c_int32), ("ms_per_step", C.c_double)]


class ModelTransform(C.Structure):
    _fields_ = [("position", C.c_double * 3), ("rotation_deg", C.c_double * 3), ("scale", C.c_double * 3)]


class MeshStats(C.Structure):
    _fields_ = [("triangle_count", C.c_int64), ("vertex_count", C.c_int64), ("open_edge_count", C.c_int64),
                ("is_watertight", C.c_int32), ("reserved", C.c_int32), ("bounding_box_size", C.c_double * 3),
                ("characteristic_length", C.c_double), ("frontal_area", C.c_double), ("volume", C.c_double)]


_P = C.c_void_p
_F32P = C.POINTER(C.c_float)
_I32P = C.POINTER(C.c_int32)
_U8P = C.POINTER(C.c_uint8)
_F64P = C.POINTER(C.c_double)

# name -> (argtypes, restype)
SIGNATURES = {
    "aerosim_abi_version": ([], C.c_int),
    "aerosim_create": ([C.c_int, C.POINTER(_P)], C.c_int),
    "aerosim_destroy": ([_P], C.c_int),
    "aerosim_last_error": ([_P], C.c_char_p),
    "aerosim_voxelize": ([_P, _F32P, C.c_int64, _I32P, C.c_int64, _F64P, Tunnel, C.c_int32,
                          C.c_int32, C.c_int32, C.c_int32, C.POINTER(VoxelInfo)], C.c_int),
    "aerosim_read_voxel_grid": ([_P, _U8P, _I32P, _I32P, _F32P, _F32P], C.c_int),
    "aerosim_get_voxel_info": ([_P, C.POINTER(VoxelInfo)], C.c_int),
    "aerosim_set_voxel_grid": ([_P, C.c_int32, C.c_int32, C.c_int32, C.c_double, _F64P, _U8P, _I32P,
                                _I32P, _F32P, C.c_int64, C.c_int32], C.c_int),
    "aerosim_set_config": ([_P, C.POINTER(Config)], C.c_int),
    "aerosim_get_config": ([_P, C.POINTER(Config)], C.c_int),
    "aerosim_reset_flow": ([_P], C.c_int),
    "aerosim_step": ([_P, C.c_int32], C.c_int),
    "aerosim_get_step_count": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "aerosim_read_forces": ([_P, C.POINTER(Forces)], C.c_int),
    "aerosim_read_macro": ([_P, _F32P, _F32P, _F32P, _F32P], C.c_int),
    "aerosim_read_populations": ([_P, _P, C.c_int32], C.c_int),
    "aerosim_write_populations": ([_P, _P, C.c_int32], C.c_int),
    "aerosim_extract_slice": ([_P, C.c_int32, C.c_double, C.c_int32, _U8P, C.POINTER(C.c_int32),
                               C.POINTER(C.c_int32)], C.c_int),
    "aerosim_step_and_extract_slice": ([_P, C.c_int32, C.c_int32, C.c_double, C.c_int32, _U8P, _I32P, _I32P,
                                        C.POINTER(Forces)], C.c_int),
    "aerosim_q_criterion": ([_P, _F32P, _F32P, _F32P, _F64P, _F64P], C.c_int),
    "aerosim_q_criterion_fields": ([_P, C.c_int32, C.c_int32, C.c_int32, C.c_double, _F32P, _F32P, _F32P, _U8P,
                                    _F32P, _F32P, _F32P, _F64P, _F64P], C.c_int),
    "aerosim_mass_stats": ([_P, C.POINTER(Mass)], C.c_int),
    "aerosim_last_step_timing": ([_P, _F64P, C.POINTER(C.c_int64)], C.c_int),
    "aerosim_step_param_bytes": ([], C.c_int),
    "aerosim_set_pipeline_wait_limit": ([_P, C.c_int32], C.c_int),
    "aerosim_batch_create": ([C.POINTER(_P), C.c_int32, C.POINTER(_P)], C.c_int),
    "aerosim_batch_destroy": ([_P], C.c_int),
    "aerosim_batch_step": ([_P, C.c_int32], C.c_int),
    "aerosim_batch_autotune": ([_P, C.c_int32, C.POINTER(BatchTuning)], C.c_int),
    "aerosim_batch_set_tuning": ([_P, C.POINTER(BatchTuning)], C.c_int),
    "aerosim_batch_get_tuning": ([_P, C.POINTER(BatchTuning)], C.c_int),
    "aerosim_batch_last_timing": ([_P, _F64P, C.POINTER(C.c_int64)], C.c_int),
    "aerosim_batch_cells": ([_P, C.POINTER(C.c_int64)], C.c_int),
    "aerosim_batch_set_pipeline_wait_limit": ([_P, C.c_int32], C.c_int),
    "aerosim_mlp_param_count": ([], C.c_int),
    "aerosim_mlp_forward": ([_F32P, _F32P, C.c_int64, _F32P], C.c_int),
    "aerosim_mlp_forward_tc": ([_F32P, _F32P, C.c_int64, _F32P], C.c_int),
    "aerosim_mlp_forward_umma": ([_F32P, _F32P, C.c_int64, _F32P], C.c_int),
    "aerosim_mlp_last_timing": ([_F64P], C.c_int),
    "aerosim_mlp_gradients": ([_F32P, _F32P, _F32P, C.c_int64, _F32P, _F64P], C.c_int),
    "aerosim_mlp_train": ([_F32P, _F32P, _F32P, C.c_int64, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _F32P],
                          C.c_int),
    "aerosim_set_sgs_mlp": ([_P, _F32P], C.c_int),
    "aerosim_set_sgs_mlp_path": ([_P, C.c_int32, C.POINTER(C.c_int32)], C.c_int),
    "aerosim_read_wall_distance": ([_P, _F32P], C.c_int),
    "aerosim_sgs_samples": ([_P, _P, C.c_float, C.c_float, C.c_int32, _F32P, _F32P, _U8P], C.c_int),
    "aerosim_frontal_area": ([_F32P, C.c_int64, _I32P, C.c_int64, _F64P, C.c_int32, _F64P], C.c_int),
    "aerosim_frontal_area_cuda": ([C.c_int32, _F32P, C.c_int64, _I32P, C.c_int64, _F64P, C.c_int32, _F64P],
                                  C.c_int),
    "aerosim_parse_stl": ([_U8P, C.c_int64, _F32P, C.c_int64, C.POINTER(C.c_int64), _I32P], C.c_int),
    "aerosim_normalize_and_center": ([_F32P, C.c_int64, _I32P], C.c_int),
    "aerosim_model_matrix": ([C.POINTER(ModelTransform), _F64P], C.c_int),
    "aerosim_compute_mesh_stats": ([_F32P, C.c_int64, _I32P, C.c_int64, C.POINTER(ModelTransform), C.c_int32,
                                    C.POINTER(MeshStats)], C.c_int),
    "aerosim_momentum_exchange_noalloc": ([_P, _P, _P, _P, C.c_int64, C.c_int32, C.c_int32, C.c_int32, _P, _P],
                                          C.c_int),
}

_lib = None


def load() -> C.CDLL:
    """Loads libaerosim.so once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m aerosim_b200.build` "
                          "(the solver has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(rc: int, handle=None) -> None:
    if rc != OK:
        msg = load().aerosim_last_error(handle)
        raise AerosimError(rc, msg.decode() if msg else "")


def ptr(a: np.ndarray | None, ctype):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(C.POINTER(ctype))


def vptr(a: np.ndarray) -> C.c_void_p:
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(a.ctypes.data)

"""B200-native AeroSim solver hot path: D3Q19 regularized LBM + Smagorinsky,
Bouzidi walls, FP64 momentum-exchange forces and the BVH voxelizer, exported by the
C-ABI library libaerosim.so (include/aerosim.h) and mirrored here for Python hosts.
"""
from ._native import AerosimError, PRECISIONS  # noqa: F401
from .engine import (LBMBatch, LBMEngine, VoxelGridResult, frontal_area, voxelize_mesh_to_lattice,  # noqa: F401
                     voxelizeMeshToLattice)
from .forces import ForceConvergenceTracker, compute_normalized_force_coefficients  # noqa: F401
from .stl import compute_mesh_stats, normalize_and_center_geometry, parse_stl  # noqa: F401

__all__ = ["LBMEngine", "LBMBatch", "VoxelGridResult", "voxelize_mesh_to_lattice", "voxelizeMeshToLattice",
           "frontal_area", "ForceConvergenceTracker", "compute_normalized_force_coefficients",
           "AerosimError", "PRECISIONS", "parse_stl", "normalize_and_center_geometry", "compute_mesh_stats"]

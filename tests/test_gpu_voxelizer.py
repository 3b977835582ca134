"""GPU voxelizer parity: libaerosim.so vs the oracle's voxelizeMeshToLattice.

Flags, the boundary index map and the ascending boundary list must be bit-exact;
q-distances must agree within 1e-6 (they are bit-exact by construction: same BVH,
same FP64 operation order, no contraction).
"""
import math

import numpy as np
import pytest

from aerosim_b200 import cases, meshes

pytestmark = pytest.mark.gpu


def _compare(gpu, orc, q_tol=1e-6):
    assert gpu.cellFlags.shape == orc.flags.shape
    assert np.array_equal(gpu.cellFlags, orc.flags), "cell flags differ"
    assert gpu.solidCellCount == orc.solid
    assert gpu.boundaryCellCount == orc.boundary_count
    assert np.array_equal(gpu.boundaryCellIndices, orc.bcells), "boundary list differs"
    assert np.array_equal(gpu.boundaryIndexMap, orc.bmap), "boundary index map differs"
    assert np.all(np.diff(gpu.boundaryCellIndices) > 0), "boundary list not ascending"
    if orc.q.size:
        assert np.max(np.abs(gpu.boundaryQValues - orc.q)) <= q_tol
        assert np.array_equal(gpu.boundaryQValues, orc.q), "q not bit-exact"
        assert np.array_equal(gpu.boundaryMinQ, orc.minq)
    assert math.isclose(gpu.dx, orc.dx, rel_tol=0, abs_tol=0)


CASES = {
    "cube_80x40x40": (lambda: meshes.box(1.0, 1.0, 1.0, 4), None, 2.0, (80, 40, 40)),
    "sphere_64x32x32": (lambda: cases.sphere_64x32x32().mesh, None, 32.0, (64, 32, 32)),
    "uvsphere_40": (lambda: meshes.uv_sphere(0.5, 96, 64), None, 2.0, (40, 40, 40)),
    "cylinder_rot": (lambda: meshes.cylinder(0.3, 1.2, 80, 4), None, 2.7, (54, 27, 27)),
    "naca_aoa12": (lambda: cases.naca_wing(12.0, 128, 64, 96).mesh, None, 64.0, (128, 64, 96)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_voxelizer_bit_exact(name, gpu_engine_cls, oracle_mod):
    from aerosim_b200 import voxelize_mesh_to_lattice
    make, world, height, (nx, ny, nz) = CASES[name]
    mesh = make()
    tunnel = {"length": nx * height / ny, "width": nz * height / ny, "height": height}
    gpu = voxelize_mesh_to_lattice(mesh, world, tunnel, {"nx": nx, "ny": ny, "nz": nz})
    orc = oracle_mod.voxelize(mesh, world, height, nx, ny, nz)
    _compare(gpu, orc)


def test_voxelizer_world_matrix_and_soup(gpu_engine_cls, oracle_mod):
    """Rotated + translated geometry (applyMatrix4) given as a non-indexed soup."""
    from aerosim_b200 import voxelize_mesh_to_lattice
    mesh = meshes.box(0.8, 0.5, 0.6, 3)
    soup = meshes.as_soup(mesh)
    a = math.radians(12.0)
    # column-major rotation about z by 12 degrees plus a translation
    m = [math.cos(a), math.sin(a), 0, 0, -math.sin(a), math.cos(a), 0, 0, 0, 0, 1, 0, 0.13, -0.07, 0.05, 1]
    tunnel = {"length": 6.0, "width": 2.8, "height": 2.4}
    gpu = voxelize_mesh_to_lattice((soup, None), m, tunnel, {"nx": 128, "ny": 64, "nz": 64})
    orc = oracle_mod.voxelize((soup, None), m, 2.4, 128, 64, 64)
    _compare(gpu, orc)
    assert gpu.solidCellCount > 100 and gpu.boundaryCellCount > 100


def test_voxelizer_non_manifold_odd_scanlines(gpu_engine_cls, oracle_mod):
    """A box with one triangle removed: odd hit counts take the 3-ray vote path."""
    from aerosim_b200 import voxelize_mesh_to_lattice
    soup = meshes.as_soup(meshes.box(1.0, 1.0, 1.0, 4))[:-3]
    tunnel = {"length": 4.0, "width": 2.0, "height": 2.0}
    gpu = voxelize_mesh_to_lattice((soup, None), None, tunnel, {"nx": 80, "ny": 40, "nz": 40})
    orc = oracle_mod.voxelize((soup, None), None, 2.0, 80, 40, 40)
    _compare(gpu, orc)


def test_voxelizer_ellipsoid_full_size(gpu_engine_cls, oracle_mod):
    """The 20480-triangle perturbed ellipsoid on the 256x128x128 lattice."""
    from aerosim_b200 import voxelize_mesh_to_lattice
    c = cases.ellipsoid_256x128x128()
    tunnel = {"length": 256.0, "width": 128.0, "height": 128.0}
    gpu = voxelize_mesh_to_lattice(c.mesh, None, tunnel, {"nx": 256, "ny": 128, "nz": 128})
    orc = oracle_mod.voxelize(c.mesh, None, 128.0, 256, 128, 128)
    _compare(gpu, orc)
    assert gpu.boundaryCellCount > 5000


def test_voxelizer_empty_and_outside(gpu_engine_cls, oracle_mod):
    """A mesh entirely outside the lattice and an empty mesh give an all-fluid grid."""
    from aerosim_b200 import voxelize_mesh_to_lattice
    tunnel = {"length": 4.0, "width": 2.0, "height": 2.0}
    far = meshes.box(0.5, 0.5, 0.5, 1, center=(10.0, 10.0, 10.0))
    gpu = voxelize_mesh_to_lattice(far, None, tunnel, {"nx": 20, "ny": 10, "nz": 10})
    orc = oracle_mod.voxelize(far, None, 2.0, 20, 10, 10)
    _compare(gpu, orc)
    assert gpu.solidCellCount == 0 and gpu.boundaryCellCount == 0
    empty = (np.zeros((0, 3), np.float32), None)
    gpu = voxelize_mesh_to_lattice(empty, None, tunnel, {"nx": 20, "ny": 10, "nz": 10})
    assert gpu.solidCellCount == 0 and int(gpu.cellFlags.sum()) == 0


def test_reference_cube_known_answer_on_gpu(gpu_engine_cls):
    """phase2.test.ts:42-60 on the GPU path: 8000 solid cells, > 2400 boundary cells."""
    from aerosim_b200 import voxelize_mesh_to_lattice
    r = voxelize_mesh_to_lattice(meshes.box(1.0, 1.0, 1.0, 4), None,
                                 {"length": 4.0, "height": 2.0, "width": 2.0}, {"nx": 80, "ny": 40, "nz": 40})
    assert r.solidCellCount == 8000
    assert r.boundaryCellCount > 2400
    assert r.cellFlags[40 + 80 * (20 + 40 * 20)] == 1
    assert r.cellFlags[2 + 80 * (2 + 40 * 2)] == 0


def test_interactive_voxelization_time(gpu_engine_cls, oracle_mod):
    """phase2.test.ts:130-150: the 'rocket_nose' ogive turned 12 degrees about z in a
    6 x 2.8 x 2.4 m tunnel on 128x64x64.  After a warm-up call, voxelization with the link
    q-distances (here the GPU voxelizer and the copy of the whole grid to the host) takes
    < 50 ms and gives > 100 solid and > 100 boundary cells; the grid is the oracle's."""
    import time
    from aerosim_b200 import voxelize_mesh_to_lattice
    mesh = meshes.ogive_nose()
    a = math.radians(12.0)
    world = [math.cos(a), math.sin(a), 0, 0, -math.sin(a), math.cos(a), 0, 0, 0, 0, 1, 0, 0, 0, 0, 1]
    tunnel = {"length": 6.0, "width": 2.8, "height": 2.4}
    grid = {"nx": 128, "ny": 64, "nz": 64}
    voxelize_mesh_to_lattice(mesh, world, tunnel, grid)
    t0 = time.perf_counter()
    gpu = voxelize_mesh_to_lattice(mesh, world, tunnel, grid)
    ms = (time.perf_counter() - t0) * 1e3
    assert gpu.solidCellCount > 100 and gpu.boundaryCellCount > 100
    assert gpu.cellFlags[gpu.boundaryCellIndices[0]] == 2
    assert ms < 50.0, ms
    _compare(gpu, oracle_mod.voxelize(mesh, world, 2.4, 128, 64, 64))

"""Batches (aerosim_batch_*): many tunnels stepped by one persistent launch per step.

Every instance of a batch must evolve exactly as the same engine stepped on its own:
populations within 1e-5 relative (FP32; the batched and the single-lattice kernels
share the cell code but are separate compilations), forces and mass-rescale history
alike, whatever the mix of lattice sizes (one row pitch for all, or several), the
CUDA-graph replay length and the launch configuration the autotuner picks.
"""
import numpy as np
import pytest

from aerosim_b200 import AerosimError, LBMBatch, LBMEngine, VoxelGridResult, cases, meshes
from aerosim_b200 import _native as N

pytestmark = pytest.mark.gpu


def _case(nx, ny, nz, r, xc):
    c = meshes.lattice_center(nx, ny, nz, 1.0, (xc, ny / 2 - 0.5, nz / 2 - 0.5))
    return cases.Case(f"b{nx}", nx, ny, nz, meshes.icosphere(r, c, 2), 0.06, 0.002, 0.1, 60)


def _engine(oracle_mod, case, precision):
    vox = oracle_mod.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    n = vox.nx * vox.ny * vox.nz
    voxel = VoxelGridResult(vox.nx, vox.ny, vox.nz, vox.dx, vox.dx, vox.dx, *vox.origin, vox.flags, vox.bmap,
                            vox.bcells, vox.q, vox.minq, vox.solid, vox.boundary_count,
                            n - vox.solid - vox.boundary_count, vox.ms)
    e = LBMEngine(0)
    a_ref = oracle_mod.frontal_area(case.mesh)
    e.set_voxel_grid(voxel, {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                             "precision": precision, "frontalAreaM2": a_ref, "characteristicLengthM": 8.0,
                             "tunnel": {"length": float(case.nx), "width": float(case.nz),
                                        "height": float(case.ny)}})
    return vox, e


def _compare(e_batch, e_alone, vox, rtol, atol=0.0):
    fb = e_batch.read_populations().astype(np.float64)
    fa = e_alone.read_populations().astype(np.float64)
    err = np.abs(fb - fa) / np.maximum(np.abs(fa), 1e-12)
    if atol:
        err = np.where(np.abs(fb - fa) <= atol, 0.0, err)
    err[np.tile(vox.flags == 1, 19)] = 0.0
    assert err.max() <= rtol, f"max relative population difference {err.max():.3e}"
    assert e_batch.get_step_count() == e_alone.get_step_count()
    gb, ga = e_batch.read_forces(), e_alone.read_forces()
    assert abs(gb.fx - ga.fx) <= 1e-4 * max(abs(ga.fx), 1e-6)
    mb, ma = e_batch.mass_stats(), e_alone.mass_stats()
    assert mb["rescaleCount"] == ma["rescaleCount"]
    mgb, mga = e_batch.read_macro(), e_alone.read_macro()
    assert np.allclose(mgb["rho"], mga["rho"], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("dims", [[(64, 24, 24), (96, 32, 24), (160, 24, 32)],   # several pitches
                                  [(128, 24, 20), (120, 32, 24), (100, 16, 16)]])  # one pitch (128)
def test_batch_matches_engines_stepped_alone(oracle_mod, dims):
    cs = [_case(nx, ny, nz, 3.0 + k, nx / 3) for k, (nx, ny, nz) in enumerate(dims)]
    pairs = [(_engine(oracle_mod, c, "f32"), _engine(oracle_mod, c, "f32")) for c in cs]
    batch = LBMBatch([p[0][1] for p in pairs])
    batch.step(37)
    batch.step(23)
    for (vox, eb), (_, ea) in pairs:
        ea.step(60)
        _compare(eb, ea, vox, 1e-5)
    batch.close()
    for (_, eb), (_, ea) in pairs:
        eb.close()
        ea.close()


@pytest.mark.parametrize("item_cells", [512, 1024])
def test_batch_with_larger_work_items_matches_engines_alone(oracle_mod, item_cells):
    """Work items of several x-rows (up to 8; the last item of an instance ragged when its
    row count is not a multiple) step every instance exactly as alone."""
    dims = [(64, 24, 24), (160, 23, 31), (100, 16, 17)]
    cs = [_case(nx, ny, nz, 3.0 + k, nx / 3) for k, (nx, ny, nz) in enumerate(dims)]
    pairs = [(_engine(oracle_mod, c, "f32"), _engine(oracle_mod, c, "f32")) for c in cs]
    batch = LBMBatch([p[0][1] for p in pairs])
    t = batch.tuning()
    batch.set_tuning(2, 1, 5, item_cells)
    assert batch.tuning()["itemCells"] == item_cells
    batch.step(40)
    for (vox, eb), (_, ea) in pairs:
        ea.step(40)
        _compare(eb, ea, vox, 1e-5)
    batch.set_tuning(t["stages"], t["ctasPerSm"], t["graphSteps"], 0)  # back to one-row items mid-run
    batch.step(10)
    for (vox, eb), (_, ea) in pairs:
        ea.step(10)
        _compare(eb, ea, vox, 1e-5)
    batch.close()
    for (_, eb), (_, ea) in pairs:
        eb.close()
        ea.close()


def test_fp16_engines_alone_match_a_batch_across_widths(oracle_mod, monkeypatch):
    """The 16-bit step kernel's multi-row work items (about 1024 cells: 4 to 32 rows, the
    last item of a lattice ragged) against the batched kernel's own item walk: each
    engine stepped alone equals its instance in a batch.  The engines stepped alone run one
    cell per thread, as the batched kernel does, so both round to 16 bits alike (two cells
    per thread is held to the one-cell kernel in tests/test_gpu_pairs.py)."""
    monkeypatch.setenv("AEROSIM_CELLS_PER_THREAD", "1")
    dims = [(33, 12, 10), (65, 10, 9), (100, 12, 7), (160, 9, 10), (300, 8, 9)]
    cs = [_case(nx, ny, nz, 2.5, nx / 3) for nx, ny, nz in dims]
    pairs = [(_engine(oracle_mod, c, "f16s"), _engine(oracle_mod, c, "f16s")) for c in cs]
    batch = LBMBatch([p[0][1] for p in pairs])
    batch.step(50)
    for (vox, eb), (_, ea) in pairs:
        ea.step(50)
        _compare(eb, ea, vox, 1e-5, atol=1e-6)
    batch.close()
    for (_, eb), (_, ea) in pairs:
        eb.close()
        ea.close()


@pytest.mark.parametrize("precision", ["f16s", "bf16s", "f16c"])
def test_batch_two_cells_per_thread_matches_engines_alone(oracle_mod, precision):
    """Instances whose rows all have an even cell count run two cells per consumer thread
    in the batched kernel, like the engines stepped alone: the same pair arithmetic, so
    within a storage rounding of each other."""
    dims = [(64, 24, 24), (96, 32, 24), (160, 24, 32)]
    cs = [_case(nx, ny, nz, 3.0 + k, nx / 3) for k, (nx, ny, nz) in enumerate(dims)]
    pairs = [(_engine(oracle_mod, c, precision), _engine(oracle_mod, c, precision)) for c in cs]
    batch = LBMBatch([p[0][1] for p in pairs])
    batch.step(50)
    for (vox, eb), (_, ea) in pairs:
        ea.step(50)
        _compare(eb, ea, vox, 1e-5, atol=1e-4 if precision == "bf16s" else 1e-5)
    batch.close()
    for (_, eb), (_, ea) in pairs:
        eb.close()
        ea.close()


def test_batch_graph_replay_equals_single_launches(oracle_mod):
    """graph_steps = 5 over 12 steps (two replays and two single launches) against
    graph_steps = 1 (every step its own launch), FP16 storage."""
    cs = [_case(64, 24, 24, 3.0, 20.0), _case(96, 24, 24, 4.0, 30.0)]
    e1 = [_engine(oracle_mod, c, "f16s") for c in cs]
    e2 = [_engine(oracle_mod, c, "f16s") for c in cs]
    b1, b2 = LBMBatch([e for _, e in e1]), LBMBatch([e for _, e in e2])
    t = b1.tuning()
    b1.set_tuning(t["stages"], t["ctasPerSm"], 5)
    b2.set_tuning(t["stages"], t["ctasPerSm"], 1)
    b1.step(12)
    b2.step(12)
    _, launches = b1.last_step_timing()
    assert launches == 12
    for (vox, x), (_, y) in zip(e1, e2):
        assert np.array_equal(x.read_populations(), y.read_populations())
    for b in (b1, b2):
        b.close()
    for _, e in e1 + e2:
        e.close()


def test_batch_autotune_picks_a_fitting_configuration_and_resets(oracle_mod):
    cs = [_case(64, 24, 24, 3.0, 20.0), _case(128, 32, 32, 5.0, 40.0)]
    es = [_engine(oracle_mod, c, "bf16s") for c in cs]
    batch = LBMBatch([e for _, e in es])
    batch.step(5)
    t = batch.autotune(4)
    assert 2 <= t["stages"] <= 6 and 1 <= t["ctasPerSm"] <= 3 and t["msPerStep"] > 0
    assert t["itemCells"] in (256, 512, 1024)
    with pytest.raises(AerosimError) as err:  # work items above 2048 cells are refused
        batch.set_tuning(2, 1, 5, 4096)
    assert err.value.code == N.ERR_ARG
    assert batch.tuning()["itemCells"] == t["itemCells"]
    for _, e in es:
        assert e.get_step_count() == 0
    batch.step(10)
    assert all(e.get_step_count() == 10 for _, e in es)
    assert batch.cells == sum(c.cells for c in cs)
    for _, e in es:
        assert not e.mass_stats()["hasNaN"]
    batch.close()
    for _, e in es:
        e.close()


def test_batch_rejects_mixed_or_unsupported_precisions(oracle_mod):
    c = _case(64, 24, 24, 3.0, 20.0)
    _, a = _engine(oracle_mod, c, "f32")
    _, b = _engine(oracle_mod, c, "f16s")
    _, m = _engine(oracle_mod, c, "f32_mirror")
    for group in ([a, b], [m], [a, a]):
        with pytest.raises(AerosimError) as e:
            LBMBatch(group)
        assert e.value.code == N.ERR_ARG
    for e in (a, b, m):
        e.close()

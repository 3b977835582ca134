"""Launch variants of the step kernel: two cells per consumer thread (packed FP32 pair
arithmetic) and the dynamic deal of work items.

* Two cells per thread is the same arithmetic on packed pairs: with FP32 storage the
  populations stay within 1e-5 relative of the oracle after 1000 steps (Cd within
  0.5 %), and every storage mode steps like the one-cell-per-thread kernel on awkward
  lattices (one and several chunks per row, nx > 256, short rows, bodies cut by the
  inlet and outlet planes, ground no-slip, a ragged last work item, rows of four cells).
  With 16-bit storage the pairs that hold a row's ends are the helper warp's (end_pair):
  the ragged item and the four-cell rows, where the consumers write nothing, test it.
* The dynamic deal changes only which CTA takes which rows: results are bit-identical
  to the static deal.
"""
import numpy as np
import pytest

from aerosim_b200 import LBMEngine, VoxelGridResult, cases, meshes

pytestmark = pytest.mark.gpu


def _engine(case, precision, ground=False):
    e = LBMEngine(0)
    e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
               {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                "precision": precision, "groundNoSlip": ground})
    return e


def _sphere_case(nx, ny, nz, r, xc, u=0.06):
    c = meshes.lattice_center(nx, ny, nz, 1.0, (xc, ny / 2 - 0.5, nz / 2 - 0.5))
    return cases.Case(f"p{nx}x{ny}x{nz}", nx, ny, nz, meshes.icosphere(r, c, 2), u, 0.002, 0.1, 100)


def test_pair_kernel_fp32_within_tolerance_of_oracle_after_1000_steps(gpu_engine_cls, oracle_mod, monkeypatch):
    monkeypatch.setenv("AEROSIM_CELLS_PER_THREAD", "2")
    case = cases.sphere_64x32x32()
    vox = oracle_mod.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    n = vox.nx * vox.ny * vox.nz
    vr = VoxelGridResult(vox.nx, vox.ny, vox.nz, vox.dx, vox.dx, vox.dx, *vox.origin, vox.flags, vox.bmap,
                         vox.bcells, vox.q, vox.minq, vox.solid, vox.boundary_count,
                         n - vox.solid - vox.boundary_count, vox.ms)
    orc = oracle_mod.Solver(vox, u_inlet=0.0, nu=case.nu, cs=case.cs)
    eng = gpu_engine_cls(0)
    eng.set_voxel_grid(vr, {"uInletLattice": 0.0, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                            "precision": "f32", "tunnel": {"length": 64.0, "width": 32.0, "height": 32.0}})
    orc.set_params(u_inlet=case.u_inlet)
    eng.update_config({"uInletLattice": case.u_inlet})
    t = oracle_mod.max_threads()
    for _ in range(10):
        orc.step(100, threads=t)
        eng.step(100)
        fg = eng.read_forces()
        me = oracle_mod.momentum_exchange(vox, orc.f(0))
        assert abs(fg.fx - me["fx"]) <= 5e-3 * abs(me["fx"]), (fg.fx, me["fx"])
    fgp, fop = eng.read_populations().astype(np.float64), orc.f(0).astype(np.float64)
    rel = np.abs(fgp - fop) / np.maximum(np.abs(fop), 1e-12)
    rel[np.tile(vox.flags == 1, 19)] = 0.0
    assert rel.max() <= 1e-5, rel.max()
    eng.close()


LATTICES = [
    (64, 32, 32, 4.0, 20.0, False),     # one chunk of 64 cells per thread row segment
    (256, 24, 20, 5.0, 70.0, False),    # the benchmark row length
    (512, 10, 8, 3.0, 100.0, False),    # two chunks per row (nx > 2 x 256 threads)
    (100, 16, 12, 4.0, 2.0, False),     # body cut by the inlet plane
    (98, 16, 12, 4.0, 96.0, True),      # body cut by the outlet plane, ground no-slip
    (6, 8, 4, 1.0, 3.0, False),         # very short rows, nz <= 4
    (64, 13, 7, 2.0, 20.0, False),      # a ragged last work item (91 rows, 16-row items at 16 bits)
    (4, 10, 6, 1.0, 1.5, False),        # every pair of a row holds a row end (nx = 4)
]


@pytest.mark.parametrize("precision", ["f32", "f16s", "bf16s", "f16c"])
@pytest.mark.parametrize("lat", LATTICES, ids=[f"{l[0]}x{l[1]}x{l[2]}" for l in LATTICES])
def test_pair_kernel_steps_like_one_cell_per_thread(gpu_engine_cls, monkeypatch, precision, lat):
    nx, ny, nz, r, xc, ground = lat
    case = _sphere_case(nx, ny, nz, r, xc)
    out = {}
    for cpt in ("1", "2"):
        monkeypatch.setenv("AEROSIM_CELLS_PER_THREAD", cpt)
        e = _engine(case, precision, ground)
        e.step(60)
        out[cpt] = (e.read_populations().astype(np.float64), e.read_macro(), e.mass_stats(),
                    e.read_voxel_grid().cellFlags)
        e.close()
    f1, m1, s1, flags = out["1"]
    f2, m2, s2, _ = out["2"]
    solid = np.tile(flags == 1, 19)
    if precision == "f32":
        rel = np.abs(f2 - f1) / np.maximum(np.abs(f1), 1e-12)
        rel[solid] = 0.0
        assert rel.max() <= 1e-5, rel.max()
    else:  # a rounding to 16 bits may fall the other way: a few storage ulps at most
        d = np.abs(f2 - f1)
        d[solid] = 0.0
        assert d.max() <= (1e-3 if precision == "bf16s" else 2e-4), d.max()
    for k in ("ux", "uy", "uz", "rho"):
        assert np.abs(m2[k] - m1[k]).max() <= (1e-5 if precision == "f32" else 1e-3), k
    assert not s2["hasNaN"]
    assert abs(s2["meanRho"] - s1["meanRho"]) <= 1e-5


@pytest.mark.parametrize("precision,cpt", [("f32", "1"), ("f32", "2"), ("f16s", "2"), ("f32_mirror", "1")])
def test_dynamic_deal_is_bit_identical_to_static(gpu_engine_cls, monkeypatch, precision, cpt):
    case = _sphere_case(128, 40, 36, 6.0, 40.0)
    monkeypatch.setenv("AEROSIM_CELLS_PER_THREAD", cpt)
    out = []
    for dyn in ("0", "1"):
        monkeypatch.setenv("AEROSIM_DYNAMIC_ITEMS", dyn)
        e = _engine(case, precision)
        e.step(41)  # odd and even steps (the walk over the items reverses on odd steps)
        out.append((e.read_populations(), e.mass_stats()))
        e.close()
    assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    assert out[0][1]["rescaleCount"] == out[1][1]["rescaleCount"]

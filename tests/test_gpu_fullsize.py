"""Solver parity at the benchmark size: the 256x128x128 perturbed-ellipsoid lattice
(4 194 304 cells, the row pitch of the timed kernel).

* The bit-parity mode (f32_mirror) against the oracle, bit for bit, for 10 steps (the
  oracle's whole-lattice steps take about a second each on one core).
* The FP32 production kernel against the bit-parity mode for 200 steps: every fluid
  population within 1e-5 relative, macro fields within 1e-5, forces within 0.5 %.
* Size-independent properties of the production kernels: a lattice at rest stays at rest
  (to a float ulp of the weights; the outlet's 3:1 blend of equal values may round) with
  no force, and the mean density stays at 1 under the mass rescale.
"""
import numpy as np
import pytest

from aerosim_b200 import VoxelGridResult, cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(oracle_mod):
    case = cases.ellipsoid_256x128x128()
    vox = oracle_mod.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    n = vox.nx * vox.ny * vox.nz
    vr = VoxelGridResult(vox.nx, vox.ny, vox.nz, vox.dx, vox.dx, vox.dx, *vox.origin, vox.flags, vox.bmap,
                         vox.bcells, vox.q, vox.minq, vox.solid, vox.boundary_count,
                         n - vox.solid - vox.boundary_count, vox.ms)
    return case, vox, vr


def _engine(gpu_engine_cls, case, vr, precision, u=None):
    eng = gpu_engine_cls(0)
    eng.set_voxel_grid(vr, {"uInletLattice": case.u_inlet if u is None else u, "nuLattice": case.nu,
                            "smagorinskyCs": case.cs, "precision": precision,
                            "tunnel": {"length": float(case.nx), "width": float(case.nz), "height": float(case.ny)}},
                       reset_flow=True)
    return eng


def test_mirror_bit_exact_at_full_size(gpu_engine_cls, oracle_mod, big):
    case, vox, vr = big
    eng = _engine(gpu_engine_cls, case, vr, "f32_mirror")
    orc = oracle_mod.Solver(vox, u_inlet=case.u_inlet, nu=case.nu, cs=case.cs)
    orc.step(10, threads=oracle_mod.max_threads())
    eng.step(10)
    fg, fo = eng.read_populations(), orc.f(0)
    nd = int(np.count_nonzero(fg.view(np.uint32) != fo.view(np.uint32)))
    assert nd == 0, f"{nd} populations differ, max |d| = {np.abs(fg - fo).max()}"
    mg, mo = eng.read_macro(), orc.macro()
    for k in ("ux", "uy", "uz", "rho"):
        assert np.array_equal(mg[k].view(np.uint32), mo[k].view(np.uint32)), k
    eng.close()


def test_fp32_against_bit_parity_mode_at_full_size(gpu_engine_cls, big):
    case, _, vr = big
    ref = _engine(gpu_engine_cls, case, vr, "f32_mirror")
    fast = _engine(gpu_engine_cls, case, vr, "f32")
    ref.step(200)
    fast.step(200)
    fr, ff = ref.read_populations().astype(np.float64), fast.read_populations()
    rel = np.abs(ff - fr) / np.maximum(np.abs(fr), 1e-12)
    rel[np.tile(vr.cellFlags == 1, 19)] = 0.0
    assert rel.max() <= 1e-5, rel.max()
    mr, mf = ref.read_macro(), fast.read_macro()
    for k in ("ux", "uy", "uz", "rho"):
        assert np.abs(mf[k] - mr[k]).max() <= 1e-5, k
    a, b = ref.read_forces(), fast.read_forces()
    assert abs(b.fx - a.fx) <= 5e-3 * abs(a.fx), (a.fx, b.fx)
    assert abs(b.cd - a.cd) <= 5e-3 * abs(a.cd), (a.cd, b.cd)
    ref.close()
    fast.close()


@pytest.mark.parametrize("precision", ["f32", "f16s", "bf16s"])
def test_rest_stays_at_rest_at_full_size(gpu_engine_cls, big, precision):
    """No inflow: every step maps the rest equilibrium onto itself, in every storage mode
    (phase4.test.ts:11-50 at the benchmark size)."""
    case, _, vr = big
    eng = _engine(gpu_engine_cls, case, vr, precision, u=0.0)
    f0 = eng.read_populations()
    eng.step(20)
    assert np.abs(eng.read_populations() - f0).max() <= 1e-7
    f = eng.read_forces()
    assert abs(f.fx) < 1e-6 and abs(f.fy) < 1e-6 and abs(f.fz) < 1e-6
    eng.close()


def test_mean_density_held_at_full_size(gpu_engine_cls, big):
    case, _, vr = big
    eng = _engine(gpu_engine_cls, case, vr, "f32")
    eng.step(500)
    m = eng.mass_stats()
    assert not m["hasNaN"]
    assert abs(m["meanRho"] - 1.0) < 2e-4, m["meanRho"]
    assert 0.05 < m["maxSpeed"] < 0.25
    eng.close()

"""FP16 storage with mass-compensated rounding (precision "f16c").

The F16C step kernels store the values of F16S (the deviation f - w_d scaled by 2^15 in
half precision) but round each cell's 18 moving populations first and give the rest
population what their rounded values leave of the cell's deviation sum.  The stored
populations of a cell then sum to the density the collision produced up to the one
rounding of f_0, where the F16S sum carries 19 independent roundings.  Checked here:

* per cell, |sum_d f_d - rho| after stepping (rho: the step's macro output, the density
  of the collision): within half an ulp of the rest population for F16C, far below the
  F16S error, on the one- and the two-cells-per-thread kernels, near-wall cells included;
* apart from that F16C steps like F16S: populations within a few storage ulps after 60
  steps.
The reference stores FP32 (lbmCpuReference.ts:76-143) and has no counterpart.
"""
import numpy as np
import pytest

from aerosim_b200 import LBMEngine, cases, meshes

pytestmark = pytest.mark.gpu


def _case(nx, ny, nz, r, xc, u=0.06):
    c = meshes.lattice_center(nx, ny, nz, 1.0, (xc, ny / 2 - 0.5, nz / 2 - 0.5))
    return cases.Case(f"c{nx}x{ny}x{nz}", nx, ny, nz, meshes.icosphere(r, c, 2), u, 0.002, 0.1, 100)


def _engine(case, precision, ground=False):
    e = LBMEngine(0)
    e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
               {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                "precision": precision, "groundNoSlip": ground})
    return e


def _cell_sum_error(e):
    """|sum_d f_d - rho| of every non-solid cell off the inlet and outlet planes (those take
    the boundary conditions' values, whose sum is not the cell's own density)."""
    info = e.voxel_info()
    n = info.nx * info.ny * info.nz
    f = e.read_populations(np.float64).reshape(19, n)
    rho = e.read_macro()["rho"].astype(np.float64)
    flags = e.read_voxel_grid().cellFlags
    x = np.arange(n) % info.nx
    sel = (flags != 1) & (x > 0) & (x < info.nx - 1)
    return np.abs(f.sum(axis=0) - rho)[sel]


# (nx, ny, nz, radius, x centre, ground): even rows run two cells per thread, odd rows one
LATTICES = [(64, 32, 32, 4.0, 20.0, False), (97, 24, 20, 5.0, 30.0, True), (256, 24, 20, 5.0, 70.0, False)]


@pytest.mark.parametrize("lat", LATTICES, ids=[f"{l[0]}x{l[1]}x{l[2]}" for l in LATTICES])
def test_compensated_cells_sum_to_the_collision_density(gpu_engine_cls, lat):
    nx, ny, nz, r, xc, ground = lat
    case = _case(nx, ny, nz, r, xc)
    err = {}
    for prec in ("f16s", "f16c"):
        e = _engine(case, prec, ground)
        e.step(200)
        err[prec] = _cell_sum_error(e)
        assert not e.mass_stats()["hasNaN"]
        e.close()
    rms = {p: float(np.sqrt(np.mean(v ** 2))) for p, v in err.items()}
    # half an ulp of a rest population below 1024 storage units (|f_0 - w_0| < 0.031)
    # is 2^-2 / 2^15 = 7.6e-6; the F16S sums carry 19 roundings of up to twice that each
    assert err["f16c"].max() <= 8e-6, (err["f16c"].max(), rms)
    assert rms["f16c"] <= 0.25 * rms["f16s"], rms


@pytest.mark.parametrize("lat", LATTICES, ids=[f"{l[0]}x{l[1]}x{l[2]}" for l in LATTICES])
def test_compensated_storage_steps_like_f16s(gpu_engine_cls, lat):
    nx, ny, nz, r, xc, ground = lat
    case = _case(nx, ny, nz, r, xc)
    out = {}
    for prec in ("f16s", "f16c"):
        e = _engine(case, prec, ground)
        e.step(60)
        out[prec] = (e.read_populations().astype(np.float64), e.read_voxel_grid().cellFlags, e.mass_stats())
        e.close()
    (fs, flags, ms), (fc, _, mc) = out["f16s"], out["f16c"]
    d = np.abs(fc - fs)
    d[np.tile(flags == 1, 19)] = 0.0
    assert d.max() <= 2e-4, d.max()
    # the mean-density rescale fires when the mean leaves 1 by 1e-4 (lbmCpuReference.ts:431-455),
    # so two storage modes may sit on either side of one rescale
    assert abs(mc["meanRho"] - ms["meanRho"]) <= 1e-4

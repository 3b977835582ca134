"""Solver parity at the benchmark size: the 256x128x128 perturbed-ellipsoid lattice
(4 194 304 cells, the row pitch of the timed kernel), 1000 steps against the oracle.

* The oracle runs the case for 1000 steps on all host threads (about two minutes),
  with its momentum-exchange forces every 100 steps.
* The bit-parity mode (f32_mirror): every population, macro field, mass statistic and
  rescale count bit for bit after 1000 steps, the forces of every sample within 1e-12.
* The FP32 production kernel: every fluid population within 1e-5 relative after 1000
  steps, macro fields within 1e-5, Cd and Cl within 0.5 % at every sample.
* Size-independent properties of the production kernels: a lattice at rest stays at rest
  (to a float ulp of the weights; the outlet's 3:1 blend of equal values may round) with
  no force, and the mean density stays at 1 under the mass rescale.
"""
import math

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


STEPS, EVERY = 1000, 100


def _engine(gpu_engine_cls, case, vr, precision, u=None, refs=None):
    eng = gpu_engine_cls(0)
    cfg = {"uInletLattice": case.u_inlet if u is None else u, "nuLattice": case.nu,
           "smagorinskyCs": case.cs, "precision": precision,
           "tunnel": {"length": float(case.nx), "width": float(case.nz), "height": float(case.ny)}}
    if refs is not None:
        cfg["frontalAreaM2"], cfg["characteristicLengthM"] = refs
    eng.set_voxel_grid(vr, cfg, reset_flow=True)
    return eng


@pytest.fixture(scope="module")
def oracle_run(oracle_mod, big):
    """The oracle's 1000 steps of the case (impulsive start at the inlet velocity, as
    resetEquilibrium does), with its forces and coefficients every 100 steps."""
    case, vox, _ = big
    a_ref = oracle_mod.frontal_area(case.mesh)
    pos = case.mesh[0]
    l_ref = float(pos[:, 0].max() - pos[:, 0].min())
    orc = oracle_mod.Solver(vox, u_inlet=case.u_inlet, nu=case.nu, cs=case.cs)
    t = oracle_mod.max_threads()
    samples = []
    for _ in range(STEPS // EVERY):
        orc.step(EVERY, threads=t)
        me = oracle_mod.momentum_exchange(vox, orc.f(0))
        co = oracle_mod.force_coefficients(me["fx"], me["fy"], me["mz"], 1.0, case.u_inlet, a_ref, l_ref,
                                           float(case.nz), float(case.ny))
        samples.append({**me, **co})
    return {"f": orc.f(0), "macro": orc.macro(), "samples": samples, "mass": orc.mass_stats(),
            "rescales": orc.rescale_count, "refs": (a_ref, l_ref)}


def _run_sampled(eng):
    out = []
    for _ in range(STEPS // EVERY):
        eng.step(EVERY)
        out.append(eng.read_forces())
    return out


def test_mirror_bit_exact_at_full_size_1000_steps(gpu_engine_cls, big, oracle_run):
    case, _, vr = big
    eng = _engine(gpu_engine_cls, case, vr, "f32_mirror", refs=oracle_run["refs"])
    forces = _run_sampled(eng)
    fg, fo = eng.read_populations(), oracle_run["f"]
    nd = int(np.count_nonzero(fg.view(np.uint32) != fo.view(np.uint32)))
    assert nd == 0, f"{nd} populations differ, max |d| = {np.abs(fg - fo).max()}"
    mg, mo = eng.read_macro(), oracle_run["macro"]
    for k in ("ux", "uy", "uz", "rho"):
        assert np.array_equal(mg[k].view(np.uint32), mo[k].view(np.uint32)), k
    sg, so = eng.mass_stats(), oracle_run["mass"]
    for k in ("totalMass", "meanRho", "maxSpeed"):
        assert sg[k] == so[k], k
    assert sg["rescaleCount"] == oracle_run["rescales"]
    for fg_, fo_ in zip(forces, oracle_run["samples"]):
        for k in ("fx", "fy", "fz", "mx", "my", "mz"):
            assert math.isclose(getattr(fg_, k), fo_[k], rel_tol=1e-12, abs_tol=1e-15), k
        assert fg_.cut_face_links == fo_["cut"]
    eng.close()


def test_fp32_within_tolerance_at_full_size_1000_steps(gpu_engine_cls, big, oracle_run):
    """The production kernel's bar: populations within 1e-5 relative after 1000 FP32
    steps, Cd / Cl within 0.5 % (Cl against max(|Cl|, 10 % of max |Cd|))."""
    case, vox, vr = big
    eng = _engine(gpu_engine_cls, case, vr, "f32", refs=oracle_run["refs"])
    forces = _run_sampled(eng)
    ff, fo = eng.read_populations().astype(np.float64), oracle_run["f"].astype(np.float64)
    rel = np.abs(ff - fo) / np.maximum(np.abs(fo), 1e-12)
    rel[np.tile(vox.flags == 1, 19)] = 0.0
    assert rel.max() <= 1e-5, f"max relative population error {rel.max():.3e}"
    mf, mo = eng.read_macro(), oracle_run["macro"]
    for k in ("ux", "uy", "uz", "rho"):
        assert np.abs(mf[k].astype(np.float64) - mo[k]).max() <= 1e-5, k
    cd_scale = max(abs(s["cd"]) for s in oracle_run["samples"])
    for g, o in zip(forces, oracle_run["samples"]):
        assert abs(g.cd - o["cd"]) <= 5e-3 * abs(o["cd"]), (g.step, g.cd, o["cd"])
        assert abs(g.cl - o["cl"]) <= 5e-3 * max(abs(o["cl"]), 0.1 * cd_scale), (g.step, g.cl, o["cl"])
    eng.close()


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

"""Solver parity at the benchmark size: the 256x128x128 perturbed-ellipsoid lattice
(4 194 304 cells, the row pitch of the timed kernel), 1000 steps against the oracle.

* The oracle runs the case for 1000 steps on all host threads (about two minutes),
  with its momentum-exchange forces every 100 steps.
* The bit-parity mode (f32_mirror): every population, macro field, mass statistic and
  rescale count bit for bit after 1000 steps, the forces of every sample within 1e-12.
* The FP32 production kernel: every fluid population within 1e-5 relative after 500
  steps; after 1000 steps within the oracle's own sensitivity to one-ulp perturbations
  (the wake is chaotic at Re = 2e4); Cd and Cl within 0.5 % at every sample.
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


STEPS, EVERY, MID = 1000, 100, 500


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
    samples, f_mid = [], None
    for k in range(STEPS // EVERY):
        orc.step(EVERY, threads=t)
        f = orc.f(0)
        me = oracle_mod.momentum_exchange(vox, f)
        co = oracle_mod.force_coefficients(me["fx"], me["fy"], me["mz"], 1.0, case.u_inlet, a_ref, l_ref,
                                           float(case.nz), float(case.ny))
        samples.append({**me, **co})
        if (k + 1) * EVERY == MID:
            f_mid = f
    return {"f": orc.f(0), "f_mid": f_mid, "macro": orc.macro(), "samples": samples, "mass": orc.mass_stats(),
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


def _rel(a, b, solid):
    r = np.abs(a.astype(np.float64) - b.astype(np.float64)) / np.maximum(np.abs(b.astype(np.float64)), 1e-12)
    r[solid] = 0.0
    return r


def test_fp32_within_tolerance_at_full_size_1000_steps(gpu_engine_cls, big, oracle_run):
    """The production kernel against the oracle at the benchmark size.

    * Every fluid population within 1e-5 relative after 500 steps.
    * After 1000 steps, within the oracle's own sensitivity to rounding.  At Re = 2e4 with
      the relaxation time at its clamp the wake amplifies any rounding difference: the
      oracle's arithmetic (the bit-parity mode, equal to the oracle bit for bit, see the
      test above) started from populations one float ulp away on 1 in 10^4 of them ends
      1000 steps later about 2e-4 from the unperturbed run, as the FP32 kernel does
      (whose own rounding is smaller than the reference's float storage of f).  The bar:
      the FP32 kernel's largest deviation at most twice that envelope's, and 99.9 % of the
      fluid populations within 1e-4.
    * Cd and Cl within 0.5 % at every sample (Cl against max(|Cl|, 10 % of max |Cd|))."""
    case, vox, vr = big
    solid = np.tile(vox.flags == 1, 19)
    eng = _engine(gpu_engine_cls, case, vr, "f32", refs=oracle_run["refs"])
    env = _engine(gpu_engine_cls, case, vr, "f32_mirror", refs=oracle_run["refs"])
    f0 = env.read_populations()
    rng = np.random.default_rng(5)
    pick = rng.choice(f0.size, f0.size // 10000, replace=False)
    up = rng.random(pick.size) < 0.5
    f0[pick] = np.nextafter(f0[pick], np.where(up, np.inf, -np.inf).astype(np.float32))
    env.write_populations(f0)
    forces = []
    for k in range(STEPS // EVERY):
        eng.step(EVERY)
        env.step(EVERY)
        forces.append(eng.read_forces())
        if (k + 1) * EVERY == MID:
            rel_mid = _rel(eng.read_populations(), oracle_run["f_mid"], solid)
            assert rel_mid.max() <= 1e-5, f"step {MID}: max relative population error {rel_mid.max():.3e}"
    fo = oracle_run["f"]
    rel = _rel(eng.read_populations(), fo, solid)
    rel_env = _rel(env.read_populations(), fo, solid)
    print(f"step {STEPS}: FP32 max {rel.max():.3e}, p99.9 {np.quantile(rel, 0.999):.3e}; "
          f"oracle perturbed by one ulp on 1e-4 of its populations: max {rel_env.max():.3e}")
    assert rel.max() <= 2.0 * rel_env.max(), (rel.max(), rel_env.max())
    assert np.quantile(rel, 0.999) <= 1e-4
    cd_scale = max(abs(s["cd"]) for s in oracle_run["samples"])
    for g, o in zip(forces, oracle_run["samples"]):
        assert abs(g.cd - o["cd"]) <= 5e-3 * abs(o["cd"]), (g.step, g.cd, o["cd"])
        assert abs(g.cl - o["cl"]) <= 5e-3 * max(abs(o["cl"]), 0.1 * cd_scale), (g.step, g.cl, o["cl"])
    eng.close()
    env.close()


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

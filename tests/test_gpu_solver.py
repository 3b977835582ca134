"""GPU solver parity: libaerosim.so vs the oracle's LBMCpuReferenceSolver.

* FP32-mirror mode (FP64 arithmetic rounded like the reference's JavaScript) must be
  bit-exact: populations, macro fields, mass statistics and rescale decisions.
* The FP32 production path must match within 1e-5 relative after 1000 steps, with
  Cd / Cl within 0.5 %.
* FP64 storage is the GPU oracle run; FP16/BF16 shifted storage is judged against it.
"""
import math

import numpy as np
import pytest

from aerosim_b200 import _native as N
from aerosim_b200 import cases, meshes

pytestmark = pytest.mark.gpu

THREADS = 0  # 0 -> all host threads for the oracle


def _threads(oracle_mod):
    return THREADS or oracle_mod.max_threads()


def _voxel_result(v):
    from aerosim_b200 import VoxelGridResult
    n = v.nx * v.ny * v.nz
    return VoxelGridResult(v.nx, v.ny, v.nz, v.dx, v.dx, v.dx, *v.origin, v.flags, v.bmap, v.bcells, v.q,
                           v.minq, v.solid, v.boundary_count, n - v.solid - v.boundary_count, v.ms)


def _pair(gpu_engine_cls, oracle_mod, case, precision, from_rest=True, a_ref=None, l_ref=None):
    """Oracle solver and GPU engine on the same oracle-voxelized grid, same start."""
    vox = oracle_mod.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    u0 = 0.0 if from_rest else case.u_inlet
    orc = oracle_mod.Solver(vox, u_inlet=u0, nu=case.nu, cs=case.cs, ground_no_slip=case.ground_no_slip)
    eng = gpu_engine_cls(0)
    cfg = {"uInletLattice": u0, "nuLattice": case.nu, "smagorinskyCs": case.cs,
           "groundNoSlip": case.ground_no_slip, "precision": precision,
           "tunnel": {"length": float(case.nx), "width": float(case.nz), "height": float(case.ny)}}
    if a_ref is not None:
        cfg["frontalAreaM2"] = a_ref
        cfg["characteristicLengthM"] = l_ref
    eng.set_voxel_grid(_voxel_result(vox), cfg, reset_flow=True)
    if from_rest:
        orc.set_params(u_inlet=case.u_inlet)
        eng.update_config({"uInletLattice": case.u_inlet})
    return vox, orc, eng


def _bitdiff(a, b):
    a32 = a.view(np.uint32)
    b32 = b.view(np.uint32)
    return int(np.count_nonzero(a32 != b32))


def test_mirror_bit_exact_sphere_1000_steps(gpu_engine_cls, oracle_mod):
    case = cases.sphere_64x32x32()
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32_mirror")
    t = _threads(oracle_mod)
    # step 0: initial equilibrium
    assert _bitdiff(eng.read_populations(), orc.f(0)) == 0
    done = 0
    for target in (1, 10, 100, 1000):
        orc.step(target - done, threads=t)
        eng.step(target - done)
        done = target
        fg, fo = eng.read_populations(), orc.f(0)
        nd = _bitdiff(fg, fo)
        assert nd == 0, f"step {target}: {nd} populations differ, max |d| = {np.max(np.abs(fg - fo))}"
        mg, mo = eng.read_macro(), orc.macro()
        for k in ("ux", "uy", "uz", "rho"):
            assert _bitdiff(mg[k], mo[k]) == 0, f"step {target}: macro {k} differs"
    sg, so = eng.mass_stats(), orc.mass_stats()
    assert sg["totalMass"] == so["totalMass"]
    assert sg["meanRho"] == so["meanRho"]
    assert sg["maxSpeed"] == so["maxSpeed"]
    assert sg["rescaleCount"] == orc.rescale_count
    # forces from identical populations: same per-cell sums, tree-ordered total
    fg = eng.read_forces()
    fo = oracle_mod.momentum_exchange(vox, orc.f(0))
    for k in ("fx", "fy", "fz", "mx", "my", "mz"):
        assert math.isclose(getattr(fg, k), fo[k], rel_tol=1e-12, abs_tol=1e-15), k
    assert fg.cut_face_links == fo["cut"]


def test_fp32_within_tolerance_after_1000_steps(gpu_engine_cls, oracle_mod):
    """Populations within 1e-5 relative after 1000 FP32 steps; Cd/Cl within 0.5 %."""
    case = cases.sphere_64x32x32()
    a_ref = oracle_mod.frontal_area(case.mesh)
    pos = case.mesh[0]
    l_ref = float(pos[:, 0].max() - pos[:, 0].min())
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32", a_ref=a_ref, l_ref=l_ref)
    t = _threads(oracle_mod)
    cd_g, cd_o, cl_g, cl_o = [], [], [], []
    for _ in range(10):
        orc.step(100, threads=t)
        eng.step(100)
        fg = eng.read_forces()
        me = oracle_mod.momentum_exchange(vox, orc.f(0))
        co = oracle_mod.force_coefficients(me["fx"], me["fy"], me["mz"], 1.0, case.u_inlet, a_ref, l_ref,
                                           float(case.nz), float(case.ny))
        cd_g.append(fg.cd); cd_o.append(co["cd"]); cl_g.append(fg.cl); cl_o.append(co["cl"])
    fgp, fop = eng.read_populations(), orc.f(0)
    rel = np.abs(fgp.astype(np.float64) - fop) / np.maximum(np.abs(fop), 1e-12)
    solid = np.tile(vox.flags == 1, 19)
    rel[solid] = 0.0
    assert rel.max() <= 1e-5, f"max relative population error {rel.max():.3e}"
    for g, o in zip(cd_g, cd_o):
        assert abs(g - o) <= 5e-3 * abs(o), (g, o)
    cl_scale = max(abs(c) for c in cd_o)
    for g, o in zip(cl_g, cl_o):
        assert abs(g - o) <= 5e-3 * max(abs(o), 0.1 * cl_scale), (g, o)


def test_f64_oracle_mode_close_to_reference(gpu_engine_cls, oracle_mod):
    case = cases.sphere_64x32x32()
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f64")
    orc.step(200, threads=_threads(oracle_mod))
    eng.step(200)
    fg = eng.read_populations(np.float64)
    fo = orc.f(0).astype(np.float64)
    assert np.max(np.abs(fg - fo)) < 1e-6


@pytest.mark.parametrize("prec,tol", [("f16s", 0.01), ("bf16s", 0.05)])
def test_reduced_storage_cd_vs_f64(gpu_engine_cls, oracle_mod, prec, tol):
    """Shifted 16-bit storage: Cd after 1000 steps against the FP64-storage GPU run."""
    case = cases.sphere_64x32x32()
    a_ref = oracle_mod.frontal_area(case.mesh)
    res = {}
    for p in ("f64", prec):
        _, _, eng = _pair(gpu_engine_cls, oracle_mod, case, p, a_ref=a_ref, l_ref=8.0)
        eng.step(1000)
        res[p] = eng.read_forces()
        m = eng.mass_stats()
        assert not m["hasNaN"]
    assert abs(res[prec].cd - res["f64"].cd) <= tol * abs(res["f64"].cd), (res[prec].cd, res["f64"].cd)


def test_mirror_ground_no_slip_and_thin_domain(gpu_engine_cls, oracle_mod):
    """ABL inlet profile + no-slip floor (groundNoSlip) and a 3-cell-deep domain
    (no side walls, nz <= 4) against the oracle, bit for bit."""
    nx, ny, nz = 48, 20, 3
    c = meshes.lattice_center(nx, ny, nz, 1.0, (12, 10, 1))
    cyl = meshes.cylinder(2.5, 6.0, 32, 1, axis=2, center=c)
    case = cases.Case("cyl", nx, ny, nz, cyl, 0.1, 0.1 * 5 / 180, 0.04, 150, ground_no_slip=True)
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32_mirror", from_rest=False)
    orc.step(150, threads=1)
    eng.step(150)
    assert _bitdiff(eng.read_populations(), orc.f(0)) == 0
    mg, mo = eng.read_macro(), orc.macro()
    for k in ("ux", "uy", "uz", "rho"):
        assert _bitdiff(mg[k], mo[k]) == 0


def test_write_read_populations_roundtrip(gpu_engine_cls, oracle_mod):
    case = cases.sphere_64x32x32()
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32_mirror")
    orc.step(7, threads=_threads(oracle_mod))
    eng.step(3)
    eng.write_populations(orc.f(0))
    assert _bitdiff(eng.read_populations(), orc.f(0)) == 0


def test_zero_inflow_zero_force(gpu_engine_cls, oracle_mod):
    """phase4.test.ts:11-50 on the GPU: u = 0 gives |F| < 1e-6 after 5 steps."""
    mesh = meshes.uv_sphere(0.5, 96, 64)
    eng = gpu_engine_cls(0)
    eng.voxelize(mesh, None, {"length": 4.8, "height": 2.4, "width": 2.4}, {"nx": 48, "ny": 24, "nz": 24},
                 {"uInletLattice": 0.0, "nuLattice": 0.005, "precision": "f32"})
    eng.step(5)
    f = eng.read_forces()
    assert abs(f.fx) < 1e-6 and abs(f.fy) < 1e-6 and abs(f.fz) < 1e-6


def test_mass_conservation_re1e5(gpu_engine_cls):
    """phase3.test.ts:8-43 on the GPU: 10 000 steps at Re = 1e5 on 16x8x8."""
    mesh = meshes.uv_sphere(0.5, 96, 64)
    eng = gpu_engine_cls(0)
    u = 0.09
    eng.voxelize(mesh, None, {"length": 4.0, "height": 2.0, "width": 2.0}, {"nx": 16, "ny": 8, "nz": 8},
                 {"uInletLattice": u, "nuLattice": u * 6.0 / 1e5, "smagorinskyCs": 0.14, "precision": "f32"})
    eng.step(10000)
    m = eng.mass_stats()
    assert not m["hasNaN"]
    assert abs(m["meanRho"] - 1.0) < 0.015
    assert 0.01 < m["maxSpeed"] < 0.25


def test_error_status_paths(gpu_engine_cls):
    from aerosim_b200 import AerosimError
    eng = gpu_engine_cls(0)
    with pytest.raises(AerosimError) as e:
        eng.step(1)
    assert e.value.code == N.ERR_STATE
    with pytest.raises(AerosimError) as e:
        eng.update_config({"precision": 99})
    assert e.value.code == N.ERR_ARG
    from aerosim_b200 import VoxelGridResult
    bad = VoxelGridResult(4, 4, 4, 1.0, 1.0, 1.0, -2, -2, -2, np.full(64, 7, np.uint8), np.full(64, -1, np.int32),
                          np.zeros(0, np.int32), np.zeros(0, np.float32), np.zeros(0, np.float32), 0, 0, 64, 0)
    eng.update_config({"precision": "f32"})
    with pytest.raises(AerosimError) as e:
        eng.set_voxel_grid(bad, {})
    assert e.value.code == N.ERR_ARG
    assert eng.step_and_extract_slice(4) is None


def test_fused_frame_without_boundary_cells(gpu_engine_cls, oracle_mod):
    """An empty tunnel has no boundary cells, so no force kernel runs in the frame and the
    steps' error code comes back by its own copy: zero forces, the step count advancing,
    the image of a split call, and the same populations as plain steps on a twin."""
    case = cases.Case("empty", 40, 16, 16, (np.zeros((0, 3), np.float32), None), 0.05, 0.01, 0.1, 8)
    _, _, fused = _pair(gpu_engine_cls, oracle_mod, case, "f32")
    _, _, split = _pair(gpu_engine_cls, oracle_mod, case, "f32")
    for k in range(3):
        a = fused.step_and_extract_slice(4, slice={"axis": "z", "fraction": 0.5, "mode": "velocity"})
        split.step(4)
        f = a["forces"]
        assert (f.fx, f.fy, f.fz, f.mz, f.cut_face_links) == (0.0, 0.0, 0.0, 0.0, 0)
        assert a["stepCount"] == 4 * (k + 1)
        b = split.extract_slice_rgba("z", 0.5, "velocity")
        assert (a["width"], a["height"]) == (40, 16) and np.array_equal(a["rgba"], b["rgba"])
    assert np.array_equal(fused.read_populations().view(np.uint32), split.read_populations().view(np.uint32))
    fused.close()
    split.close()


@pytest.mark.parametrize("dims", [(33, 12, 10), (97, 9, 7), (289, 6, 6), (3, 5, 6), (40, 20, 3), (64, 1, 8),
                                  (65, 10, 8), (150, 8, 6), (200, 6, 6)])
def test_mirror_bit_exact_awkward_lattices(gpu_engine_cls, oracle_mod, dims):
    """Row lengths that shift the thread mapping (nx = 1 mod 32), split a row over
    several chunks (nx > 256), leave consumer warps without a row (row spans of 96,
    160 and 224 threads), the minimum nx = 3, thin domains and ny = 1."""
    nx, ny, nz = dims
    r = max(1.0, min(ny, nz) / 4.0)
    c = meshes.lattice_center(nx, ny, nz, 1.0, (nx / 3, ny / 2 - 0.5, nz / 2 - 0.5))
    mesh = meshes.icosphere(r, c, 2) if nx > 8 and ny > 2 else (np.zeros((0, 3), np.float32), None)
    case = cases.Case("awkward", nx, ny, nz, mesh, 0.05, 0.01, 0.1, 60)
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32_mirror")
    orc.step(60, threads=1)
    eng.step(60)
    assert _bitdiff(eng.read_populations(), orc.f(0)) == 0
    mg, mo = eng.read_macro(), orc.macro()
    for k in ("ux", "uy", "uz", "rho"):
        assert _bitdiff(mg[k], mo[k]) == 0, k


@pytest.mark.parametrize("dims,xc", [((33, 12, 10), None), ((97, 9, 7), None), ((289, 6, 6), None), ((3, 5, 6), None),
                                     ((40, 20, 3), None), ((64, 1, 8), None), ((150, 8, 6), None),
                                     ((200, 6, 6), None), ((64, 16, 16), 1.0),
                                     ((64, 16, 16), 62.0), ((65, 16, 16), 63.4), ((96, 16, 16), 0.2)])
def test_fp32_awkward_lattices_and_bodies_at_the_faces(gpu_engine_cls, oracle_mod, dims, xc):
    """FP32 path on the awkward row lengths, and with a body cut by the inlet or outlet
    plane: solid and near-wall cells at ix = 0, 1, nx-2, nx-1 (inlet from a solid
    neighbour's unit density, deferred inlet/outlet, outlet from a never-written
    solid cell).  Populations within 1e-5 relative, macro fields within 1e-5."""
    nx, ny, nz = dims
    if xc is None:
        r = max(1.0, min(ny, nz) / 4.0)
        center = (nx / 3, ny / 2 - 0.5, nz / 2 - 0.5)
    else:
        r = 4.0
        center = (xc, ny / 2 - 0.5, nz / 2 - 0.5)
    c = meshes.lattice_center(nx, ny, nz, 1.0, center)
    mesh = meshes.icosphere(r, c, 2) if nx > 8 and ny > 2 else (np.zeros((0, 3), np.float32), None)
    case = cases.Case("awkward", nx, ny, nz, mesh, 0.05, 0.01, 0.1, 60)
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32")
    if xc is not None:
        fl = vox.flags.reshape(nz, ny, nx)
        edge = fl[:, :, [0, 1, nx - 2, nx - 1]]
        assert (edge != 0).any(), "the body must reach the x faces"
    orc.step(60, threads=1)
    eng.step(60)
    fg, fo = eng.read_populations().astype(np.float64), orc.f(0)
    rel = np.abs(fg - fo) / np.maximum(np.abs(fo), 1e-12)
    rel[np.tile(vox.flags == 1, 19)] = 0.0
    assert rel.max() <= 1e-5, f"max relative population error {rel.max():.3e}"
    mg, mo = eng.read_macro(), orc.macro()
    for k in ("ux", "uy", "uz", "rho"):
        assert np.allclose(mg[k], mo[k], rtol=1e-5, atol=1e-6), k


def test_engines_sharing_a_kernel_with_different_rings(gpu_engine_cls, oracle_mod):
    """Two engines whose lattices use the same kernel instance (same row pitch) but
    different shared-memory rings step alternately: configuring the second must not
    shrink the first one's shared-memory limit."""
    engines = []
    for dims in [(128, 24, 20), (120, 48, 24)]:
        c = cases.Case("pair", *dims, (np.zeros((0, 3), np.float32), None), 0.05, 0.01, 0.1, 5)
        _, orc, eng = _pair(gpu_engine_cls, oracle_mod, c, "f32")
        engines.append(eng)
    for _ in range(2):
        for eng in engines:
            eng.step(3)
    assert [e.get_step_count() for e in engines] == [6, 6]


@pytest.mark.parametrize("precision", ["f32_mirror", "f32"])
def test_slice_images_match_the_oracle(gpu_engine_cls, oracle_mod, precision):
    """extractSliceRGBA on the three axes and the three field modes after 150 steps:
    byte-identical to the oracle in the bit-parity mode; in FP32 at most a few pixels
    one colour level apart."""
    case = cases.sphere_64x32x32()
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, precision)
    orc.step(150, threads=_threads(oracle_mod))
    eng.step(150)
    for axis in ("x", "y", "z"):
        for mode in ("velocity", "vorticity", "pressure"):
            ref = oracle_mod.extract_slice(orc, axis, 0.45, mode)
            got = eng.extract_slice_rgba(axis, 0.45, mode)
            img = got["rgba"].reshape(got["height"], got["width"], 4)
            assert img.shape == ref.shape
            diff = np.abs(img.astype(int) - ref.astype(int))
            if precision == "f32_mirror":
                assert diff.max() == 0, (axis, mode)
            else:
                assert diff.max() <= 2 and np.mean(diff > 0) < 0.01, (axis, mode, diff.max())


def test_fused_frame_equals_separate_calls(gpu_engine_cls, oracle_mod):
    """aerosim_step_and_extract_slice (one synchronization) gives the same force sums,
    coefficients and slice bytes as aerosim_step + aerosim_read_forces +
    aerosim_extract_slice on a twin engine, frame after frame, with and without a slice."""
    case = cases.sphere_64x32x32()
    _, _, fused = _pair(gpu_engine_cls, oracle_mod, case, "f32")
    _, _, split = _pair(gpu_engine_cls, oracle_mod, case, "f32")
    sl = {"axis": "y", "fraction": 0.5, "mode": "vorticity"}
    for k in range(4):
        a = fused.step_and_extract_slice(4, slice=sl if k % 2 == 0 else None)
        split.step(4)
        fb = split.read_forces()
        fa = a["forces"]
        assert (fa.fx, fa.fy, fa.fz, fa.mz, fa.cd, fa.cl, fa.step) == (fb.fx, fb.fy, fb.fz, fb.mz, fb.cd, fb.cl, fb.step)
        if k % 2 == 0:
            b = split.extract_slice_rgba("y", 0.5, "vorticity")
            assert (a["width"], a["height"]) == (b["width"], b["height"])
            assert np.array_equal(a["rgba"], b["rgba"])
    fused.close()
    split.close()

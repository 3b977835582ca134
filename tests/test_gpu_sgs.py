"""Learned SGS closure on the GPU (libaerosim.so): the training kernels' loss and
gradient against the float64 oracle (oracle/mlp.py), the FP32 and tensor-core forward
passes, training, the jump-flood wall distance against a brute-force distance, the
closure's wiring into the step kernel, and the training samples of a fine / coarse
engine pair."""
import numpy as np
import pytest

from aerosim_b200 import LBMEngine, cases, meshes, sgs
from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(0.0, 1.0, (n, 8)).astype(np.float32)
    Y = (np.log1p(np.exp(X[:, 0] - 0.5 * X[:, 7])) + 0.2 * X[:, 6] ** 2).astype(np.float32)
    return X, Y


def test_gpu_gradients_match_the_oracle():
    X, Y = _data(3000)
    p = sgs.init_params(1)
    g, loss = sgs.gradients(p, X, Y)
    lo, go = omlp.loss_and_grad(p.astype(np.float64), X, Y)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    scale = np.abs(go).max()
    assert np.abs(g - go).max() <= 1e-4 * scale, np.abs(g - go).max() / scale


def test_forward_fp32_and_tensor_cores():
    X, _ = _data(4099, 2)
    p = sgs.init_params(3)
    ref, _ = omlp.forward(p.astype(np.float64), X)
    f32 = sgs.forward(p, X)
    tc = sgs.forward(p, X, tensor_cores=True)
    assert np.allclose(f32, ref, rtol=1e-5, atol=1e-6)
    # BF16 weights and activations, FP32 accumulation
    assert np.abs(tc - ref).max() <= 0.03 * np.abs(ref).max() + 1e-3


@pytest.mark.parametrize("n", [1, 127, 128, 129, 70001])
def test_forward_tcgen05_tiles(n):
    """128-row tiles on tcgen05 (TMEM accumulators): the oracle within the BF16 bound, and
    the warp-level tensor-core path within FP32 summation-order differences."""
    X, _ = _data(n, 11)
    X[::7] *= 3.0
    p = sgs.init_params(12)
    ref, _ = omlp.forward(p.astype(np.float64), X)
    umma = sgs.forward(p, X, tensor_cores="tcgen05")
    warp = sgs.forward(p, X, tensor_cores=True)
    assert np.isfinite(umma).all()
    assert np.abs(umma - ref).max() <= 0.03 * np.abs(ref).max() + 1e-3
    assert np.abs(umma - warp).max() <= 1e-4 * np.abs(warp).max() + 1e-5, np.abs(umma - warp).max()


def test_training_lowers_the_loss_and_beats_a_constant():
    X, Y = _data(20000, 4)
    p0 = sgs.init_params(5)
    p, curve = sgs.train(p0, X, Y, iters=600, batch=2048, lr=3e-3, seed=7)
    assert curve[-50:].mean() < 0.2 * curve[:10].mean()
    Xv, Yv = _data(5000, 9)
    mse = float(np.mean((sgs.forward(p, Xv) - Yv) ** 2))
    assert mse < 0.1 * float(np.var(Yv))


def test_wall_distance_matches_brute_force():
    nx, ny, nz = 40, 20, 16
    c = meshes.lattice_center(nx, ny, nz, 1.0, (12.0, 9.5, 7.5))
    case = cases.Case("wd", nx, ny, nz, meshes.icosphere(4.0, c, 2), 0.05, 0.01, 0.1, 1)
    e = LBMEngine(0)
    e.voxelize(case.mesh, None, case.tunnel, {"nx": nx, "ny": ny, "nz": nz}, {"precision": "f32"})
    d = e.read_wall_distance().reshape(nz, ny, nx)
    flags = e.read_voxel_grid().cellFlags.reshape(nz, ny, nx)
    sol = np.argwhere(flags == 1).astype(np.float64)
    pts = np.argwhere(np.ones_like(flags, bool)).astype(np.float64)
    ref = np.sqrt(((pts[:, None, :] - sol[None, :, :]) ** 2).sum(-1).min(1)).reshape(nz, ny, nx)
    err = np.abs(d - ref)
    assert np.mean(err < 1e-4) > 0.995 and err.max() < 0.5
    e.close()


def test_constant_closure_equals_plain_viscosity():
    """A network whose output is a constant ratio r (W3 = 0, softplus(b3) = r) must step
    exactly like the plain method without Smagorinsky at nu = nu_0 (1 + r).  Empty
    tunnel: near-wall cells keep Smagorinsky, so a body would differ there."""
    case = cases.Case("empty", 64, 32, 32, (np.zeros((0, 3), np.float32), None), 0.05, 0.004, 0.1, 200)
    r = 0.5
    p = sgs.init_params(0)
    p[-33:-1] = 0.0
    p[-1] = np.log(np.expm1(r))
    out = []
    for closure in (True, False):
        e = LBMEngine(0)
        nu = case.nu * (1.0 + r) if not closure else case.nu
        e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
                   {"uInletLattice": case.u_inlet, "nuLattice": nu, "smagorinskyCs": 0.1 if closure else 0.0,
                    "precision": "f32"})
        if closure:
            e.set_sgs_mlp(p)
        e.step(200)
        out.append(e.read_populations().astype(np.float64))
        e.close()
    rel = np.abs(out[0] - out[1]) / np.maximum(np.abs(out[1]), 1e-12)
    assert rel.max() <= 1e-4, rel.max()


def test_trained_closure_runs_stably_and_samples_are_sane():
    fine_case = cases.scaled_ellipsoid(128, 64, 64)
    coarse_case = cases.scaled_ellipsoid(64, 32, 32)
    eng = []
    for c in (fine_case, coarse_case):
        e = LBMEngine(0)
        e.voxelize(c.mesh, None, c.tunnel, {"nx": c.nx, "ny": c.ny, "nz": c.nz},
                   {"uInletLattice": c.u_inlet, "nuLattice": c.nu, "smagorinskyCs": c.cs, "precision": "f32"})
        eng.append(e)
    fine, coarse = eng
    fine.step(400)
    X, Y = sgs.samples(fine, coarse)
    assert X.shape[0] > 10000 and np.all(np.isfinite(X)) and np.all(Y >= 0.0)
    p, _ = sgs.train(sgs.init_params(0), X, Y, iters=300, batch=4096, lr=2e-3)
    coarse.set_sgs_mlp(p)
    coarse.step(300)
    m = coarse.mass_stats()
    assert not m["hasNaN"] and abs(m["meanRho"] - 1.0) < 1e-3
    coarse.set_sgs_mlp(None)
    coarse.step(10)
    for e in eng:
        e.close()


def test_trained_closure_beats_smagorinsky_on_held_out_samples():
    """What the trained network gains over the method without it.  The solver generates
    a fine 128x64x64 run of the perturbed ellipsoid (Smagorinsky, FP32); its flow,
    box-filtered onto the 2x coarser 64x32x32 lattice, gives the eddy viscosity the coarse
    grid needs (least-squares fit of the filtered subgrid stress per cell).  The network
    is trained on one snapshot and scored on a later one it has not seen: its nu_t / nu_0
    must have a clearly lower mean squared error than the Smagorinsky eddy viscosity of
    the same cells (lbmCpuReference.ts:264-282, the closure it replaces), and lower than
    predicting no eddy viscosity at all."""
    fine_case = cases.scaled_ellipsoid(128, 64, 64)
    coarse_case = cases.scaled_ellipsoid(64, 32, 32)
    eng = []
    for c in (fine_case, coarse_case):
        e = LBMEngine(0)
        e.voxelize(c.mesh, None, c.tunnel, {"nx": c.nx, "ny": c.ny, "nz": c.nz},
                   {"uInletLattice": c.u_inlet, "nuLattice": c.nu, "smagorinskyCs": c.cs, "precision": "f32"})
        eng.append(e)
    fine, coarse = eng
    fine.step(1600)
    Xt, Yt = sgs.samples(fine, coarse)
    fine.step(400)
    Xv, Yv = sgs.samples(fine, coarse)
    for e in eng:
        e.close()
    assert Xt.shape[0] > 20000 and Xv.shape[0] > 20000
    p, curve = sgs.train(sgs.init_params(0), Xt, Yt, iters=1500, batch=8192, lr=2e-3, seed=0)
    assert np.all(np.isfinite(curve))
    nu0 = (max(3.0 * coarse_case.nu + 0.5, 0.5015) - 0.5) / 3.0
    mse_mlp = float(np.mean((sgs.forward(p, Xv).astype(np.float64) - Yv) ** 2))
    mse_smag = float(np.mean((sgs.smagorinsky_ratio(Xv, nu0, coarse_case.cs) - Yv) ** 2))
    mse_zero = float(np.mean(Yv.astype(np.float64) ** 2))
    print(f"held-out MSE of nu_t/nu_0: closure {mse_mlp:.4g}, Smagorinsky {mse_smag:.4g}, zero {mse_zero:.4g}")
    assert mse_mlp < 0.9 * mse_smag, (mse_mlp, mse_smag)
    assert mse_mlp < mse_zero, (mse_mlp, mse_zero)


def _closure_params(seed):
    """A network with a non-trivial response over the flow's features (larger weights
    than the initialisation, output around nu_t / nu_0 ~ 1)."""
    p = sgs.init_params(seed)
    p[: 32 * 8] *= 4.0
    return p


@pytest.mark.parametrize("dims", [(128, 64, 64), (256, 32, 32), (100, 24, 20), (120, 15, 9)])
def test_in_step_closure_tcgen05_tiles_match_warp_tiles(dims):
    """The closure inside the step kernel as 128-cell tcgen05 tiles (four consumer warps,
    one thread issuing each layer, TMEM accumulators) steps like the warp-level mma.sync
    tiles: the same BF16 network with FP32 accumulation in another summation order, so
    populations agree within 1e-5 relative after 60 steps.  Row pitches 128 and 256, one
    or two rows per work item, an odd row count (the last item's second row is empty)."""
    nx, ny, nz = dims
    case = cases.scaled_ellipsoid(nx, ny, nz)
    p = _closure_params(21)
    out = {}
    for path in ("mma_sync", "tcgen05"):
        e = LBMEngine(0)
        e.voxelize(case.mesh, None, case.tunnel, {"nx": nx, "ny": ny, "nz": nz},
                   {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                    "precision": "f32"})
        e.set_sgs_mlp(p)
        assert e.set_sgs_path(path) == path
        e.step(60)
        m = e.mass_stats()
        assert not m["hasNaN"]
        out[path] = (e.read_populations().astype(np.float64), e.read_macro(), e.read_voxel_grid().cellFlags)
        e.close()
    fw, mw, flags = out["mma_sync"]
    ft, mt, _ = out["tcgen05"]
    rel = np.abs(ft - fw) / np.maximum(np.abs(fw), 1e-12)
    rel[np.tile(flags == 1, 19)] = 0.0
    assert rel.max() <= 1e-5, rel.max()
    for k in ("ux", "uy", "uz", "rho"):
        assert np.abs(mt[k] - mw[k]).max() <= 1e-5, k


def test_in_step_closure_tcgen05_constant_network_equals_plain_viscosity():
    """W3 = 0 and softplus(b3) = r: the tcgen05 tiles must return r for every cell, so the
    run equals the plain method at nu_0 (1 + r) (empty tunnel, as the warp-path test)."""
    case = cases.Case("empty", 128, 32, 32, (np.zeros((0, 3), np.float32), None), 0.05, 0.004, 0.1, 200)
    r = 0.5
    p = sgs.init_params(0)
    p[-33:-1] = 0.0
    p[-1] = np.log(np.expm1(r))
    out = []
    for closure in (True, False):
        e = LBMEngine(0)
        nu = case.nu * (1.0 + r) if not closure else case.nu
        e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
                   {"uInletLattice": case.u_inlet, "nuLattice": nu, "smagorinskyCs": 0.1 if closure else 0.0,
                    "precision": "f32"})
        if closure:
            e.set_sgs_mlp(p, tensor_cores="tcgen05")
            assert e.set_sgs_path("tcgen05") == "tcgen05"
        e.step(200)
        out.append(e.read_populations().astype(np.float64))
        e.close()
    rel = np.abs(out[0] - out[1]) / np.maximum(np.abs(out[1]), 1e-12)
    assert rel.max() <= 1e-4, rel.max()


def test_in_step_closure_path_selection():
    """tcgen05 tiles need every work item to keep the 8 consumer warps busy (row pitch
    128 or 256); other lattices keep the warp-level tiles."""
    for (nx, expect) in ((64, "mma_sync"), (160, "mma_sync"), (128, "tcgen05"), (250, "tcgen05")):
        case = cases.scaled_ellipsoid(nx, 32, 32)
        e = LBMEngine(0)
        e.voxelize(case.mesh, None, case.tunnel, {"nx": nx, "ny": 32, "nz": 32}, {"precision": "f32"})
        assert e.set_sgs_path("tcgen05") == "default"  # no closure set yet
        e.set_sgs_mlp(sgs.init_params(1))
        assert e.set_sgs_path("tcgen05") == expect, nx
        assert e.set_sgs_path("mma_sync") == "mma_sync"
        e.step(3)
        e.close()

"""Failure path of the step kernels: a ring wait that runs out ends the step with an
error status, not a hang, and the engine recovers.

Every wait of the step kernels' shared-memory ring (consumers waiting for a bulk copy,
the producer waiting for a free slot) is bounded; when the bound is reached the CTA
sets the device error flag, waits with the full bound for its own copies still in
flight and returns, and the step call reports AEROSIM_ERR_DEVICE.  The tests set the
bound to 0 polls, so every wait gives up without looking -- a flag that nothing sets,
made on purpose without any fault -- and check the status and the recovery: after
aerosim_reset_flow the engine steps exactly like a fresh one.  The reference's own
guard is the null result of stepAndExtractSlice when the engine cannot step
(lbmEngine.ts:420, 593-600).
"""
import numpy as np
import pytest

from aerosim_b200 import AerosimError, LBMBatch, LBMEngine, cases, meshes
from aerosim_b200 import _native as N

pytestmark = pytest.mark.gpu


def _engine(case, precision):
    e = LBMEngine(0)
    e.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
               {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                "precision": precision})
    return e


@pytest.mark.parametrize("precision", ["f32", "f16s", "f32_mirror"])
def test_step_wait_timeout_reports_device_error_and_recovers(gpu_engine_cls, precision):
    case = cases.sphere_64x32x32()
    fresh = _engine(case, precision)
    fresh.step(10)
    f_fresh = fresh.read_populations()
    fresh.close()

    e = _engine(case, precision)
    e.set_pipeline_wait_limit(0)
    with pytest.raises(AerosimError) as err:
        e.step(3)
    assert err.value.code == N.ERR_DEVICE
    assert "timed out" in str(err.value)
    # the error stays reported until the flow is reset
    e.set_pipeline_wait_limit(-1)
    with pytest.raises(AerosimError):
        e.step(1)
    e.reset_flow()
    e.step(10)
    assert e.get_step_count() == 10
    assert np.array_equal(e.read_populations().view(np.uint32), f_fresh.view(np.uint32))
    e.close()


def test_closure_tcgen05_groups_leave_together_on_timeout(gpu_engine_cls):
    """With the closure on tcgen05 tiles, the four warps of a group agree on a failed ring
    wait at a named barrier and leave together (none waits for a warp that has left);
    the TMEM is released and the engine recovers."""
    from aerosim_b200 import sgs
    case = cases.scaled_ellipsoid(128, 32, 32)
    fresh = _engine(case, "f32")
    fresh.set_sgs_mlp(sgs.init_params(2), tensor_cores="tcgen05")
    fresh.step(10)
    f_fresh = fresh.read_populations()
    fresh.close()
    e = _engine(case, "f32")
    e.set_sgs_mlp(sgs.init_params(2), tensor_cores="tcgen05")
    assert e.set_sgs_path("tcgen05") == "tcgen05"
    e.set_pipeline_wait_limit(0)
    with pytest.raises(AerosimError) as err:
        e.step(3)
    assert err.value.code == N.ERR_DEVICE
    e.set_pipeline_wait_limit(-1)
    e.reset_flow()
    e.step(10)
    assert np.array_equal(e.read_populations().view(np.uint32), f_fresh.view(np.uint32))
    e.close()


def test_batch_wait_timeout_reports_device_error_and_recovers(gpu_engine_cls):
    def case(nx, r):
        c = meshes.lattice_center(nx, 24, 24, 1.0, (nx / 3, 11.5, 11.5))
        return cases.Case(f"b{nx}", nx, 24, 24, meshes.icosphere(r, c, 2), 0.06, 0.002, 0.1, 40)

    cs = [case(64, 3.0), case(96, 4.0)]
    engines = [_engine(c, "f16s") for c in cs]
    batch = LBMBatch(engines)
    batch.set_tuning(stages=2, ctas_per_sm=1, graph_steps=4, item_cells=256)
    batch.set_pipeline_wait_limit(0)
    with pytest.raises(AerosimError) as err:
        batch.step(8)  # graph replays and single launches
    assert err.value.code == N.ERR_DEVICE
    batch.set_pipeline_wait_limit(-1)
    batch.autotune(4)  # resets every instance and the batch's error flag
    batch.step(10)
    for e in engines:
        m = e.mass_stats()
        assert not m["hasNaN"] and abs(m["meanRho"] - 1.0) < 1e-3
    batch.close()
    for e in engines:
        e.close()

"""Flow diagnostics on the GPU: computeQCriterion (vortexIso.ts:22-122) against the
oracle, bit for bit, on the reference's known-answer fields and on a solver flow."""
import numpy as np
import pytest

from aerosim_b200 import cases
from test_oracle_known_answers import _rotation_and_shear

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def test_q_criterion_fields_match_the_oracle(gpu_engine_cls, oracle_mod):
    nx, ny, nz, dx, rot, shear = _rotation_and_shear()
    eng = gpu_engine_cls(0)
    for field in (rot, shear):
        u = [a.astype(np.float32).ravel() for a in field]
        ref = oracle_mod.q_criterion(nx, ny, nz, dx, *u)
        got = eng.q_criterion({"nx": nx, "ny": ny, "nz": nz, "ux": u[0], "uy": u[1], "uz": u[2]}, dx)
        for k in ("qValues", "omegaMag", "omegaVec"):
            assert _same(got[k], ref[k]), k
        assert got["maxQ"] == ref["maxQ"] and got["maxOmega"] == ref["maxOmega"]
    eng.close()


def test_q_criterion_of_a_solver_flow(gpu_engine_cls, oracle_mod):
    from test_gpu_solver import _pair
    case = cases.sphere_64x32x32()
    vox, orc, eng = _pair(gpu_engine_cls, oracle_mod, case, "f32_mirror")
    orc.step(120, threads=oracle_mod.max_threads())
    eng.step(120)
    m = orc.macro()
    ref = oracle_mod.q_criterion(case.nx, case.ny, case.nz, 1.0, m["ux"], m["uy"], m["uz"], vox.flags)
    got = eng.q_criterion()
    for k in ("qValues", "omegaMag", "omegaVec"):
        assert _same(got[k], ref[k]), k
    assert got["maxQ"] == ref["maxQ"]
    eng.close()

"""The committed golden fixtures (tests/golden/sphere_64x32x32.json): the oracle must
regenerate them exactly (CPU), and the GPU bit-parity path must reproduce every digest
without running the oracle (GPU)."""
import hashlib
import json
import math
import os

import numpy as np
import pytest

from aerosim_b200 import cases

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "sphere_64x32x32.json")))


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_oracle_regenerates_the_golden_fixture():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = mg.generate()
    assert g["grid"] == GOLDEN["grid"]
    assert g["steps"] == GOLDEN["steps"]
    for a, b in zip(g["forces"], GOLDEN["forces"]):
        for k in b:
            assert math.isclose(a[k], b[k], rel_tol=1e-12, abs_tol=1e-15), (b["step"], k)


@pytest.mark.gpu
def test_gpu_mirror_path_reproduces_the_golden_digests(gpu_engine_cls):
    case = cases.sphere_64x32x32()
    eng = gpu_engine_cls(0)
    eng.voxelize(case.mesh, None, case.tunnel, {"nx": case.nx, "ny": case.ny, "nz": case.nz},
                 {"uInletLattice": 0.0, "nuLattice": case.nu, "smagorinskyCs": case.cs, "precision": "f32_mirror",
                  "frontalAreaM2": GOLDEN["a_ref"], "characteristicLengthM": GOLDEN["l_ref"],
                  "tunnel": {"length": float(case.nx), "width": float(case.nz), "height": float(case.ny)}})
    v = eng.read_voxel_grid()
    assert {"flags": sha(v.cellFlags), "bmap": sha(v.boundaryIndexMap), "bcells": sha(v.boundaryCellIndices),
            "q": sha(v.boundaryQValues), "minq": sha(v.boundaryMinQ), "solid": int(v.solidCellCount),
            "boundary": int(v.boundaryCellCount)} == GOLDEN["grid"]
    eng.update_config({"uInletLattice": case.u_inlet})
    forces = {f["step"]: f for f in GOLDEN["forces"]}
    done = 0
    for target in sorted({int(k) for k in GOLDEN["steps"]} | set(forces)):
        if target > done:
            eng.step(target - done)
            done = target
        if str(target) in GOLDEN["steps"]:
            ref = GOLDEN["steps"][str(target)]
            m = eng.read_macro()
            assert sha(eng.read_populations()) == ref["f"], f"populations at step {target}"
            for k in ("ux", "uy", "uz", "rho"):
                assert sha(m[k]) == ref[k], f"macro {k} at step {target}"
            ms = eng.mass_stats()
            assert ms["totalMass"] == ref["total_mass"] and ms["rescaleCount"] == ref["rescale_count"]
        if target in forces:
            f, ref = eng.read_forces(), forces[target]
            for k in ("fx", "fy", "fz", "mz", "cd", "cl", "cm"):
                assert math.isclose(getattr(f, k), ref[k], rel_tol=1e-10, abs_tol=1e-14), (target, k)
            assert f.cut_face_links == ref["cut"]
    eng.close()

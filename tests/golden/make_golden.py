"""Generates tests/golden/sphere_64x32x32.json from the oracle (oracle/, the C++
restatement of the reference's CPU solver): the seeded 64x32x32 sphere case (1280-
triangle icosphere, u = 0.05, Re = 100, Cs = 0.1, started from rest), with

  * SHA-256 digests of the voxel grid arrays (flags, boundary index map, boundary
    list, q values, min q) and their counts;
  * SHA-256 digests of the float32 populations (dense SoA f[d * N + idx]) and the
    macro fields after 0, 1, 10, 100 and 1000 steps, and the mass statistics;
  * the momentum-exchange forces and coefficients every 100 steps.

The reference itself cannot run here (TypeScript, no JavaScript runtime) and ships no
vectors, so these fixtures are the oracle's; the bit-parity (f32_mirror) GPU path must
reproduce every digest, and the oracle is re-checked against them on the CPU.

  python tests/golden/make_golden.py     (rewrites the JSON; commit it with the change)
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from aerosim_b200 import cases  # noqa: E402

OUT = os.path.join(HERE, "sphere_64x32x32.json")
STEPS = (0, 1, 10, 100, 1000)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def generate(threads: int = 0) -> dict:
    case = cases.sphere_64x32x32()
    vox = oracle.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    a_ref = oracle.frontal_area(case.mesh)
    pos = case.mesh[0]
    l_ref = float(pos[:, 0].max() - pos[:, 0].min())
    s = oracle.Solver(vox, u_inlet=0.0, nu=case.nu, cs=case.cs)
    s.set_params(u_inlet=case.u_inlet)
    t = threads or oracle.max_threads()
    out = {"case": "sphere_64x32x32 (u 0.05, nu 0.004, Cs 0.1, from rest)",
           "grid": {"flags": sha(vox.flags), "bmap": sha(vox.bmap), "bcells": sha(vox.bcells), "q": sha(vox.q),
                    "minq": sha(vox.minq), "solid": int(vox.solid), "boundary": int(vox.boundary_count)},
           "a_ref": a_ref, "l_ref": l_ref, "steps": {}, "forces": []}
    done = 0
    for target in range(0, 1001, 100):
        # advance through the digest steps and the force samples in order
        for stop in sorted({x for x in STEPS if done < x <= target} | {target}):
            if stop > done:
                s.step(stop - done, threads=t)
                done = stop
            if stop in STEPS and str(stop) not in out["steps"]:
                m = s.macro()
                ms = s.mass_stats()
                out["steps"][str(stop)] = {"f": sha(s.f(0)), "ux": sha(m["ux"]), "uy": sha(m["uy"]),
                                           "uz": sha(m["uz"]), "rho": sha(m["rho"]),
                                           "total_mass": ms["totalMass"], "rescale_count": int(s.rescale_count)}
        if target > 0:
            me = oracle.momentum_exchange(vox, s.f(0))
            co = oracle.force_coefficients(me["fx"], me["fy"], me["mz"], 1.0, case.u_inlet, a_ref, l_ref,
                                           float(case.nz), float(case.ny))
            out["forces"].append({"step": target, "fx": me["fx"], "fy": me["fy"], "fz": me["fz"], "mz": me["mz"],
                                  "cut": int(me["cut"]), "cd": co["cd"], "cl": co["cl"], "cm": co["cm"],
                                  "xcp": co["xcp"]})
    return out


if __name__ == "__main__":
    g = generate()
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print(OUT)

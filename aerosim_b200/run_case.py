"""Steps one workload and prints its device time: the command the ncu summaries in
profiles/ were captured with.

  python -m aerosim_b200.run_case ellipsoid PRECISION STEPS [CLOSURE_PATH]
  python -m aerosim_b200.run_case naca_batch STEPS

ellipsoid: the 256x128x128 perturbed-ellipsoid lattice, 20 steps then STEPS steps
(PRECISION f32, f16s, bf16s, f32_mirror or f64; CLOSURE_PATH mma_sync or tcgen05 runs the
shipped learned closure on that tensor-core path).  naca_batch: the 32 NACA 0012 wings
(FP16S) in one batch with a fixed launch shape (2 ring slots, 2 CTAs per SM, 1024-cell
items, no CUDA graph), STEPS single launches.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from . import LBMBatch, LBMEngine, cases


def _engine(c, precision: str) -> LBMEngine:
    e = LBMEngine(0)
    e.voxelize(c.mesh, None, c.tunnel, {"nx": c.nx, "ny": c.ny, "nz": c.nz},
               {"uInletLattice": c.u_inlet, "nuLattice": c.nu, "smagorinskyCs": c.cs, "precision": precision})
    return e


def main(argv: list[str]) -> None:
    if argv and argv[0] == "ellipsoid":
        precision, steps = argv[1], int(argv[2])
        closure = argv[3] if len(argv) > 3 else ""
        e = _engine(cases.ellipsoid_256x128x128(), precision)
        if closure:
            w = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "sgs_mlp_ellipsoid.npz"))
            e.set_sgs_mlp(w["params"])
            print("closure path", e.set_sgs_path(closure))
        e.step(20)
        e.step(steps)
        ms, launches = e.last_step_timing()
        print(f"{precision} {closure}: {ms / steps * 1e3:.2f} us per step over {steps} steps ({launches} launches)",
              flush=True)
        e.close()
    elif argv and argv[0] == "naca_batch":
        steps = int(argv[1])
        engines = [_engine(c, "f16s") for c in cases.naca_batch(steps=steps)]
        b = LBMBatch(engines)
        b.set_tuning(stages=2, ctas_per_sm=2, graph_steps=1, item_cells=1024)
        b.step(steps)
        ms, launches = b.last_step_timing()
        print(f"naca_batch: {ms / steps * 1e3:.1f} us per batched step over {steps} steps, {b.cells} cells", flush=True)
        b.close()
        for e in engines:
            e.close()
    else:
        print(__doc__)
        sys.exit(2)


if __name__ == "__main__":
    main(sys.argv[1:])

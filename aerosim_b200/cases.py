"""Workload definitions of the solver's parity and benchmark cases.

Each case fixes the lattice, the body mesh (synthetic, seeded) and the solver
parameters.  Lattice units: h = tunnel height / ny = 1 m, so cell counts and metres
coincide and the tunnel is nx x ny x nz metres.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import meshes


@dataclass
class Case:
    name: str
    nx: int
    ny: int
    nz: int
    mesh: meshes.Mesh
    u_inlet: float
    nu: float
    cs: float
    steps: int
    start_from_rest: bool = True       # construct with u = 0, then switch the inlet on
    ground_no_slip: bool = False
    notes: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def tunnel(self) -> tuple[float, float, float]:
        """(length, width, height) in metres with h = 1 m."""
        return (float(self.nx), float(self.nz), float(self.ny))

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz


def sphere_64x32x32() -> Case:
    """64x32x32 lattice, sphere of diameter 8 cells (1280-triangle icosphere) centred on
    cell (16, 16, 16), u = 0.05, Re = 100 on the diameter (nu = 0.004), Cs = 0.1, 1000
    steps from rest."""
    nx, ny, nz = 64, 32, 32
    c = meshes.lattice_center(nx, ny, nz, 1.0, (16, 16, 16))
    return Case("sphere_64x32x32", nx, ny, nz, meshes.icosphere(4.0, c, 3), 0.05, 0.004, 0.1, 1000)


def ellipsoid_256x128x128(steps: int = 20000) -> Case:
    """256x128x128 lattice, seeded perturbed ellipsoid (semi-axes 40x16x12 cells, 20480
    triangles, 1.5-cell radial noise from 8 degree-1/2 spherical harmonics, seed 0) at
    x = nx/4, centred in y and z; u = 0.08, Re = 2e4 on the 80-cell body length
    (nu = 3.2e-4), Cs = 0.1."""
    nx, ny, nz = 256, 128, 128
    c = meshes.lattice_center(nx, ny, nz, 1.0, (nx / 4 - 0.5, ny / 2 - 0.5, nz / 2 - 0.5))
    mesh = meshes.perturbed_ellipsoid((40.0, 16.0, 12.0), 1.5, 0, 5, c)
    return Case("ellipsoid_256x128x128", nx, ny, nz, mesh, 0.08, 0.08 * 80 / 2e4, 0.1, steps)


def scaled_ellipsoid(nx: int, ny: int, nz: int, steps: int = 100) -> Case:
    """The perturbed-ellipsoid case scaled to another lattice (same proportions)."""
    s = ny / 128.0
    c = meshes.lattice_center(nx, ny, nz, 1.0, (nx / 4 - 0.5, ny / 2 - 0.5, nz / 2 - 0.5))
    mesh = meshes.perturbed_ellipsoid((40.0 * s, 16.0 * s, 12.0 * s), 1.5 * s, 0, 5 if s >= 0.5 else 4, c)
    return Case(f"ellipsoid_{nx}x{ny}x{nz}", nx, ny, nz, mesh, 0.08, 0.08 * 80 * s / 2e4, 0.1, steps)


def naca_wing(aoa_deg: float, nx: int, ny: int, nz: int, steps: int = 10000) -> Case:
    """Extruded NACA 0012 wing (chord 48, span 64 cells) at angle of attack `aoa_deg`,
    u = 0.06, Re = 5e3 on the chord (nu = 5.76e-4)."""
    c = meshes.lattice_center(nx, ny, nz, 1.0, (nx / 3 - 0.5, ny / 2 - 0.5, nz / 2 - 0.5))
    mesh = meshes.naca0012_wing(48.0, 64.0, aoa_deg, c)
    return Case(f"naca0012_{aoa_deg:+.1f}deg_{nx}x{ny}x{nz}", nx, ny, nz, mesh, 0.06, 0.06 * 48 / 5e3, 0.1,
                steps, extra={"aoa_deg": aoa_deg})


def naca_batch(n: int = 32, seed: int = 0, steps: int = 10000, span: float = 64.0) -> list[Case]:
    """The batched sweep: `n` extruded NACA 0012 wings (chord 48 cells) at angles of
    attack drawn uniformly from [-8, 22] degrees (numpy default_rng(seed)), on lattices
    growing from 128x64x64 to 190x95x95 (nx = 128 + 2i, ny = nz = nx / 2); u = 0.06,
    Re = 5e3 on the chord (nu = 5.76e-4), Cs = 0.1.  The span is min(span, nz - 8)
    cells so that the wing tips stay 4 cells clear of the side walls on the narrowest
    lattices (nz = 64)."""
    rng = np.random.default_rng(seed)
    aoa = rng.uniform(-8.0, 22.0, n)
    out = []
    for i in range(n):
        nx = 128 + 2 * i
        ny = nz = nx // 2
        c = meshes.lattice_center(nx, ny, nz, 1.0, (nx / 3 - 0.5, ny / 2 - 0.5, nz / 2 - 0.5))
        mesh = meshes.naca0012_wing(48.0, min(span, nz - 8.0), float(aoa[i]), c)
        out.append(Case(f"naca0012_{aoa[i]:+.1f}deg_{nx}x{ny}x{nz}", nx, ny, nz, mesh, 0.06, 0.06 * 48 / 5e3,
                        0.1, steps, extra={"aoa_deg": float(aoa[i])}))
    return out


def mesh_reference_quantities(mesh: meshes.Mesh, frontal_fn) -> tuple[float, float]:
    """(A_ref, L_ref): projected frontal area on the Y-Z plane at 512^2 (frontalArea.ts)
    and the streamwise bounding-box length (stlLoader.ts:231)."""
    pos, idx = mesh
    a_ref = frontal_fn(pos, idx)
    l_ref = max(1e-4, float(pos[:, 0].max()) - float(pos[:, 0].min()))
    return a_ref, l_ref


def flag_counts(flags: np.ndarray) -> dict:
    return {int(k): int(v) for k, v in zip(*np.unique(flags, return_counts=True))}

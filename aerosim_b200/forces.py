"""Host-side force post-processing: computeNormalizedForceCoefficients and
ForceConvergenceTracker (src/solver/forceIntegrator.ts:240-424).

The momentum-exchange sums themselves are computed on the GPU (FP64) by
libaerosim.so; these are the scalar host steps the reference runs on top of them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import jsfmt

# FLUID_PRESETS.air_20c, src/core/types.ts:15-22
AIR_20C = {"id": "air_20c", "name": "Air (Sea Level, 20°C)", "density": 1.204,
           "kinematicViscosity": 1.516e-5, "speedOfSound": 343.2}

NEWTONS_TO_LBF = 0.224808943   # lbmConstants.ts:101
NEWTONS_TO_KGF = 0.101971621   # lbmConstants.ts:102
MASKELL_EPSILON = 2.5          # lbmConstants.ts:92


def compute_normalized_force_coefficients(fx_lat: float, fy_lat: float, fz_lat: float, mz_lat: float,
                                          dx: float, u_inlet_lattice: float, frontal_area_m2: float,
                                          characteristic_length_m: float, tunnel_width: float,
                                          tunnel_height: float) -> dict:
    """forceIntegrator.ts:240-315 (Cd_raw, Maskell-corrected Cd, Cl, Cm, X_cp)."""
    cell_area = dx * dx
    q_lat = max(1e-9, 0.5 * 1.0 * u_inlet_lattice * u_inlet_lattice)
    a_ref = max(1e-4, frontal_area_m2 / cell_area)
    l_ref = max(1.0, characteristic_length_m / dx)
    cd_raw = fx_lat / (q_lat * a_ref)
    cl = fy_lat / (q_lat * a_ref)
    cm = mz_lat / (q_lat * a_ref * l_ref)
    tunnel_area = max(1e-4, tunnel_width * tunnel_height)
    blockage = min(0.40, frontal_area_m2 / tunnel_area)
    cd = cd_raw / (1.0 + MASKELL_EPSILON * max(0.0, cd_raw) * blockage)
    half = characteristic_length_m * 0.5
    xcp = max(-half, min(half, -(mz_lat / fy_lat) * dx)) if abs(fy_lat) > 1e-5 else 0.0
    return {"cdRaw": cd_raw, "cdCorrected": cd, "cl": cl, "cmPitch": cm, "centerOfPressureX": xcp,
            "fxLattice": fx_lat, "fyLattice": fy_lat, "fzLattice": fz_lat}


def _round_half_up(x: float, digits: int) -> float:
    """Number(x.toFixed(digits)): ties of the exact binary value round up."""
    return float(jsfmt.to_fixed(x, digits))


@dataclass
class _Sample:
    step: int
    cd: float
    cl: float
    cm: float
    xcp: float


class ForceConvergenceTracker:
    """forceIntegrator.ts:321-424: 180-sample history, rolling window statistics."""

    def __init__(self) -> None:
        self.window_size = 60
        self.samples: list[_Sample] = []
        self._history: list[dict] = []  # readout history entries, kept in step with samples
        self._history_q = None          # the q_inf * A_ref they were computed with

    def reset(self, window_size: int = 60) -> None:
        self.window_size = window_size
        self.samples = []
        self._history = []
        self._history_q = None

    @staticmethod
    def _entry(s: _Sample, q_area: float) -> dict:
        return {"step": s.step, "cd": s.cd, "cl": s.cl, "cm": s.cm, "xcp": s.xcp,
                "dragForceN": s.cd * q_area, "liftForceN": s.cl * q_area}

    def push_sample(self, step: int, cd: float, cl: float, cm: float, xcp: float, wind_speed: float,
                    fluid: dict, frontal_area_m2: float) -> dict:
        self.samples.append(_Sample(step, cd, cl, cm, xcp))
        dropped = len(self.samples) > 180
        if dropped:
            self.samples.pop(0)
        recent = self.samples[-self.window_size:]
        n = len(recent)
        # plain left-to-right sums as the reference adds them (:355-366); Python's sum()
        # of floats compensates the rounding and can differ in the last bit
        sum_cd = sum_cl = sum_cm = sum_xcp = 0.0
        for s in recent:
            sum_cd += s.cd
            sum_cl += s.cl
            sum_cm += s.cm
            sum_xcp += s.xcp
        mean_cd = sum_cd / n
        mean_cl = sum_cl / n
        mean_cm = sum_cm / n
        mean_xcp = sum_xcp / n
        var_cd = 0.0
        for s in recent:
            diff = s.cd - mean_cd
            var_cd += diff * diff
        std_cd = math.sqrt(var_cd / max(1, n))
        rel_std = std_cd / max(0.02, abs(mean_cd))
        fill = min(1.0, n / 25)
        stability = _round_half_up(max(0.0, min(99.9, fill * (1.0 - min(1.0, rel_std * 4.0)) * 100)), 1)
        converged = n >= 20 and stability >= 96.0
        q_area = 0.5 * fluid["density"] * wind_speed * wind_speed * frontal_area_m2
        drag_n = q_area * mean_cd
        lift_n = q_area * mean_cl
        return {
            "instantCd": cd, "instantCl": cl, "meanCd": mean_cd, "meanCl": mean_cl, "stdCd": std_cd,
            "dragForceNewtons": drag_n, "dragForceLbs": drag_n * NEWTONS_TO_LBF,
            "dragForceKgf": drag_n * NEWTONS_TO_KGF, "liftForceNewtons": lift_n,
            "liftForceLbs": lift_n * NEWTONS_TO_LBF, "pitchingMomentCm": mean_cm,
            "centerOfPressureX": mean_xcp, "stabilityPercent": stability, "isConverged": converged,
            "history": self._history_list(q_area, dropped),
        }

    def _history_list(self, q_area: float, dropped: bool) -> list:
        """The per-sample entries of every readout (forces from this call's q_inf * A_ref),
        updated by one entry per sample instead of rebuilt; the entries are shared between
        readouts and must be treated as read-only."""
        if q_area != self._history_q or len(self._history) != len(self.samples) - 1 + dropped:
            self._history = [self._entry(s, q_area) for s in self.samples]
            self._history_q = q_area
        else:
            if dropped:
                self._history.pop(0)
            self._history.append(self._entry(self.samples[-1], q_area))
        return list(self._history)

    pushSample = push_sample

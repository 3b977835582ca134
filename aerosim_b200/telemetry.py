"""Telemetry export with the reference's schemas: exportTelemetryToCSV and
exportRunReportToJSON (src/solver/domainWorkflows.ts:323-402), and the mapping
main.ts applies to a force readout's history before exporting (main.ts:305-315,
368-378).

A history sample is a dict with the keys of TelemetryHistorySample
(domainWorkflows.ts:41-50): step, timeSec, cd, cl and the optional cm, dragForceN,
liftForceN, xcpMeters.  An optional key that is missing or None is JavaScript's
`undefined`: the CSV falls back to the metadata (then 0), the JSON omits it.
Metadata is a dict with SimulationRunMetadata's keys (domainWorkflows.ts:18-39);
missing keys take the CSV's defaults.  Numbers are printed with JavaScript's
toFixed / Number::toString (aerosim_b200.jsfmt), so the text equals the browser's.
"""
from __future__ import annotations

import datetime as _dt
import math
import numbers

from . import jsfmt
from .forces import NEWTONS_TO_KGF, NEWTONS_TO_LBF

CSV_COLUMNS = ("step,time_sec,cd,cl,cm,drag_force_n,drag_force_lbf,drag_force_kgf,lift_force_n,"
               "lift_force_lbf,xcp_meters")
APPLICATION = "AeroSim — 3D WebGPU Wind Tunnel Platform"
VERSION = "0.1.0"
UNITS = {"windSpeed": "m/s", "forces": "Newtons", "pressure": "Pascals", "lengths": "meters",
         "areas": "square_meters"}


def iso_timestamp(now: _dt.datetime | None = None) -> str:
    """Date.prototype.toISOString: UTC, millisecond precision, trailing Z."""
    t = (now or _dt.datetime.now(_dt.timezone.utc)).astimezone(_dt.timezone.utc)
    return t.strftime("%Y-%m-%dT%H:%M:%S.") + f"{t.microsecond // 1000:03d}Z"


def _coalesce(*values):
    """JavaScript `a ?? b ?? c`: the first value that is not None."""
    for v in values:
        if v is not None:
            return v
    return None


def _fixed_or(value, digits: int, default: str) -> str:
    return default if value is None else jsfmt.to_fixed(value, digits)


def export_telemetry_to_csv(history, metadata: dict) -> str:
    """exportTelemetryToCSV(history, metadata), domainWorkflows.ts:323-367: comment header,
    column row, one row per sample, lines joined by CRLF (no trailing newline)."""
    md = metadata or {}
    mesh = md.get("meshStats")
    lines = [
        "# AeroSim Aerodynamic Wind Tunnel Telemetry Export",
        f"# Generated: {_coalesce(md.get('timestamp'), iso_timestamp())}",
        f"# Specimen: {_coalesce(md.get('specimenName'), 'Specimen')}",
        f"# Wind Speed: {_fixed_or(md.get('windSpeedMps'), 1, '0.0')} m/s",
        f"# Reynolds Number: {_fixed_or(md.get('reynolds'), 0, '0')}",
        f"# Frontal Area: {'0' if mesh is None else jsfmt.to_fixed(mesh['frontalArea'], 4)} m2",
        f"# Mean Cd: {_fixed_or(md.get('meanCd'), 4, '0')}",
        f"# Mean Cl: {_fixed_or(md.get('meanCl'), 4, '0')}",
        f"# Pitching Moment Cm: {_fixed_or(md.get('meanCm'), 4, '0')}",
        f"# Center of Pressure X: {_fixed_or(md.get('centerOfPressureX'), 3, '0')} m",
        "",
        CSV_COLUMNS,
    ]
    for s in history:
        cm = _coalesce(s.get("cm"), md.get("meanCm"), 0.0)
        drag = _coalesce(s.get("dragForceN"), md.get("dragForceN"), 0.0)
        lift = _coalesce(s.get("liftForceN"), md.get("liftForceN"), 0.0)
        xcp = _coalesce(s.get("xcpMeters"), md.get("centerOfPressureX"), 0.0)
        lines.append(",".join((
            jsfmt.to_string(s["step"]), jsfmt.to_fixed(s["timeSec"], 4), jsfmt.to_fixed(s["cd"], 5),
            jsfmt.to_fixed(s["cl"], 5), jsfmt.to_fixed(cm, 5), jsfmt.to_fixed(drag, 2),
            jsfmt.to_fixed(drag * NEWTONS_TO_LBF, 2), jsfmt.to_fixed(drag * NEWTONS_TO_KGF, 2),
            jsfmt.to_fixed(lift, 2), jsfmt.to_fixed(lift * NEWTONS_TO_LBF, 2), jsfmt.to_fixed(xcp, 3))))
    return "\r\n".join(lines)


class _Undefined:
    """JavaScript `undefined`: omitted from JSON objects, `null` in arrays."""


UNDEFINED = _Undefined()


def _rounded(v, digits: int):
    return UNDEFINED if v is None else float(jsfmt.to_fixed(v, digits))


def export_run_report_to_json(metadata: dict, history, export_timestamp: str | None = None) -> str:
    """exportRunReportToJSON(metadata, history), domainWorkflows.ts:372-402, as
    JSON.stringify(payload, null, 2) prints it."""
    run = dict(metadata)
    run["units"] = dict(UNITS)
    run["telemetryHistory"] = [{
        "step": s["step"],
        "timeSec": float(jsfmt.to_fixed(s["timeSec"], 4)),
        "cd": float(jsfmt.to_fixed(s["cd"], 5)),
        "cl": float(jsfmt.to_fixed(s["cl"], 5)),
        "cm": _rounded(s.get("cm"), 5),
        "dragForceN": _rounded(s.get("dragForceN"), 2),
        "liftForceN": _rounded(s.get("liftForceN"), 2),
        "xcpMeters": _rounded(s.get("xcpMeters"), 3),
    } for s in history]
    payload = {"application": APPLICATION, "version": VERSION,
               "exportTimestamp": export_timestamp or iso_timestamp(), "simulationRun": run}
    return json_stringify(payload, 2)


def history_from_readout(readout: dict, fluid_density: float, wind_speed: float, frontal_area: float) -> list:
    """The samples main.ts exports from a ForceConvergenceTracker readout (main.ts:305-315):
    time = step x 1 ms, missing forces from Cd / Cl x q A, missing Cm / xcp from the means."""
    q_area = 0.5 * fluid_density * wind_speed * wind_speed * frontal_area
    out = []
    for h in readout["history"]:
        out.append({
            "step": h["step"], "timeSec": h["step"] * 0.001, "cd": h["cd"], "cl": h["cl"],
            "cm": _coalesce(h.get("cm"), readout["pitchingMomentCm"]),
            "dragForceN": _coalesce(h.get("dragForceN"), h["cd"] * q_area),
            "liftForceN": _coalesce(h.get("liftForceN"), h["cl"] * q_area),
            "xcpMeters": _coalesce(h.get("xcp"), readout["centerOfPressureX"]),
        })
    return out


# ---- JSON.stringify ----------------------------------------------------------------

_ESCAPES = {'"': '\\"', "\\": "\\\\", "\b": "\\b", "\f": "\\f", "\n": "\\n", "\r": "\\r", "\t": "\\t"}


def _quote(s: str) -> str:
    out = ['"']
    for ch in s:
        c = ord(ch)
        if ch in _ESCAPES:
            out.append(_ESCAPES[ch])
        elif c < 0x20 or 0xD800 <= c <= 0xDFFF:
            out.append(f"\\u{c:04x}")
        else:
            out.append(ch)
    out.append('"')
    return "".join(out)


def _value(v, indent: str, level: int):
    """Serialized v, or None where JSON.stringify skips the value (undefined)."""
    if v is UNDEFINED:
        return None
    if v is None:
        return "null"
    if v is True:
        return "true"
    if v is False:
        return "false"
    if isinstance(v, numbers.Real):
        return jsfmt.to_string(float(v)) if math.isfinite(v) else "null"
    if isinstance(v, str):
        return _quote(v)
    inner = "\n" + indent * (level + 1)
    outer = "\n" + indent * level
    if isinstance(v, dict):
        items = []
        for k, x in v.items():
            sx = _value(x, indent, level + 1)
            if sx is not None:
                items.append(f"{_quote(str(k))}: {sx}")
        return "{" + inner + ("," + inner).join(items) + outer + "}" if items else "{}"
    if isinstance(v, (list, tuple)):
        if not v:
            return "[]"
        items = [_value(x, indent, level + 1) or "null" for x in v]
        return "[" + inner + ("," + inner).join(items) + outer + "]"
    raise TypeError(f"cannot serialise {type(v).__name__}")


def json_stringify(value, space: int = 2) -> str:
    """JSON.stringify(value, null, space) for dicts, lists, strings, numbers, booleans,
    None (null) and UNDEFINED."""
    out = _value(value, " " * space, 0)
    return "undefined" if out is None else out


exportTelemetryToCSV = export_telemetry_to_csv
exportRunReportToJSON = export_run_report_to_json

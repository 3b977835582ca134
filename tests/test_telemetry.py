"""Telemetry export (src/solver/domainWorkflows.ts:323-402): the reference's CSV / JSON
known answers (phase6.test.ts:180-261), JavaScript number formatting against the
ECMA-262 restatement in oracle/jsnum.py, and the JSON.stringify layout."""
import json
import math
import random
import struct

import pytest

from aerosim_b200 import forces, jsfmt, telemetry

HISTORY = [
    {"step": 100, "timeSec": 0.1, "cd": 0.52, "cl": 0.02, "cm": 0.005, "dragForceN": 155.0, "liftForceN": 6.0,
     "xcpMeters": 0.25},
    {"step": 200, "timeSec": 0.2, "cd": 0.48, "cl": 0.01, "cm": 0.004, "dragForceN": 143.0, "liftForceN": 3.0,
     "xcpMeters": 0.26},
    {"step": 300, "timeSec": 0.3, "cd": 0.47, "cl": 0.00, "cm": 0.002, "dragForceN": 140.0, "liftForceN": 0.0,
     "xcpMeters": 0.26},
]
METADATA = {
    "timestamp": "2026-11-01T12:00:00Z", "specimenName": "Calibration Sphere (1m)", "presetId": "sphere",
    "solverMode": "interactive", "groundPlaneEnabled": False, "windSpeedMps": 25.0,
    "fluid": dict(forces.AIR_20C), "tunnel": {"length": 6.0, "width": 2.8, "height": 2.4},
    "meshStats": {"name": "Calibration Sphere (1m)", "triangleCount": 1024, "vertexCount": 514,
                  "isWatertight": True, "openEdgeCount": 0, "boundingBoxSize": {"x": 1, "y": 1, "z": 1},
                  "characteristicLength": 1.0, "frontalArea": 0.7854, "volume": 0.5236},
    "meanCd": 0.47, "meanCl": 0.005, "meanCm": 0.003, "centerOfPressureX": 0.26, "dragForceN": 140.0,
    "liftForceN": 1.5, "reynolds": 400000, "dynamicPressurePa": 376.25, "blockageRatioPercent": 11.69,
    "totalSteps": 300, "isConverged": True,
}


@pytest.fixture(scope="module")
def jsnum():
    from oracle import jsnum as o
    return o


def test_csv_known_answers():
    """phase6.test.ts:220-244."""
    csv = telemetry.export_telemetry_to_csv(HISTORY, METADATA)
    assert "# AeroSim Aerodynamic Wind Tunnel Telemetry Export" in csv
    assert telemetry.CSV_COLUMNS in csv
    rows = [r for r in csv.split("\r\n") if r.strip() and not r.startswith("#") and not r.startswith("step")]
    assert len(rows) == 3
    step, t, cd, cl, cm, drag, drag_lbf, drag_kgf, lift, lift_lbf, xcp = rows[0].split(",")
    assert int(step) == 100
    assert abs(float(t) - 0.1) < 5e-4 and abs(float(cd) - 0.52) < 5e-3 and abs(float(cl) - 0.02) < 5e-3
    assert abs(float(cm) - 0.005) < 5e-4 and abs(float(drag) - 155.0) < 0.05 and abs(float(lift) - 6.0) < 0.05
    assert float(drag_lbf) > 0 and float(drag_kgf) > 0 and float(lift_lbf) > 0
    assert abs(float(xcp) - 0.25) < 5e-3


def test_csv_exact_text():
    csv = telemetry.export_telemetry_to_csv(HISTORY[:1], METADATA)
    assert csv.split("\r\n") == [
        "# AeroSim Aerodynamic Wind Tunnel Telemetry Export",
        "# Generated: 2026-11-01T12:00:00Z",
        "# Specimen: Calibration Sphere (1m)",
        "# Wind Speed: 25.0 m/s",
        "# Reynolds Number: 400000",
        "# Frontal Area: 0.7854 m2",
        "# Mean Cd: 0.4700",
        "# Mean Cl: 0.0050",
        "# Pitching Moment Cm: 0.0030",
        "# Center of Pressure X: 0.260 m",
        "",
        telemetry.CSV_COLUMNS,
        "100,0.1000,0.52000,0.02000,0.00500,155.00,34.85,15.81,6.00,1.35,0.250",
    ]
    assert not csv.endswith("\r\n")


def test_csv_fallbacks():
    """`sample.x ?? metadata.x ?? 0` and the header defaults."""
    rows = telemetry.export_telemetry_to_csv([{"step": 5, "timeSec": 0.005, "cd": 1.0, "cl": -0.25}],
                                             {"meanCm": -0.0125, "dragForceN": 2.5}).split("\r\n")
    assert rows[2:10] == ["# Specimen: Specimen", "# Wind Speed: 0.0 m/s", "# Reynolds Number: 0",
                          "# Frontal Area: 0 m2", "# Mean Cd: 0", "# Mean Cl: 0", "# Pitching Moment Cm: -0.0125",
                          "# Center of Pressure X: 0 m"]
    assert rows[-1] == "5,0.0050,1.00000,-0.25000,-0.01250,2.50,0.56,0.25,0.00,0.00,0.000"


def test_json_known_answers():
    """phase6.test.ts:246-259."""
    text = telemetry.export_run_report_to_json(METADATA, HISTORY)
    parsed = json.loads(text)
    assert parsed["application"] == "AeroSim — 3D WebGPU Wind Tunnel Platform"
    assert parsed["version"] == "0.1.0"
    run = parsed["simulationRun"]
    assert run["specimenName"] == "Calibration Sphere (1m)"
    assert abs(run["meanCd"] - 0.47) < 5e-3 and run["isConverged"] is True
    assert len(run["telemetryHistory"]) == 3
    assert run["telemetryHistory"][1]["step"] == 200 and abs(run["telemetryHistory"][1]["cd"] - 0.48) < 5e-3
    assert list(run)[-2:] == ["units", "telemetryHistory"] and run["units"]["areas"] == "square_meters"


def test_json_layout_matches_json_stringify():
    """Two-space layout, key order, `undefined` dropped from objects and `null` in arrays,
    NaN as null, integral numbers without a fraction, exponents as JavaScript prints them."""
    hist = [{"step": 1, "timeSec": 0.001, "cd": 0.123456789, "cl": float("nan"), "xcpMeters": 1e21}]
    text = telemetry.export_run_report_to_json({"specimenName": "a\"b\\c\n\u0001é", "empty": {}, "list": [],
                                                "tiny": 1.5e-7, "big": 2.0 ** 70, "arr": [None, 3.0]},
                                               hist, export_timestamp="T")
    assert text == "\n".join([
        "{",
        '  "application": "AeroSim — 3D WebGPU Wind Tunnel Platform",',
        '  "version": "0.1.0",',
        '  "exportTimestamp": "T",',
        '  "simulationRun": {',
        '    "specimenName": "a\\"b\\\\c\\n\\u0001é",',
        '    "empty": {},',
        '    "list": [],',
        '    "tiny": 1.5e-7,',
        '    "big": 1.1805916207174113e+21,',
        '    "arr": [',
        "      null,",
        "      3",
        "    ],",
        '    "units": {',
        '      "windSpeed": "m/s",',
        '      "forces": "Newtons",',
        '      "pressure": "Pascals",',
        '      "lengths": "meters",',
        '      "areas": "square_meters"',
        "    },",
        '    "telemetryHistory": [',
        "      {",
        '        "step": 1,',
        '        "timeSec": 0.001,',
        '        "cd": 0.12346,',
        '        "cl": null,',
        '        "xcpMeters": 1e+21',
        "      }",
        "    ]",
        "  }",
        "}"])
    assert json.loads(text)["simulationRun"]["telemetryHistory"][0]["cd"] == 0.12346


def test_js_number_formatting_known_outputs(jsnum):
    """Outputs of JavaScript's toFixed / String(x) stated by ECMA-262 and its examples."""
    fixed = [(0.125, 2, "0.13"), (1.005, 2, "1.00"), (2.5, 0, "3"), (-2.5, 0, "-3"), (-0.0, 2, "0.00"),
             (1e21, 2, "1e+21"), (0.000001, 7, "0.0000010"), (123.456, 0, "123"), (-0.001, 2, "-0.00"),
             (1.45, 1, "1.4"), (10.235, 2, "10.23"), (1.255, 2, "1.25"), (float("nan"), 2, "NaN")]
    strings = [(1e21, "1e+21"), (1e-7, "1e-7"), (1.23e-18, "1.23e-18"), (0.000001, "0.000001"), (100.0, "100"),
               (-0.0, "0"), (2.0 ** 53, "9007199254740992"), (1.7976931348623157e308, "1.7976931348623157e+308"),
               (5e-324, "5e-324"), (0.1 + 0.2, "0.30000000000000004"), (1e20, "100000000000000000000"),
               (-1.5e-7, "-1.5e-7"), (float("inf"), "Infinity")]
    for x, f, want in fixed:
        assert jsfmt.to_fixed(x, f) == want == jsnum.to_fixed(x, f), (x, f)
    for x, want in strings:
        assert jsfmt.to_string(x) == want == jsnum.to_string(x), x


def test_js_number_formatting_matches_oracle(jsnum):
    rng = random.Random(11)
    values = []
    for _ in range(20000):
        e = rng.uniform(-12, 25)
        values.append(rng.choice((-1, 1)) * rng.random() * 10 ** e)
    for _ in range(3000):  # exact binary ties at the rounding digit
        values.append(rng.randint(-10 ** 6, 10 ** 6) / 8)
    for _ in range(2000):  # random bit patterns, finite
        x = struct.unpack("<d", struct.pack("<Q", rng.getrandbits(64)))[0]
        if math.isfinite(x):
            values.append(x)
    for x in values:
        assert jsfmt.to_string(x) == jsnum.to_string(x), x
        for f in (0, 1, 2, 3, 4, 5):
            if abs(x) < 1e30:
                assert jsfmt.to_fixed(x, f) == jsnum.to_fixed(x, f), (x, f)


def test_tracker_rounds_stability_like_tofixed():
    """Number(x.toFixed(1)) rounds exact binary ties up (97.25 -> 97.3)."""
    assert forces._round_half_up(97.25, 1) == 97.3
    assert forces._round_half_up(0.125, 2) == 0.13


def test_history_from_readout():
    """main.ts:305-315: time = step x 1 ms, forces from the tracker's per-sample values."""
    tr = forces.ForceConvergenceTracker()
    for i in range(5):
        r = tr.push_sample(100 * (i + 1), 0.5 + 0.01 * i, 0.1, 0.02, 0.3, 20.0, forces.AIR_20C, 0.25)
    hist = telemetry.history_from_readout(r, forces.AIR_20C["density"], 20.0, 0.25)
    q_area = 0.5 * forces.AIR_20C["density"] * 20.0 * 20.0 * 0.25
    assert [h["step"] for h in hist] == [100, 200, 300, 400, 500]
    assert hist[2]["timeSec"] == 300 * 0.001 and hist[2]["dragForceN"] == (0.5 + 0.02) * q_area
    assert hist[4]["xcpMeters"] == 0.3 and hist[0]["cm"] == 0.02
    csv = telemetry.export_telemetry_to_csv(hist, {"specimenName": "s"})
    assert csv.split("\r\n")[-1].startswith("500,0.5000,0.54000,0.10000,0.02000,")


def test_tracker_history_matches_a_full_rebuild():
    """The readout history is kept entry by entry (180 samples at most); it equals the
    list built from all samples with the call's q_inf * A_ref, also after q changes."""
    tr = forces.ForceConvergenceTracker()
    rng = random.Random(5)
    for i in range(400):
        u = 20.0 if i < 300 else 25.0
        r = tr.push_sample(4 * i, rng.random(), rng.random() - 0.5, 0.01, 0.3, u, forces.AIR_20C, 0.25)
        q = 0.5 * forces.AIR_20C["density"] * u * u * 0.25
        if i % 37 == 0 or i in (179, 180, 181, 300, 399):
            ref = [{"step": s.step, "cd": s.cd, "cl": s.cl, "cm": s.cm, "xcp": s.xcp,
                    "dragForceN": s.cd * q, "liftForceN": s.cl * q} for s in tr.samples]
            assert r["history"] == ref
    assert len(r["history"]) == 180 and r["history"][0]["step"] == 4 * 220


def test_tracker_means_are_plain_left_to_right_sums():
    """forceIntegrator.ts:355-377 adds the window's samples in order with no compensation:
    1e16 + 1 rounds back to 1e16, so the window {1e16, 1, -1e16} has mean 0, not 1/3."""
    tr = forces.ForceConvergenceTracker()
    for i, cd in enumerate((1e16, 1.0, -1e16)):
        r = tr.push_sample(i, cd, cd, cd, cd, 20.0, forces.AIR_20C, 0.25)
    assert r["meanCd"] == 0.0 and r["meanCl"] == 0.0 and r["pitchingMomentCm"] == 0.0
    assert r["centerOfPressureX"] == 0.0
    # the variance adds diff * diff in the same order: (1e16)^2 + 1 + (1e16)^2 over 3
    var = 0.0
    for cd in (1e16, 1.0, -1e16):
        var += cd * cd
    assert r["stdCd"] == math.sqrt(var / 3)

"""STL reader, normalisation, mesh statistics and the frontal-area raster
(src/geometry/stlLoader.ts, frontalArea.ts:22-179) against the Python oracle
(oracle/stl.py) and the reference's known answers (phase1.test.ts:11-97).

CPU tests run the library's host code (device = -1); the `gpu` tests check the CUDA
raster against the host raster bit for bit."""
import math
import random
import struct

import numpy as np
import pytest

from aerosim_b200 import _native, frontal_area, meshes, stl


@pytest.fixture(scope="module")
def ostl(oracle_mod):
    from oracle import stl as o
    return o


def binary_stl(mesh, header: bytes = b"binary stl", extra: bytes = b"") -> bytes:
    soup = meshes.as_soup(mesh).reshape(-1, 3, 3)
    out = bytearray(header.ljust(80, b" ")[:80])
    out += struct.pack("<I", soup.shape[0])
    for tri in soup:
        out += struct.pack("<3f", 0.0, 0.0, 1.0)
        out += struct.pack("<9f", *tri.reshape(-1).tolist())
        out += b"\0\0"
    return bytes(out) + extra


def ascii_stl(mesh, fmt=repr, sep=" ", name="body") -> bytes:
    soup = meshes.as_soup(mesh).reshape(-1, 3, 3)
    lines = [f"solid {name}"]
    for tri in soup:
        lines.append("  facet normal 0 0 0")
        lines.append("    outer loop")
        for v in tri:
            lines.append("      vertex" + sep + sep.join(fmt(float(c)) for c in v))
        lines.append("    endloop")
        lines.append("  endfacet")
    lines.append(f"endsolid {name}")
    return "\n".join(lines).encode()


def right_tetrahedron() -> bytes:
    """ASCII STL of the tetrahedron with legs 1 along x, y and z (outward facets)."""
    o, x, y, z = (0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)
    facets = [(o, y, x), (o, x, z), (o, z, y), (x, y, z)]
    text = "solid tetra\n"
    for f in facets:
        text += "facet normal 0 0 0\n outer loop\n"
        text += "".join(f"  vertex {a} {b} {c}\n" for a, b, c in f)
        text += " endloop\nendfacet\n"
    return (text + "endsolid tetra\n").encode()


def parse_both(buf, ostl):
    """(library result, oracle result); each an array or the error's class name."""
    try:
        lib = stl.parse_stl(buf)[0]
    except _native.AerosimError as e:
        assert e.code == _native.ERR_FORMAT, e
        lib = "format"
    try:
        orc = ostl.parse_stl(buf)[0]
    except ostl.STLFormatError:
        orc = "format"
    return lib, orc


def assert_same_parse(buf, ostl):
    lib, orc = parse_both(buf, ostl)
    if isinstance(orc, str) or isinstance(lib, str):
        assert lib == orc if isinstance(lib, str) and isinstance(orc, str) else False, (buf[:120], lib, orc)
    else:
        assert lib.shape == orc.shape and lib.tobytes() == orc.tobytes(), buf[:120]


# ---- known answers of the reference (phase1.test.ts) ------------------------------

@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_known_answers(impl, ostl):
    def stats(mesh, rot=(0, 0, 0)):
        if impl == "oracle":
            return ostl.mesh_stats(mesh[0], mesh[1], (0, 0, 0), rot, (1, 1, 1))
        return stl.compute_mesh_stats(mesh, "m", ((0, 0, 0), rot, (1, 1, 1)), device=-1)

    sphere = stats(meshes.uv_sphere(0.5, 96, 64))  # phase1.test.ts:11-20
    assert abs(sphere["frontalArea"] - math.pi * 0.25) / (math.pi * 0.25) < 0.005
    cube = stats(meshes.box(1.0, 1.0, 1.0, 4))  # phase1.test.ts:38-50
    assert cube["isWatertight"] and cube["openEdgeCount"] == 0
    assert round(cube["volume"], 3) == 1.0 and round(cube["frontalArea"], 3) == 1.0
    rotated = stats(meshes.box(1.0, 1.0, 1.0, 4), (0, 45, 0))  # phase1.test.ts:30-36
    assert abs(rotated["frontalArea"] - math.sqrt(2)) / math.sqrt(2) < 0.005
    # phase1.test.ts:52-97: ASCII right tetrahedron
    buf = right_tetrahedron()
    pos = ostl.parse_stl(buf)[0] if impl == "oracle" else stl.parse_stl(buf)[0]
    tet = stats((pos, None))
    assert tet["triangleCount"] == 4 and tet["isWatertight"]
    assert abs(tet["volume"] - 1 / 6) < 5e-5
    assert abs(tet["frontalArea"] - 0.5) < 5e-3


# ---- parser parity ------------------------------------------------------------------

def test_parse_binary_and_ascii_match_oracle(ostl):
    sphere = meshes.uv_sphere(0.5, 24, 16)
    wing = meshes.naca0012_wing(1.0, 2.0, 6.0)
    cases = [binary_stl(sphere), binary_stl(wing, header=b"solid but binary"),
             binary_stl(sphere, extra=b"\0" * 17),  # trailing bytes: the fit-in-buffer fallback
             ascii_stl(sphere), ascii_stl(wing, fmt=lambda c: f"{c:.6e}"),
             ascii_stl(sphere, fmt=lambda c: f"{c:+.9f}", sep="\t"),
             ascii_stl(wing, fmt=lambda c: f"{c:.3E}", sep=" \r\n "),
             "\ufeff  \n".encode() + ascii_stl(sphere),
             ascii_stl(sphere).replace(b"vertex ", b"vertex\xc2\xa0"),  # U+00A0 is \s in JavaScript
             ascii_stl(sphere).replace(b"vertex ", b"vertex\xe2\x80\x83")]  # U+2003
    for buf in cases:
        assert_same_parse(buf, ostl)
    assert stl.stl_format(cases[0]) == "binary" and stl.stl_format(cases[1]) == "binary"
    assert stl.stl_format(cases[2]) == "binary" and stl.stl_format(cases[3]) == "ascii"
    ref = meshes.as_soup(sphere)
    assert stl.parse_stl(cases[0])[0].tobytes() == ref.tobytes()
    assert stl.parse_stl(cases[3])[0].tobytes() == ref.tobytes()


def test_parse_errors_and_number_forms(ostl):
    tri = b"facet outer loop vertex 0 0 0 vertex 1 0 0 vertex 0 1 0 endloop endfacet "
    cases = [b"", b"solid x\nendsolid x\n", b"solid x facet vertex 1 2\n" + b" " * 90,
             b"solid " + tri * 2 + b"vertex 1 2 3",  # 21 numbers: not a multiple of 9
             b"SoLiD x " + tri,
             b"x" * 83,
             b"\x00" * 80 + struct.pack("<I", 5) + b"\x00" * 10,  # facets do not fit
             b"solid nothing here" + b"." * 200]
    for buf in cases:
        assert_same_parse(buf, ostl)
    with pytest.raises(_native.AerosimError) as e:
        stl.parse_stl(b"")
    assert e.value.code == _native.ERR_FORMAT and "no valid triangles" in str(e.value)
    with pytest.raises(_native.AerosimError) as e:
        stl.parse_stl(b"\x00" * 80 + struct.pack("<I", 5) + b"\x00" * 10)
    assert "Invalid or corrupted STL file." in str(e.value)


def test_parse_fuzzed_vertex_lines(ostl):
    """Random vertex lines built from awkward number forms: the library's matcher and the
    reference's regular expression accept and reject the same ones."""
    rng = random.Random(7)
    good = ["1", "-2", "+3", "0.5", ".5", "-.25", "2E-3", "+1e+2", "007", "-0", "3e38", "1e40", "1e-50",
            "4.0e-7", "6.02E23", "0.1", "16777217", "1.00000005960464477539"]
    bad = ["1.", "12.e5", "1e", "1e+", "1.5.3", "0x10", "..5", "+-1", "inf", "1,5"]
    spaces = [" ", "  ", "\t", "\r\n", "", "\u00a0", "\u2028", "\u3000", "\u0085", "\x1c", "\u200b"]
    accepted = 0
    for _ in range(400):
        lines = []
        for _ in range(3 * rng.randint(1, 4)):
            parts = ["vertex" if rng.random() < 0.97 else "vertexx"]
            for _ in range(3):
                parts.append(rng.choice(spaces) if rng.random() < 0.1 else " ")
                parts.append(rng.choice(good) if rng.random() < 0.95 else rng.choice(bad))
            lines.append("".join(parts))
        text = "solid f\nfacet\n" + "\n".join(lines) + "\nendsolid\n"
        accepted += not isinstance(parse_both(text.encode(), ostl)[1], str)
        assert_same_parse(text.encode(), ostl)
    assert accepted > 100


# ---- normalisation and statistics parity -----------------------------------------

@pytest.mark.parametrize("scale", [1.0, 7.5, 30.0, 250.0])
def test_normalize_matches_oracle(scale, ostl):
    pos, idx = meshes.perturbed_ellipsoid((40.0, 16.0, 12.0), seed=2, subdivisions=3)
    pos = (pos.astype(np.float64) * (scale / 40.0) + np.array([3.25, -1.5, 0.75]) * scale).astype(np.float32)
    (out, _), scaled = stl.normalize_and_center_geometry((pos, idx))
    ref, ref_scaled = ostl.normalize_and_center(pos)
    assert scaled == ref_scaled == (2 * scale > 10.0)
    assert out.tobytes() == ref.tobytes()
    if scaled:
        span = out.max(axis=0) - out.min(axis=0)
        assert span.max() <= 1.0 + 1e-6


def _open_box():
    pos, idx = meshes.box(1.0, 0.5, 0.25, 3)
    return pos, np.ascontiguousarray(idx[:-2])


STATS_CASES = {
    "box": (lambda: meshes.box(1.0, 1.0, 1.0, 4), ((0, 0, 0), (0, 0, 0), (1, 1, 1))),
    "box_rotated": (lambda: meshes.box(1.0, 0.6, 0.3, 2), ((0.5, -1, 2), (10, 35, -20), (1.5, 1, 0.5))),
    "sphere": (lambda: meshes.uv_sphere(0.5, 96, 64), ((0, 0.1, 0), (0, 0, 15), (1, 1, 1))),
    "wing_soup": (lambda: (meshes.as_soup(meshes.naca0012_wing(1.0, 2.0, 8.0)), None),
                  ((0, 0, 0), (-5, 0, 0), (2, 2, 2))),
    "open_box": (_open_box, ((0, 0, 0), (0, 90, 0), (1, 1, 1))),
}


@pytest.mark.parametrize("name", list(STATS_CASES))
def test_mesh_stats_match_oracle(name, ostl):
    make, (p, r, s) = STATS_CASES[name]
    pos, idx = make()
    got = stl.compute_mesh_stats((pos, idx), name, (p, r, s), device=-1)
    ref = ostl.mesh_stats(pos, idx, p, r, s)
    for k, v in ref.items():
        assert got[k] == v, (k, got[k], v)
    assert np.array_equal(stl.model_matrix((p, r, s)), np.asarray(ostl.model_matrix(p, r, s)))
    if name == "open_box":
        assert not got["isWatertight"] and got["openEdgeCount"] > 0
    else:
        assert got["isWatertight"]


def test_mesh_stats_skip_edges_above_100k_triangles():
    """computeMeshStats only checks watertightness up to 100 000 triangles."""
    rng = np.random.default_rng(3)
    soup = rng.random((100001 * 3, 3), dtype=np.float32)
    s = stl.compute_mesh_stats((soup, None), "noise", None, device=-1)
    assert s["triangleCount"] == 100001 and s["openEdgeCount"] == 0 and s["isWatertight"]
    s = stl.compute_mesh_stats((soup[:300], None), "noise", None, device=-1)
    assert s["openEdgeCount"] == 300 and not s["isWatertight"]


# ---- CUDA raster -------------------------------------------------------------------

RASTER_CASES = [
    (lambda: meshes.uv_sphere(0.5, 96, 64), None, 512),
    (lambda: meshes.box(1.0, 1.0, 1.0, 4), "rot_y45", 512),
    (lambda: meshes.naca0012_wing(1.0, 2.0, 8.0), "general", 300),
    (lambda: meshes.perturbed_ellipsoid((40.0, 16.0, 12.0), seed=0, subdivisions=5), None, 1024),
    (lambda: (meshes.as_soup(meshes.cylinder(0.3, 1.0, 40, 3, axis=0)), None), "general", 97),
]


def _world(kind):
    if kind is None:
        return None
    if kind == "rot_y45":
        return stl.model_matrix(((0, 0, 0), (0, 45, 0), (1, 1, 1)))
    return stl.model_matrix(((0.2, -0.4, 1.0), (12, -30, 55), (1.2, 0.8, 1.1)))


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(RASTER_CASES)))
def test_frontal_area_cuda_equals_host(case, gpu_engine_cls, oracle_mod):
    make, kind, res = RASTER_CASES[case]
    mesh = make()
    w = _world(kind)
    host = frontal_area(mesh, w, res)
    dev = stl.frontal_area_cuda(mesh, w, res, device=0)
    assert dev == host
    assert dev == oracle_mod.frontal_area(mesh, w, res)


@pytest.mark.gpu
def test_mesh_stats_on_gpu_equal_host(gpu_engine_cls):
    for name, (make, t) in STATS_CASES.items():
        mesh = make()
        assert stl.compute_mesh_stats(mesh, name, t, device=0) == stl.compute_mesh_stats(mesh, name, t, device=-1)


@pytest.mark.gpu
def test_frontal_area_cuda_degenerate_and_errors(gpu_engine_cls):
    flat = (np.array([[0, 0, 0], [0, 1, 0], [0, 2, 0]], dtype=np.float32), None)  # zero z extent
    assert stl.frontal_area_cuda(flat) == 0.0 == frontal_area(flat)
    assert stl.frontal_area_cuda((np.zeros((2, 3), np.float32), None)) == 0.0
    pos, idx = meshes.box(1.0, 1.0, 1.0, 1)
    bad = idx.copy()
    bad[3, 1] = pos.shape[0]
    with pytest.raises(_native.AerosimError) as e:
        stl.frontal_area_cuda((pos, bad))
    assert e.value.code == _native.ERR_ARG
    with pytest.raises(_native.AerosimError):
        stl.frontal_area_cuda((pos, idx), grid_resolution=0)

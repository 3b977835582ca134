"""The C-ABI library loads on a CPU-only machine and exports every entry point
declared in include/aerosim.h (no compute calls are made here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aerosim.h")


def declared_functions(path=HEADER):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(aerosim_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("aerosim_create", "aerosim_destroy", "aerosim_voxelize", "aerosim_set_voxel_grid",
                     "aerosim_step", "aerosim_read_forces", "aerosim_read_macro"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from aerosim_b200 import _native
    lib = _native.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} not exported"
    assert lib.aerosim_abi_version() == 1


def test_bindings_cover_header():
    from aerosim_b200 import _native
    assert set(declared_functions()) == set(_native.SIGNATURES)


def test_create_without_gpu_reports_error():
    """Without a usable device, aerosim_create fails with a status, not a crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from aerosim_b200 import _native
    lib = _native.load()
    h = ctypes.c_void_p()
    rc = lib.aerosim_create(0, ctypes.byref(h))
    assert rc != 0 and not h.value
    assert lib.aerosim_last_error(None)


def test_frontal_area_host_function_matches_oracle(oracle_mod):
    """aerosim_frontal_area is host code: comparable to the oracle without a GPU."""
    from aerosim_b200 import frontal_area, meshes
    for mesh in (meshes.uv_sphere(0.5, 96, 64), meshes.box(1.0, 1.0, 1.0, 4), meshes.naca0012_wing(1.0, 2.0, 8.0)):
        assert frontal_area(mesh) == oracle_mod.frontal_area(mesh)

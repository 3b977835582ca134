"""The allocation-free force reduction, aerosim_momentum_exchange_noalloc.

Callers that cannot allocate device memory themselves (hosts whose allocator owns all
of it, frame loops that cannot afford cudaMalloc's synchronisation) pass device buffers
they already hold.  Here those buffers are torch tensors; the result must match the
engine's own force readout (aerosim_read_forces) and the oracle's momentum exchange on
the same populations, on two calls in a row (the scratch array is shared and keeps the
previous call's contents), and the calls must leave the device's free memory unchanged.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _engine_state(gpu_engine_cls, oracle_mod):
    from aerosim_b200 import VoxelGridResult, cases
    case = cases.sphere_64x32x32()
    vox = oracle_mod.voxelize(case.mesh, None, float(case.ny), case.nx, case.ny, case.nz)
    n = vox.nx * vox.ny * vox.nz
    voxel = VoxelGridResult(vox.nx, vox.ny, vox.nz, vox.dx, vox.dx, vox.dx, *vox.origin, vox.flags, vox.bmap,
                            vox.bcells, vox.q, vox.minq, vox.solid, vox.boundary_count,
                            n - vox.solid - vox.boundary_count, vox.ms)
    eng = gpu_engine_cls(0)
    eng.set_voxel_grid(voxel, {"uInletLattice": case.u_inlet, "nuLattice": case.nu, "smagorinskyCs": case.cs,
                               "precision": "f32_mirror"})
    eng.step(200)
    return vox, eng


def _call(lib, f_d, flags_d, cells_d, q_d, vox, out_d, stream):
    return lib.aerosim_momentum_exchange_noalloc(
        C.c_void_p(f_d.data_ptr()), C.c_void_p(flags_d.data_ptr()), C.c_void_p(cells_d.data_ptr()),
        C.c_void_p(q_d.data_ptr()), vox.boundary_count, vox.nx, vox.ny, vox.nz, C.c_void_p(out_d.data_ptr()),
        C.c_void_p(stream))


def test_noalloc_matches_engine_readout_twice(gpu_engine_cls, oracle_mod):
    import torch
    from aerosim_b200 import _native as N
    lib = N.load()
    vox, eng = _engine_state(gpu_engine_cls, oracle_mod)
    ref = eng.read_forces()
    f = eng.read_populations()
    orc = oracle_mod.momentum_exchange(vox, f)
    dev = torch.device("cuda:0")
    f_d = torch.from_numpy(f).to(dev)
    flags_d = torch.from_numpy(vox.flags).to(dev)
    cells_d = torch.from_numpy(vox.bcells).to(dev)
    q_d = torch.from_numpy(vox.q).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        out_d = torch.full((8,), float("nan"), dtype=torch.float64, device=dev)
        rc = _call(lib, f_d, flags_d, cells_d, q_d, vox, out_d, stream)
        assert rc == 0, lib.aerosim_last_error(None).decode()
        torch.cuda.synchronize(dev)
        out = out_d.cpu().numpy()
        for k, name in enumerate(("fx", "fy", "fz", "mx", "my", "mz")):
            assert math.isclose(out[k], getattr(ref, name), rel_tol=1e-12, abs_tol=1e-15), name
            assert math.isclose(out[k], orc[name], rel_tol=1e-12, abs_tol=1e-15), name
        assert int(out[6]) == ref.cut_face_links == orc["cut"]
        assert int(out[7]) == (vox.boundary_count + 255) // 256
    eng.close()


def test_noalloc_calls_allocate_no_device_memory(gpu_engine_cls, oracle_mod):
    """After a first call (which loads the kernel's module on the device), further calls
    leave the device's free memory exactly as it was."""
    import torch
    from aerosim_b200 import _native as N
    lib = N.load()
    vox, eng = _engine_state(gpu_engine_cls, oracle_mod)
    f = eng.read_populations()
    eng.close()
    dev = torch.device("cuda:0")
    f_d = torch.from_numpy(f).to(dev)
    flags_d = torch.from_numpy(vox.flags).to(dev)
    cells_d = torch.from_numpy(vox.bcells).to(dev)
    q_d = torch.from_numpy(vox.q).to(dev)
    outs = [torch.zeros(8, dtype=torch.float64, device=dev) for _ in range(4)]
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert _call(lib, f_d, flags_d, cells_d, q_d, vox, outs[0], stream) == 0
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    for o in outs[1:]:
        assert _call(lib, f_d, flags_d, cells_d, q_d, vox, o, stream) == 0
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    for o in outs[1:]:
        assert torch.equal(o, outs[0])


def test_noalloc_rejects_oversized_input(gpu_engine_cls):
    import torch
    from aerosim_b200 import _native as N
    lib = N.load()
    dev = torch.device("cuda:0")
    dummy = torch.zeros(16, dtype=torch.float32, device=dev)
    out_d = torch.zeros(8, dtype=torch.float64, device=dev)
    too_many = 4096 * 256 + 1
    rc = lib.aerosim_momentum_exchange_noalloc(C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                               C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
                                               too_many, 64, 32, 32, C.c_void_p(out_d.data_ptr()), None)
    assert rc == N.ERR_ARG
    assert b"exceeds the maximum" in lib.aerosim_last_error(None)

"""Learned subgrid-scale closure: host side of the MLP that replaces the Smagorinsky
eddy viscosity (csrc/sgs_mlp.cuh, csrc/sgs.cu).

  x (8)  = 100 * strain rate (xx yy zz xy xz yz), 100 * (rho - 1), wall distance / 16
  nu_t / nu_0 = softplus(W3 GELU(W2 GELU(W1 x + b1) + b2) + b3)

Training, gradients and both forward passes run in libaerosim.so on the GPU; this
module holds the parameter vector (FP32, layout W1[32][8], b1, W2[32][32], b2, W3[32],
b3), the sample extraction from a fine / coarse engine pair and the Smagorinsky
baseline the closure is judged against.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

N_IN, N_HID = 8, 32


def param_count() -> int:
    return int(N.load().aerosim_mlp_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases, output bias so that softplus(b3) = 1."""
    rng = np.random.default_rng(seed)

    def glorot(o, i):
        a = np.sqrt(6.0 / (i + o))
        return rng.uniform(-a, a, (o, i))

    p = np.concatenate([glorot(N_HID, N_IN).ravel(), np.zeros(N_HID), glorot(N_HID, N_HID).ravel(), np.zeros(N_HID),
                        glorot(1, N_HID).ravel(), [np.log(np.expm1(1.0))]]).astype(np.float32)
    assert p.size == param_count()
    return p


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def forward(params, X, tensor_cores: bool | str = False) -> np.ndarray:
    """nu_t / nu_0 for rows of X[n][8] on the GPU: FP32 CUDA cores (False), the step
    kernel's warp-level BF16 tensor-core path (True), or 128-row tiles on the
    5th-generation tensor cores with accumulators in tensor memory ("tcgen05")."""
    p, x = _f32(params), _f32(X).reshape(-1, N_IN)
    out = np.empty(x.shape[0], np.float32)
    lib = N.load()
    fn = (lib.aerosim_mlp_forward_umma if tensor_cores == "tcgen05" else
          lib.aerosim_mlp_forward_tc if tensor_cores else lib.aerosim_mlp_forward)
    N.check(fn(N.ptr(p, C.c_float), N.ptr(x, C.c_float), x.shape[0], N.ptr(out, C.c_float)))
    return out


def last_forward_ms() -> float:
    """Device time of the kernel of the last tensor-core forward call."""
    ms = C.c_double()
    N.check(N.load().aerosim_mlp_last_timing(C.byref(ms)))
    return ms.value


def gradients(params, X, Y) -> tuple[np.ndarray, float]:
    """(gradient, loss) of the mean squared error on the GPU."""
    p, x, y = _f32(params), _f32(X).reshape(-1, N_IN), _f32(Y).ravel()
    g = np.empty_like(p)
    loss = C.c_double()
    N.check(N.load().aerosim_mlp_gradients(N.ptr(p, C.c_float), N.ptr(x, C.c_float), N.ptr(y, C.c_float),
                                           x.shape[0], N.ptr(g, C.c_float), C.byref(loss)))
    return g, loss.value


def train(params, X, Y, iters: int = 2000, batch: int = 8192, lr: float = 2e-3, seed: int = 0):
    """Adam on the GPU; returns (trained parameters, mini-batch loss curve)."""
    p, x, y = _f32(params).copy(), _f32(X).reshape(-1, N_IN), _f32(Y).ravel()
    curve = np.empty(iters, np.float32)
    N.check(N.load().aerosim_mlp_train(N.ptr(p, C.c_float), N.ptr(x, C.c_float), N.ptr(y, C.c_float), x.shape[0],
                                       int(iters), int(batch), float(lr), int(seed), N.ptr(curve, C.c_float)))
    return p, curve


def samples(fine, coarse, max_ratio: float = 50.0, average_radius: int = 0, min_ratio: float = 0.0):
    """(X, Y) of the valid coarse cells from the flow of engine `fine` box-filtered onto
    engine `coarse` (a lattice exactly half as fine); the eddy-viscosity target is the
    least-squares fit over each cell's (2 average_radius + 1)^3 neighbourhood, clipped to
    [min_ratio, max_ratio] x nu_0 (a negative min_ratio keeps backscatter)."""
    n = coarse.voxel_info().nx * coarse.voxel_info().ny * coarse.voxel_info().nz
    X = np.empty((n, N_IN), np.float32)
    Y = np.empty(n, np.float32)
    V = np.empty(n, np.uint8)
    N.check(N.load().aerosim_sgs_samples(fine._h.h, coarse._h.h, float(min_ratio), float(max_ratio),
                                         int(average_radius),
                                         N.ptr(X, C.c_float),
                                         N.ptr(Y, C.c_float), N.ptr(V, C.c_uint8)))
    ok = V != 0
    return X[ok], Y[ok]


def smagorinsky_ratio(X, nu0: float, cs: float = 0.1) -> np.ndarray:
    """The Smagorinsky eddy viscosity (filter width one coarse cell) of the samples'
    strain rates, as nu_t / nu_0: (Cs)^2 sqrt(2 S:S) / nu_0."""
    s = np.asarray(X, np.float64)[:, :6] / 100.0
    ss = s[:, 0] ** 2 + s[:, 1] ** 2 + s[:, 2] ** 2 + 2.0 * (s[:, 3] ** 2 + s[:, 4] ** 2 + s[:, 5] ** 2)
    return cs * cs * np.sqrt(2.0 * ss) / nu0

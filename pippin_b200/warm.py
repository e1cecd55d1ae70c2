"""The learned Newton warm start: its network and the data it learns from.

The network (24 contact features -> 128 -> 128 -> 128 -> 3 frame forces,
ReLU) runs on the tensor cores in BF16 with FP32 accumulation and trains with
this library's own FP32 kernels (`pg_mlp_*`, include/pippin_b200_mlp.h).
The reference has no learned warm start: it warm-starts Newton from the
previous step's acceleration behind a cost gate
(crates/pippin/src/newton.rs:238-245), and that gate stays in front of the
learned guess, so a poor prediction costs nothing but its own evaluation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

WEIGHTS = 36662
PARAMS = 36611
N_IN, N_OUT = 24, 3


class MlpError(RuntimeError):
    pass


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        raise MlpError(f"expected shape {shape}, got {a.shape}")
    return a


def _pf(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc):
    if rc != 0:
        raise MlpError(_native.last_error() or f"pippin_b200 error {rc}")


def forward(weights, X) -> np.ndarray:
    """Frame forces (n, 3) for features (n, 24), tensor-core inference."""
    L = _native.load()
    w = _f32(weights, (WEIGHTS,))
    X = _f32(X)
    n = X.shape[0]
    Y = np.zeros((n, N_OUT), np.float32)
    _check(L.pg_mlp_forward(_pf(w), w.size, _pf(X), n, _pf(Y)))
    return Y


def loss_grad(weights, X, Y):
    """(mean squared error of the normalised output, gradient (36611,))."""
    L = _native.load()
    w = _f32(weights, (WEIGHTS,))
    X, Y = _f32(X), _f32(Y)
    g = np.zeros(PARAMS, np.float32)
    loss = C.c_double()
    _check(L.pg_mlp_loss_grad(_pf(w), w.size, _pf(X), _pf(Y), X.shape[0], _pf(g), g.size, C.byref(loss)))
    return loss.value, g


def train(X, Y, epochs=20, batch=4096, lr=1e-3, seed=0):
    """Fit a network to (X (n, 24), Y (n, 3)); returns (weights, epoch losses)."""
    L = _native.load()
    X, Y = _f32(X), _f32(Y)
    w = np.zeros(WEIGHTS, np.float32)
    losses = np.zeros(max(epochs, 1), np.float64)
    _check(L.pg_mlp_train(_pf(X), _pf(Y), X.shape[0], int(epochs), int(batch), float(lr), int(seed), _pf(w), w.size,
                          losses.ctypes.data_as(C.POINTER(C.c_double))))
    return w, losses[:epochs]


def collect(phys, steps, controls=None, skip=0):
    """Step `phys` (all envs) `steps` substeps, gathering (features, frame
    forces) of the touching contacts after the first `skip` substeps.
    controls(t) returns the (envs, nu) controls of substep t, or None."""
    from .physics import Field
    n = phys.num_envs()
    xs, fs = [], []
    for t in range(steps):
        if controls is not None:
            phys.set(Field.CTRL, range(n), controls(t))
        if t < skip:
            phys.step(range(n), 1)
            continue
        X, F = phys.warm_samples(range(n))
        xs.append(X)
        fs.append(F)
    if not xs:
        return np.zeros((0, N_IN), np.float32), np.zeros((0, N_OUT), np.float32)
    return np.concatenate(xs), np.concatenate(fs)

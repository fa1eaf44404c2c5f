"""Learned scatter surrogate: weights files and a thin wrapper over the C ABI
(irlcu_sur_* in include/irlcu.h).

The network maps a view's rotated activity, attenuation and depth (pooled to
32^3 x 3, BF16) to the view's ESSE scatter projection (128 x 128).  Training
and inference run on the library's own kernels; this module only moves
pointers and files.

Weights file: b"IRLSUR01", uint32 parameter count, float32 parameters
(little-endian), the layout IrlSetScatterSurrogate reads.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

MAGIC = b"IRLSUR01"
HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "sur128.bin")
# the same network trained on the 256^3 / 128-view phantoms (inputs pooled
# 8 x 8 x 8, output interpolated to 256 x 256)
WEIGHTS_256 = os.path.join(HERE, "sur256.bin")
INPUT_SHAPE = (32, 32, 32, 3)
OUTPUT_SIZE = 128 * 128
MODEL_SRF = 7  # projector bits: attenuation 1 | DRF 2 | scatter 4


def save_weights(path: str, w: np.ndarray) -> None:
    w = np.ascontiguousarray(w, dtype="<f4")
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", w.size))
        f.write(w.tobytes())


def load_weights(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path} is not a surrogate weights file")
        (n,) = struct.unpack("<I", f.read(4))
        w = np.frombuffer(f.read(4 * n), dtype="<f4")
    if w.size != n:
        raise ValueError(f"{path} is truncated")
    return w.astype(np.float32)


class Network:
    """One network instance on the current device (irlcu_sur_create)."""

    def __init__(self, lib, max_batch: int, seed: int = 1):
        self.lib = lib
        self.ptr = C.c_void_p()
        self._check(lib.irlcu_sur_create(max_batch, seed, C.byref(self.ptr)))
        self.max_batch = max_batch
        self.nparams = int(lib.irlcu_sur_nparams(self.ptr))

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.irlcu_error_string().decode())

    def close(self):
        if self.ptr:
            self.lib.irlcu_sur_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def get_weights(self) -> np.ndarray:
        w = np.empty(self.nparams, np.float32)
        self._check(self.lib.irlcu_sur_get_weights(self.ptr, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.lib.irlcu_sur_set_weights(self.ptr, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))

    # device pointers (ints) of BF16 inputs and FP32 outputs / targets
    def forward(self, batch: int, x_ptr: int, y_ptr: int) -> None:
        self._check(self.lib.irlcu_sur_forward(self.ptr, batch, x_ptr, y_ptr))

    def gradient(self, batch: int, x_ptr: int, t_ptr: int):
        loss = C.c_float()
        g = np.empty(self.nparams, np.float32)
        self._check(self.lib.irlcu_sur_gradient(self.ptr, batch, x_ptr, t_ptr, C.byref(loss),
                                                g.ctypes.data_as(C.POINTER(C.c_float))))
        return float(loss.value), g

    def train_step(self, batch: int, x_ptr: int, t_ptr: int, lr: float) -> float:
        loss = C.c_float()
        self._check(self.lib.irlcu_sur_train_step(self.ptr, batch, x_ptr, t_ptr, lr, C.byref(loss)))
        return float(loss.value)


def layer_specs():
    """(ci, co, kd, stride, relu, upsample) per layer, in parameter order."""
    return [(3, 32, 3, 1, True, False), (32, 32, 3, 2, True, False), (32, 64, 3, 2, True, False),
            (512, 256, 1, 1, True, True), (256, 128, 1, 1, True, True), (128, 64, 1, 1, True, True),
            (64, 32, 1, 1, True, True), (32, 1, 1, 1, False, False)]


def split_params(w: np.ndarray):
    """[(weights [co][kd][3][3][ci], bias [co]), ...] views of a parameter vector."""
    out, off = [], 0
    for ci, co, kd, _, _, _ in layer_specs():
        k = kd * 9 * ci
        wt = w[off:off + k * co].reshape(co, kd, 3, 3, ci)
        off += k * co
        b = w[off:off + co]
        off += co
        out.append((wt, b))
    assert off == w.size
    return out

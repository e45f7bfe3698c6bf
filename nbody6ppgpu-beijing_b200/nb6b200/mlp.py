"""ctypes front end of the learned neighbour-radius model (libnb6b200's
nb6_mlp_* extension calls; the reference has no learned component).

The model proposes dlog = log(RS_next / RS) for a particle from five features
of its regular step (see ``features``).  It is trained on the GPU by the
library's own kernels on (features, target) samples logged from plain
Ahmad-Cohen runs (``nb6b200.drive.run(..., mlp_mode=1)``), and once enabled
its bf16 inference runs inside every regular-force call's epilogue.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load_cdll

_f = C.POINTER(C.c_float)
_d = C.POINTER(C.c_double)


def _lib():
    lib = load_cdll()
    lib.nb6_mlp_size_.restype = C.c_int
    return lib


def size() -> int:
    return int(_lib().nb6_mlp_size_())


def init(seed: int = 0) -> None:
    _lib().nb6_mlp_init_(C.byref(C.c_int(seed)))


def set_model(model) -> None:
    m = np.ascontiguousarray(model, dtype=np.float32)
    assert m.shape == (size(),)
    _lib().nb6_mlp_set_(m.ctypes.data_as(_f))


def get_model() -> np.ndarray:
    m = np.zeros(size(), dtype=np.float32)
    _lib().nb6_mlp_get_(m.ctypes.data_as(_f))
    return m


def _xy(x, y=None):
    x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 5)
    if y is not None:
        y = np.ascontiguousarray(y, dtype=np.float32).reshape(-1)
        assert y.shape[0] == x.shape[0]
    return x, y


def grad(x, y):
    """(gradient, loss) of the mean squared error over (x, y) at the current
    parameters (the bf16 values the forward pass uses)."""
    x, y = _xy(x, y)
    g = np.zeros(size() - 12, dtype=np.float32)
    loss = C.c_float(0)
    _lib().nb6_mlp_grad_(C.byref(C.c_int(x.shape[0])), x.ctypes.data_as(_f), y.ctypes.data_as(_f),
                         g.ctypes.data_as(_f), C.byref(loss))
    return g, float(loss.value)


def train(x, y, epochs=10, batch=1024, lr=1e-3, seed=0) -> np.ndarray:
    """Adam on the GPU; returns the mean training loss of each epoch."""
    x, y = _xy(x, y)
    hist = np.zeros(max(epochs, 1), dtype=np.float32)
    _lib().nb6_mlp_train_(C.byref(C.c_int(x.shape[0])), x.ctypes.data_as(_f), y.ctypes.data_as(_f),
                          C.byref(C.c_int(epochs)), C.byref(C.c_int(batch)), C.byref(C.c_float(lr)),
                          C.byref(C.c_int(seed)), hist.ctypes.data_as(_f))
    return hist[:epochs]


def predict(x) -> np.ndarray:
    x, _ = _xy(x)
    y = np.zeros(x.shape[0], dtype=np.float32)
    _lib().nb6_mlp_predict_(C.byref(C.c_int(x.shape[0])), x.ctypes.data_as(_f), y.ctypes.data_as(_f))
    return y


def enable(flag: bool) -> None:
    _lib().nb6_mlp_enable_(C.byref(C.c_int(1 if flag else 0)))


def proposals(ni: int) -> np.ndarray:
    """dlog RS proposed in the last regular-force call, per active particle."""
    out = np.zeros(ni)
    _lib().nb6_regf_proposals_(C.byref(C.c_int(ni)), out.ctypes.data_as(_d))
    return out


def features(nnb, h2, a2, dtr) -> np.ndarray:
    """Model inputs as the CUDA epilogue forms them (mlp.cuh): log(1+nnb)
    (self included), log RS, log(1+nnb) - 1.5 log h2, log|a_reg|, -log2 dtr."""
    n = np.abs(np.asarray(nnb, dtype=np.float64))
    ln = np.log(1.0 + n)
    lh = np.log(np.maximum(np.asarray(h2, dtype=np.float64), 1e-300))
    return np.stack([ln, 0.5 * lh, ln - 1.5 * lh,
                     0.5 * np.log(np.maximum(np.asarray(a2, dtype=np.float64), 1e-300)),
                     -np.log2(np.maximum(np.asarray(dtr, dtype=np.float64), 1e-300))],
                    axis=-1).astype(np.float32)

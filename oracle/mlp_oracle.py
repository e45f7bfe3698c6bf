"""FP64 CPU restatement of the learned neighbour-radius model (test
infrastructure only: the checker for the CUDA training and inference kernels,
never part of the product).

The model is this package's own (the reference has no learned component):
5 -> 64 -> 64 -> 1, SiLU hidden units, parameters used in bf16, inputs
standardised with stored moments; loss = mean squared error in standardised
units.  Parameter layout (flat float vector, then the moments in_mean[5],
in_scale[5], out_mean, out_std):
    W1[k][r] (5 x 64), b1[64], W2[k][r] (64 x 64), b2[64], W3[64], b3
where W[k][r] connects input unit k to output unit r.

``grad`` evaluates the forward pass with the bf16-rounded parameters (as the
GPU does) and differentiates with respect to those parameters, in float64.
"""
from __future__ import annotations

import numpy as np

IN, H = 5, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + IN * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1
NNORM = 2 * IN + 2


def bf16_round(a) -> np.ndarray:
    """float32 -> nearest bf16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def split(w64):
    """Views of a float64 parameter vector: W1, b1, W2, b2, W3, b3."""
    return (w64[OFF_W1:OFF_B1].reshape(IN, H), w64[OFF_B1:OFF_W2], w64[OFF_W2:OFF_B2].reshape(H, H),
            w64[OFF_B2:OFF_W3], w64[OFF_W3:OFF_B3], w64[OFF_B3])


def params_used(model):
    """The parameters every forward pass uses (bf16-rounded), as float64,
    and the moments."""
    w = bf16_round(np.asarray(model[:NPARAM], dtype=np.float32)).astype(np.float64)
    nm = np.asarray(model[NPARAM:NPARAM + NNORM], dtype=np.float32).astype(np.float64)
    return w, nm


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward64(w, nm, x):
    """Standardised outputs and the activations for float64 parameters w."""
    W1, b1, W2, b2, W3, b3 = split(w)
    xf = np.asarray(x, dtype=np.float32).astype(np.float64)
    xn = (xf - nm[:IN]) * nm[IN:2 * IN]
    z1 = xn @ W1 + b1
    h1 = _silu(z1)
    z2 = h1 @ W2 + b2
    h2 = _silu(z2)
    out = h2 @ W3 + b3
    return out, (xn, z1, h1, z2, h2)


def loss64(w, nm, x, y):
    out, _ = forward64(w, nm, x)
    yn = (np.asarray(y, dtype=np.float32).astype(np.float64) - nm[2 * IN]) / nm[2 * IN + 1]
    return float(np.mean((out - yn) ** 2))


def grad64(w, nm, x, y):
    """(gradient [NPARAM], loss) of mean((out - yn)^2) at float64 parameters w."""
    W1, b1, W2, b2, W3, b3 = split(w)
    out, (xn, z1, h1, z2, h2) = forward64(w, nm, x)
    yn = (np.asarray(y, dtype=np.float32).astype(np.float64) - nm[2 * IN]) / nm[2 * IN + 1]
    n = len(out)
    err = out - yn
    d = 2.0 * err / n
    g = np.zeros(NPARAM)
    g[OFF_B3] = d.sum()
    g[OFF_W3:OFF_B3] = h2.T @ d
    dz2 = (d[:, None] * W3[None, :]) * _dsilu(z2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W2:OFF_B2] = (h1.T @ dz2).ravel()
    dh1 = dz2 @ W2.T
    dz1 = dh1 * _dsilu(z1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (xn.T @ dz1).ravel()
    return g, float(np.mean(err ** 2))


def forward(model, x):
    w, nm = params_used(model)
    return forward64(w, nm, x)


def predict(model, x):
    """De-standardised model output (dlog RS)."""
    w, nm = params_used(model)
    out, _ = forward64(w, nm, x)
    return out * nm[2 * IN + 1] + nm[2 * IN]


def grad(model, x, y):
    """Gradient and loss with respect to the bf16 parameters the GPU uses."""
    w, nm = params_used(model)
    return grad64(w, nm, x, y)


def features(nnb, h2, a2, dtr):
    """The model inputs of one particle (float32), as the CUDA epilogue
    forms them: log(1+nnb), log RS, log(1+nnb) - 1.5 log h2, log|a|, -log2 dtr."""
    n = np.abs(np.asarray(nnb, dtype=np.float64))
    ln = np.log(1.0 + n)
    lh = np.log(np.maximum(h2, 1e-300))
    return np.stack([ln, 0.5 * lh, ln - 1.5 * lh, 0.5 * np.log(np.maximum(a2, 1e-300)),
                     -np.log2(np.maximum(dtr, 1e-300))], axis=-1).astype(np.float32)

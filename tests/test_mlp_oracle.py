"""The FP64 oracle of the learned-radius model, pinned before it is used to
check the CUDA kernels: its analytic gradient equals central finite
differences of its own loss, and its bf16 rounding matches torch's."""
import numpy as np

import mlp_oracle as M


def _model(seed):
    rng = np.random.default_rng(seed)
    model = np.zeros(M.NPARAM + M.NNORM, dtype=np.float32)
    model[:M.NPARAM] = rng.normal(size=M.NPARAM) * 0.2
    model[M.NPARAM:M.NPARAM + M.IN] = rng.normal(size=M.IN) * 0.1
    model[M.NPARAM + M.IN:M.NPARAM + 2 * M.IN] = rng.uniform(0.5, 2.0, M.IN)
    model[-2], model[-1] = 0.1, 0.7
    return model


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    w, nm = M.params_used(_model(2))
    x = rng.normal(size=(37, M.IN)).astype(np.float32)
    y = rng.normal(size=37).astype(np.float32)
    g, _ = M.grad64(w, nm, x, y)
    idx = np.r_[0:5, M.OFF_B1:M.OFF_B1 + 3, M.OFF_W2:M.OFF_W2 + 5, M.OFF_W2 + 2000,
                M.OFF_B2 + 7, M.OFF_W3:M.OFF_W3 + 4, M.OFF_B3]
    for k in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        fd = (M.loss64(wp, nm, x, y) - M.loss64(wm, nm, x, y)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7 + 1e-6 * abs(g[k]), (k, fd, g[k])


def test_bf16_rounding_matches_torch():
    import torch
    a = np.random.default_rng(3).normal(size=4096).astype(np.float32) * 10
    a[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0]        # ties to even
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(M.bf16_round(a), ref)

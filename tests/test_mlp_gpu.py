"""The learned-radius model on the GPU against its FP64 oracle: gradients of
the hand-written backward kernel, forward outputs, a training run, and the
proposal fused into the regular-force epilogue.

Tolerances: the GPU forward pass uses the same bf16 parameters as the oracle
with FP32 sums and expf, so outputs agree to ~1e-6 relative; the gradient
vector within 2e-5 of its norm (FP32 accumulation over the batch)."""
import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _model(seed):
    rng = np.random.default_rng(seed)
    model = np.zeros(M.NPARAM + M.NNORM, dtype=np.float32)
    model[:M.NPARAM] = rng.normal(size=M.NPARAM) * 0.15
    model[M.NPARAM:M.NPARAM + M.IN] = rng.normal(size=M.IN) * 0.1
    model[M.NPARAM + M.IN:M.NPARAM + 2 * M.IN] = rng.uniform(0.5, 2.0, M.IN)
    model[-2], model[-1] = 0.05, 0.4
    return model


def test_gradient_matches_fp64_oracle():
    from nb6b200 import mlp
    rng = np.random.default_rng(5)
    for n, seed in ((1, 1), (777, 2), (4096, 3)):
        model = _model(seed)
        mlp.set_model(model)
        x = rng.normal(size=(n, 5)).astype(np.float32) * 2
        y = rng.normal(size=n).astype(np.float32)
        g, loss = mlp.grad(x, y)
        gr, lr = M.grad(model, x, y)
        assert abs(loss - lr) <= 1e-5 * abs(lr) + 1e-7, (loss, lr)
        err = np.linalg.norm(g - gr) / np.linalg.norm(gr)
        assert err <= 2e-5, (n, err)
        assert np.max(np.abs(g - gr)) <= 2e-5 * np.max(np.abs(gr)) + 1e-8
        # deterministic: the same gradient bit for bit on a second call
        g2, _ = mlp.grad(x, y)
        np.testing.assert_array_equal(g, g2)


def test_forward_matches_fp64_oracle():
    from nb6b200 import mlp
    model = _model(7)
    mlp.set_model(model)
    x = np.random.default_rng(8).normal(size=(1000, 5)).astype(np.float32)
    np.testing.assert_allclose(mlp.predict(x), M.predict(model, x), rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(mlp.get_model(), model)


def test_training_fits_a_smooth_target():
    from nb6b200 import mlp
    rng = np.random.default_rng(11)
    x = rng.normal(size=(20000, 5)).astype(np.float32)
    y = (np.tanh(x[:, 0] - 0.5 * x[:, 2]) + 0.3 * x[:, 1] * x[:, 4]).astype(np.float32)
    mlp.init(3)
    hist = mlp.train(x, y, epochs=12, batch=512, lr=3e-3, seed=1)
    assert hist[-1] < 0.1 * hist[0], hist
    pred = mlp.predict(x[:2000])
    assert np.mean((pred - y[:2000]) ** 2) < 0.1 * np.var(y)


def test_proposal_fused_into_regular_force_epilogue(nb6):
    """Every gpunb_regf_ call with the model enabled writes, per particle,
    the model's proposal evaluated on that call's own neighbour count, h2,
    regular acceleration and dtr."""
    from nb6b200 import ics, mlp
    cl = ics.plummer(3000, seed=4)
    model = _model(9)
    mlp.set_model(model)
    isel = np.arange(0, 3000, 3)
    h2, dtr = cl.h2(0)[isel], cl.dtr[isel]
    mlp.enable(True)
    try:
        nb6.gpunb_open(3010, 0)
        nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
        acc, jrk, pot, lst = nb6.gpunb_regf(h2, dtr, cl.pos[isel], cl.vel[isel], 512, 400, 0)
        prop = mlp.proposals(len(isel))
        nb6.gpunb_close()
    finally:
        mlp.enable(False)
    f = mlp.features(lst[:, 0], h2, (acc ** 2).sum(1), dtr)
    np.testing.assert_allclose(prop, M.predict(model, f), rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(prop, mlp.predict(f), rtol=1e-6, atol=1e-6)

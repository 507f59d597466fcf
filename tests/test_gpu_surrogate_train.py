"""The surrogate's training kernels (tcgen05 forward and backward GEMMs, loss,
Adam) against the FP64 CPU network of oracle/mlp.py.

Gradient tolerances (relative L2 error per weight or bias tensor): the device
computes the gradient of the BF16-rounded network with FP32 sums and the
hardware tanh in SiLU and SiLU'; an activation can land one BF16 step away
from the oracle's, so against the oracle with the same roundings the
gradient agrees to 1e-2, and against the plain FP64 network to 6e-2 (with
cosine similarity above 0.998)."""
import numpy as np
import pytest

from oracle import mlp
from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def rows(rng, n):
    X = np.stack([rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), rng.uniform(-0.8, 0.8, n), rng.uniform(-0.8, 0.8, n),
                  rng.uniform(-1, 1, n)], 1).astype(np.float32)
    hit = (np.hypot(X[:, 2], X[:, 3]) > 0.35).astype(np.float32)
    T = np.stack([hit, hit * (0.5 * X[:, 2] - 0.2 * X[:, 0]), hit * (0.6 + 0.3 * X[:, 3] * X[:, 1]),
                  0.2 * np.sin(3 * X[:, 2]) * X[:, 4]], 1).astype(np.float32)
    w = rng.uniform(0.05, 1.0, n).astype(np.float32)
    return X, T, w


def device(*arrays):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in arrays]


@pytest.mark.parametrize("n", [256, 1024])
def test_gradient_matches_the_fp64_network(engine, n):
    rng = np.random.default_rng(3)
    p = mlp.init_params(rng)
    X, T, w = rows(rng, n)
    dX, dT, dw = device(X, T, w)
    engine.train_init(p, abi.train_config(batch=1024))
    parts, g = engine.train_gradient(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), n)
    pr, gr = mlp.loss_and_grad(p, X, T, w, rounded=True)
    pe, ge = mlp.loss_and_grad(p, X, T, w, rounded=False)
    np.testing.assert_allclose(parts, pr, rtol=5e-3, atol=1e-7)
    for name, sl in mlp.layer_slices():
        ref = np.linalg.norm(gr[sl])
        assert np.linalg.norm(g[sl] - gr[sl]) < 1e-2 * ref, (name, np.linalg.norm(g[sl] - gr[sl]) / ref)
        assert np.linalg.norm(g[sl] - ge[sl]) < 6e-2 * np.linalg.norm(ge[sl]), name
        cos = g[sl] @ ge[sl] / (np.linalg.norm(g[sl]) * np.linalg.norm(ge[sl]))
        assert cos > 0.998, (name, cos)
    # the gradient call leaves no trace: a second call gives the same result
    parts2, g2 = engine.train_gradient(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), n)
    np.testing.assert_allclose(g2, g, rtol=1e-4, atol=1e-6 * np.abs(g).max())


def test_first_adam_step(engine):
    """One optimiser step on a training set of exactly one batch: with zero
    moments the Adam update is lr_0 g / (|g| + eps) per parameter, lr_0 = max_lr / 25."""
    rng = np.random.default_rng(4)
    p = mlp.init_params(rng)
    X, T, w = rows(rng, 512)
    dX, dT, dw = device(X, T, w)
    cfg = abi.train_config(batch=512, total_steps=100, max_lr=1e-3)
    engine.train_init(p, cfg)
    _, g = engine.train_gradient(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), 512)
    engine.train_steps(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), 512, 1)
    p1, steps = engine.train_params()
    assert steps == 1
    lr0 = 1e-3 / 25
    step = p.astype(np.float64) - p1
    big = np.abs(g) > 1e-4 * np.abs(g).max()
    expect = lr0 * g[big] / (np.abs(g[big]) + 1e-8)
    # the batch's rows come in a permuted order (other FP32 sums): the sign and size agree
    assert np.mean(np.abs(step[big] - expect) < 0.05 * lr0) > 0.99
    assert np.all(np.abs(step) <= lr0 * 1.001 + 1e-7)


def test_training_reduces_the_validation_loss(engine):
    """A few hundred replayed steps on a smooth synthetic problem cut the held-out loss severalfold."""
    rng = np.random.default_rng(5)
    n_train, n_val = 64 * 1024, 8192
    X, T, w = rows(rng, n_train + n_val)
    dX, dT, dw = device(X, T, w)
    steps = 400
    engine.train_init(mlp.init_params(rng), abi.train_config(batch=2048, total_steps=steps, max_lr=2e-3, seed=1))
    v = lambda: engine.train_evaluate(dX[n_train:].data_ptr(), dT[n_train:].data_ptr(),  # noqa: E731
                                      dw[n_train:].data_ptr(), n_val)
    before = mlp.total_loss(v())
    engine.train_steps(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), n_train, steps)
    after = mlp.total_loss(v())
    p, done = engine.train_params()
    assert done == steps and np.all(np.isfinite(p))
    assert after < 0.2 * before, (before, after)
    # the evaluation agrees with the FP64 network's loss on the same rows and trained weights
    Y, _, _ = mlp.forward(p, X[n_train:], rounded=True)
    parts, _ = mlp.loss_parts_and_dy(Y, T[n_train:].astype(np.float64), w[n_train:].astype(np.float64))
    np.testing.assert_allclose(mlp.total_loss(parts), after, rtol=2e-2)
    # and the inference kernel, loaded with the trained weights, reproduces the trainer's forward pass
    import torch
    engine.surrogate_load(p)
    d_out = torch.zeros((n_val, 4), dtype=torch.float32, device="cuda")
    engine.surrogate_infer(dX[n_train:].data_ptr(), n_val, d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()
    assert np.abs(out - Y).max() < 2e-2 * np.abs(Y).max()


def test_argument_checks(engine):
    from sirius_b200.engine import SiriusError
    rng = np.random.default_rng(6)
    X, T, w = rows(rng, 256)
    dX, dT, dw = device(X, T, w)
    with pytest.raises(SiriusError):
        engine.train_init(mlp.init_params(rng), abi.train_config(batch=100))
    engine.train_init(mlp.init_params(rng), abi.train_config(batch=256))
    with pytest.raises(SiriusError):
        engine.train_gradient(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), 200)
    with pytest.raises(SiriusError):
        engine.train_steps(dX.data_ptr(), dT.data_ptr(), dw.data_ptr(), 128, 1)

"""The FP64 CPU restatement of the surrogate network and its loss (the checker
for the tensor-core training kernels): its analytic gradient against central
finite differences, its BF16 rounding, and the size of the gradient change
that the device's roundings make."""
import numpy as np

from oracle import mlp


def batch(rng, n):
    X = rng.uniform(-1.0, 1.0, size=(n, 5))
    T = np.stack([rng.integers(0, 2, n), rng.normal(size=n), rng.uniform(0.0, 1.5, n), 0.1 * rng.normal(size=n)], 1)
    w = rng.uniform(0.05, 1.0, n)
    return X, T, w


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = mlp.init_params(rng).astype(np.float64)
    X, T, w = batch(rng, 32)
    _, g = mlp.loss_and_grad(p, X, T, w)
    eps = 1e-6
    # a sample of every tensor: weights and biases of all five layers
    idx = np.concatenate([rng.choice(np.arange(sl.start, sl.stop), size=min(6, sl.stop - sl.start), replace=False)
                          for _, sl in mlp.layer_slices()])
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp = mlp.total_loss(mlp.loss_parts_and_dy(mlp.forward(q, X)[0], T, w)[0])
        q[i] -= 2 * eps
        lm = mlp.total_loss(mlp.loss_parts_and_dy(mlp.forward(q, X)[0], T, w)[0])
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 5e-5 * max(abs(g[i]), 1e-3), (i, fd, g[i])


def test_bf16_rounds_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -9, np.pi, -2.5e-3, 0.0])
    r = mlp.bf16(x)
    np.testing.assert_array_equal(r[:3], [1.0, 1.0, 1.0 + 2.0 ** -7])
    assert r[3] == 3.140625
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)  # unit roundoff of an 8-bit significand


def test_rounded_gradient_stays_close_to_the_exact_one():
    rng = np.random.default_rng(1)
    p = mlp.init_params(rng)
    X, T, w = batch(rng, 256)
    pe, ge = mlp.loss_and_grad(p, X, T, w, rounded=False)
    pr, gr = mlp.loss_and_grad(p, X, T, w, rounded=True)
    np.testing.assert_allclose(pr, pe, rtol=2e-2)
    for name, sl in mlp.layer_slices():
        rel = np.linalg.norm(gr[sl] - ge[sl]) / np.linalg.norm(ge[sl])
        assert rel < 5e-2, (name, rel)

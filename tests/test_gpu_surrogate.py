"""The surrogate MLP on the tensor cores (tcgen05, BF16 operands, FP32
accumulation) against a plain PyTorch FP32 reference of the same network with
the same BF16 roundings of weights and activations.

Tolerance: the device rounds each hidden activation to BF16 (2^-8 relative)
after an FP32 sum whose order differs from the reference's, and evaluates the
SiLU's sigmoid with the hardware tanh (relative error ~2^-11): an activation
can land one BF16 step away. Outputs agree to 2 % of the output scale at worst
and 0.2 % on average."""
import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def init_params(rng):
    sizes = [(256, 5), (256, 256), (256, 256), (256, 256), (4, 256)]
    parts = []
    for out, inp in sizes:
        bound = 1.0 / np.sqrt(inp)
        parts.append(rng.uniform(-bound, bound, size=(out, inp)).astype(np.float32).ravel())
        parts.append(rng.uniform(-bound, bound, size=out).astype(np.float32))
    p = np.concatenate(parts)
    assert p.size == abi.SURROGATE_PARAMS
    return p


def mlp_reference(params, x):
    import torch
    bf = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    sizes = [(256, 5), (256, 256), (256, 256), (256, 256), (4, 256)]
    h = bf(torch.from_numpy(x))
    off = 0
    for i, (out, inp) in enumerate(sizes):
        W = torch.from_numpy(params[off:off + out * inp].reshape(out, inp)); off += out * inp
        b = torch.from_numpy(params[off:off + out]); off += out
        h = h @ bf(W).T + b
        if i < 4:
            h = bf(torch.nn.functional.silu(h))
    return h.numpy()


@pytest.mark.parametrize("n", [1000, 128 * 300 + 5])
def test_mlp_matches_fp32_reference(engine, n):
    import torch
    rng = np.random.default_rng(7)
    params = init_params(rng)
    x = rng.uniform(-1.0, 1.0, size=(n, 5)).astype(np.float32)
    engine.surrogate_load(params)
    dev = torch.device("cuda", 0)
    d_x = torch.from_numpy(x).to(dev)
    d_y = torch.full((n, 4), float("nan"), dtype=torch.float32, device=dev)
    engine.surrogate_infer(d_x.data_ptr(), n, d_y.data_ptr(), torch.cuda.current_stream(dev).cuda_stream)
    y = d_y.cpu().numpy()
    ref = mlp_reference(params, x)
    assert np.all(np.isfinite(y))
    scale = np.abs(ref).max()
    err = np.abs(y - ref) / scale
    assert err.max() < 2e-2, err.max()
    assert err.mean() < 2e-3, err.mean()


def test_mlp_rejects_wrong_parameter_count(engine):
    from sirius_b200.engine import SiriusError
    with pytest.raises(SiriusError):
        engine.surrogate_load(np.zeros(100, dtype=np.float32))

"""FP64 CPU restatement of the surrogate network, its training loss and the
loss's gradient.

TEST INFRASTRUCTURE ONLY — the checker for the library's tensor-core training
kernels (tests/ import it); never imported by the product package. The
surrogate has no counterpart in the reference, so this module restates the
library's own definition of the network and loss (5 -> 256 -> 256 -> 256 ->
256 -> 4, SiLU after the hidden layers, parameters in nn.Linear order W1 b1 ...
W5 b5) in plain numpy float64.

`rounded=True` applies the roundings the device arithmetic applies — each
input feature as the sum of two BF16 terms (hi = bf16(x), lo = bf16(x - hi),
the kernels' pack_input_row), BF16 weights and hidden activations in the
forward pass, BF16 dL/dY and dZ as operands of the backward products — with
exact sums and an exact SiLU, so that the device gradient can be compared with
the gradient of the same rounded network. `rounded=False` is the plain FP64
network.
"""
import numpy as np

SIZES = [(256, 5), (256, 256), (256, 256), (256, 256), (4, 256)]
N_PARAMS = sum(o * i + o for o, i in SIZES)


def unpack(params):
    """[(W, b)] per layer, views into the flat parameter vector."""
    p = np.asarray(params, dtype=np.float64)
    assert p.size == N_PARAMS
    out, off = [], 0
    for o, i in SIZES:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((W, b))
    return out


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (r.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def bf16_pair(x):
    """The two-term BF16 form of FP32 inputs: bf16(x) + bf16(x - bf16(x))."""
    f = np.asarray(x, dtype=np.float32)
    hi = bf16(f)
    lo = bf16((f.astype(np.float64) - hi).astype(np.float32))
    return hi + lo


def sigmoid(x):
    return 0.5 * (1.0 + np.tanh(0.5 * x))


def silu(x):
    return x * sigmoid(x)


def dsilu(x):
    s = sigmoid(x)
    return s * (1.0 + x * (1.0 - s))


def _identity(a):
    return np.asarray(a, dtype=np.float64)


def forward(params, X, rounded=False):
    """Outputs (n x 4), and the pre-activations and activations of the hidden layers
    (activations[0] is the input)."""
    layers = unpack(params)
    rnd = bf16 if rounded else _identity
    h = bf16_pair(X) if rounded else _identity(X)
    zs, hs = [], [h]
    for li, (W, b) in enumerate(layers):
        z = h @ rnd(W).T + b
        if li == len(layers) - 1:
            return z, zs, hs
        zs.append(z)
        h = rnd(silu(z))
        hs.append(h)


def loss_parts_and_dy(Y, T, w):
    """Loss parts (BCE, l_r, l_g, l_h) of one batch and dL/dY, with
    L = BCE + 100 (l_r + l_g) + 10 l_h."""
    B = Y.shape[0]
    hit = T[:, 0]
    s_w = max(w.sum(), 1e-30)
    s_hw = max((hit * w).sum(), 1e-12 * B)
    o0 = Y[:, 0]
    bce = np.mean(np.maximum(o0, 0) - hit * o0 + np.log1p(np.exp(-np.abs(o0))))
    e = Y[:, 1:] - T[:, 1:]
    parts = np.array([bce, (hit * w * e[:, 0] ** 2).sum() / s_hw, (hit * w * e[:, 1] ** 2).sum() / s_hw,
                      (w * e[:, 2] ** 2).sum() / s_w])
    dY = np.stack([(sigmoid(o0) - hit) / B, 200.0 * hit * w * e[:, 0] / s_hw, 200.0 * hit * w * e[:, 1] / s_hw,
                   20.0 * w * e[:, 2] / s_w], axis=1)
    return parts, dY


def total_loss(parts):
    return parts[0] + 100.0 * (parts[1] + parts[2]) + 10.0 * parts[3]


def loss_and_grad(params, X, T, w, rounded=False):
    """Loss parts and the flat gradient (parameter order) of one batch."""
    layers = unpack(params)
    rnd = bf16 if rounded else _identity
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    Y, zs, hs = forward(params, X, rounded)
    parts, dY = loss_parts_and_dy(Y, T, w)
    grads = [None] * len(layers)
    d = rnd(dY)
    grads[4] = (d.T @ hs[4], dY.sum(axis=0))
    dh = d @ rnd(layers[4][0])
    for li in range(3, -1, -1):
        dz = dh * dsilu(zs[li])
        dzr = rnd(dz)
        grads[li] = (dzr.T @ hs[li], dz.sum(axis=0))
        if li > 0:
            dh = dzr @ rnd(layers[li][0])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return parts, flat


def layer_slices():
    """(name, slice) of each weight and bias in the flat parameter vector."""
    out, off = [], 0
    for li, (o, i) in enumerate(SIZES):
        out.append((f"W{li + 1}", slice(off, off + o * i)))
        off += o * i
        out.append((f"b{li + 1}", slice(off, off + o)))
        off += o
    return out


def init_params(rng):
    """nn.Linear's default initialisation: U(-1/sqrt(in), 1/sqrt(in)) for weights and biases."""
    parts = []
    for o, i in SIZES:
        bound = 1.0 / np.sqrt(i)
        parts.append(rng.uniform(-bound, bound, size=o * i))
        parts.append(rng.uniform(-bound, bound, size=o))
    return np.concatenate(parts).astype(np.float32)

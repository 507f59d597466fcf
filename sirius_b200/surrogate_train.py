"""Fit the surrogate MLP (5 -> 256 -> 256 -> 256 -> 256 -> 4, SiLU) to rays
traced by the engine, and write its parameters (nn.Linear order, float32) for
sirius_cuda_surrogate_load.

Training set: 2^24 rays of 4096 Kerr frames with a* ~ U[0, 0.99], inclination
~ U[5, 89] deg, r_obs ~ U[20, 200] M, each a 64^2 30 deg pinhole camera (pixel
centres with a random sub-pixel offset per frame, so alpha and beta cover the
field of view), thin Novikov-Thorne disk r_ISCO..30 M, traced by the
mixed-precision integrator at tol 1e-8.

Features are those of sirius_cuda_surrogate_features (computed by the library,
so training and inference see the same inputs). Targets per ray:
  t0 = 1 if the ray crosses the disk, else 0          (logit, binary cross-entropy)
  t1 = r_1 / 15 - 1, t2 = g_1 at the first crossing    (squared error, crossing rays)
  t3 = (I - g_1^4 F(r_1)) * 1e3, the higher-order part (squared error)
The squared errors are weighted by the ray's brightness relative to its
frame's brightest primary, as the image error is measured against the image
scale.

The fitting itself runs in PyTorch (an offline step, not the rendering path);
inference runs on the library's tensor-core kernel, which rounds the inputs,
weights and hidden activations to BF16: the last 40 % of the epochs train
through the same roundings (straight-through gradients), so the fitted network
is the one the kernel evaluates.

Usage: python -m sirius_b200.surrogate_train [--rays N] [--epochs E] [--out PATH]
"""
import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "surrogate_kerr.npy")
SIDE = 64


def sample_frames(abi, rng, n):
    frames = []
    for _ in range(n):
        a = rng.uniform(0.0, 0.99)
        th = rng.uniform(5.0, 89.0)
        r = rng.uniform(20.0, 200.0)
        cam = abi.make_camera(r=r, theta_deg=th, width=SIDE, height=SIDE, fov=30.0)
        # a random sub-pixel offset of the whole frame (pixel centres stay the sample points)
        cam.yaw, cam.pitch = rng.uniform(-0.5, 0.5, size=2) * (30.0 / SIDE) * np.pi / 180.0
        frames.append(abi.make_frame(abi.make_metric(a=a), cam, 0.0, 30.0))
    return frames


def trace_config(abi):
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              initial_step=0.1, escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                              precision=abi.PRECISION_MIXED, enable_disk=1, enable_volumetric=0)


def targets_from_results(res, n_frames):
    """Targets (hit, r_1/15 - 1, g_1, higher * 1e3) and the brightness weight of each ray."""
    hit = res["n_crossings"] >= 1
    r1 = np.where(hit, res["disk_r"][:, 0], 15.0).astype(np.float64)
    g1 = np.where(hit, res["disk_g"][:, 0], 0.0).astype(np.float64)
    prim = np.where(hit, g1 ** 4 * res["disk_flux"][:, 0], 0.0)
    higher = res["intensity"].astype(np.float64) - prim
    t = np.stack([hit.astype(np.float64), r1 / 15.0 - 1.0, g1, higher * 1e3], axis=1)
    peak = np.maximum(prim.reshape(n_frames, -1).max(axis=1, keepdims=True), 1e-30)
    w = (0.05 + prim.reshape(n_frames, -1) / peak).ravel()
    return t.astype(np.float32), w.astype(np.float32)


def make_dataset(eng, abi, torch, n_rays, seed, chunk_frames=256):
    rng = np.random.default_rng(seed)
    n_frames = max(n_rays // (SIDE * SIDE), 1)
    dev = torch.device("cuda", 0)
    X, Y, W = [], [], []
    eng.configure(trace_config(abi))
    for c0 in range(0, n_frames, chunk_frames):
        frames = sample_frames(abi, rng, min(chunk_frames, n_frames - c0))
        n = len(frames) * SIDE * SIDE
        d_feat = torch.empty((n, 5), dtype=torch.float32, device=dev)
        eng.surrogate_features(frames, d_feat.data_ptr())
        res, _, _ = eng.trace_frames(frames, results=True, image=False)
        t, w = targets_from_results(res, len(frames))
        X.append(d_feat)
        Y.append(torch.from_numpy(t).to(dev))
        W.append(torch.from_numpy(w).to(dev))
    return torch.cat(X), torch.cat(Y), torch.cat(W)


def build_mlp(torch):
    nn = torch.nn
    layers = []
    dims = [5, 256, 256, 256, 256]
    for i in range(4):
        layers += [nn.Linear(dims[i], dims[i + 1]), nn.SiLU()]
    layers.append(nn.Linear(256, 4))
    return nn.Sequential(*layers)


def forward_bf16(torch, model, x):
    """The kernel's arithmetic: BF16 inputs, weights and hidden activations, FP32
    sums and biases; rounding with straight-through gradients."""
    def rnd(t):
        return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()
    h = rnd(x)
    lin = [m for m in model if hasattr(m, "weight")]
    for i, m in enumerate(lin):
        h = h @ rnd(m.weight).T + m.bias
        if i < len(lin) - 1:
            h = rnd(torch.nn.functional.silu(h))
    return h


def loss_fn(torch, out, y, w):
    F = torch.nn.functional
    hit = y[:, 0]
    l_hit = F.binary_cross_entropy_with_logits(out[:, 0], hit)
    wh = hit * w
    wh = wh / wh.mean().clamp_min(1e-12)
    l_r = (wh * (out[:, 1] - y[:, 1]) ** 2).mean()
    l_g = (wh * (out[:, 2] - y[:, 2]) ** 2).mean()
    l_h = (w * (out[:, 3] - y[:, 3]) ** 2).mean() / w.mean()
    return l_hit + 100.0 * (l_r + l_g) + 10.0 * l_h, (l_hit, l_r, l_g, l_h)


def flatten_params(model):
    parts = []
    for m in model:
        if hasattr(m, "weight"):
            parts.append(m.weight.detach().float().cpu().numpy().ravel())
            parts.append(m.bias.detach().float().cpu().numpy().ravel())
    return np.concatenate(parts).astype(np.float32)


def train(n_rays=1 << 24, epochs=8, batch=16384, lr=2e-3, seed=0, out=DEFAULT_OUT, log=print):
    import torch

    from sirius_b200 import abi
    from sirius_b200.engine import Engine

    torch.manual_seed(seed)
    eng = Engine(0)
    t0 = time.time()
    X, Y, Wt = make_dataset(eng, abi, torch, n_rays, seed)
    log(f"dataset: {X.shape[0]} rays in {time.time() - t0:.1f} s, disk-hit fraction {Y[:, 0].mean().item():.3f}")
    n = X.shape[0]
    perm = torch.randperm(n, device=X.device)
    n_val = max(n // 50, 1)
    val, tr = perm[:n_val], perm[n_val:]
    model = build_mlp(torch).to(X.device)
    opt = torch.optim.AdamW(model.parameters(), lr=lr, weight_decay=0.0)
    steps = epochs * (tr.numel() // batch)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=steps, pct_start=0.05)
    step = 0
    t0 = time.time()
    q_from = int(0.6 * epochs)
    for ep in range(epochs):
        fwd = (lambda x: forward_bf16(torch, model, x)) if ep >= q_from else model
        order = tr[torch.randperm(tr.numel(), device=X.device)]
        for i in range(0, order.numel() - batch + 1, batch):
            idx = order[i:i + batch]
            loss, _ = loss_fn(torch, fwd(X[idx]), Y[idx], Wt[idx])
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            step += 1
        with torch.no_grad():
            outv = torch.cat([fwd(X[val[j:j + 65536]]) for j in range(0, val.numel(), 65536)])
            _, parts = loss_fn(torch, outv, Y[val], Wt[val])
        log(f"epoch {ep}: loss parts (hit bce, r, g, higher) = {[round(p.item(), 8) for p in parts]}, "
            f"{time.time() - t0:.1f} s")
    train.model = model  # the fitted torch module, for inspection
    params = flatten_params(model)
    assert params.size == abi.SURROGATE_PARAMS
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.save(out, params)
    log(f"wrote {out} ({params.size} parameters)")
    return params


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rays", type=int, default=1 << 24)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    train(a.rays, a.epochs, a.batch, a.lr, a.seed, a.out, log=lambda m: print(m, flush=True))


if __name__ == "__main__":
    main()

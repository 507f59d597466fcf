"""Fit the surrogate MLP (5 -> 256 -> 256 -> 256 -> 256 -> 4, SiLU) to rays
traced by the engine, with the library's own training kernels, and write its
parameters (nn.Linear order, float32) for sirius_cuda_surrogate_load.

Training set: 2^26 rays of 16384 Kerr frames with a* ~ U[0, 0.99], inclination
~ U[5, 89] deg, r_obs ~ U[20, 200] M, each a 64^2 30 deg pinhole camera (pixel
centres with a random sub-pixel offset per frame, so alpha and beta cover the
field of view), thin Novikov-Thorne disk r_ISCO..30 M, traced by the
mixed-precision integrator at tol 1e-8. The last 2 % of the frames are held
out for validation.

Features are those of sirius_cuda_surrogate_features (computed by the library,
so training and inference see the same inputs). Targets per ray:
  t0 = 1 if the ray crosses the disk, else 0          (logit, binary cross-entropy)
  t1 = r_1 / 15 - 1, t2 = g_1 at the first crossing    (squared error, crossing rays)
  t3 = (I - g_1^4 F(r_1)) * 1e3, the higher-order part (squared error)
The squared errors are weighted by the ray's brightness relative to its
frame's brightest primary, as the image error is measured against the image
scale.

The fit runs on the tensor cores (sirius_cuda_train_*): BF16 tcgen05 forward
and backward GEMMs with the inference kernel's roundings, Adam on FP32 master
weights, one optimiser step per replay of a captured CUDA graph, the rows of
each epoch in a fresh keyed permutation. PyTorch only holds the device
buffers of the training set.

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


def init_params(rng):
    """nn.Linear's default initialisation: U(-1/sqrt(in), 1/sqrt(in)) for weights and biases."""
    parts = []
    for o, i in [(256, 5), (256, 256), (256, 256), (256, 256), (4, 256)]:
        bound = 1.0 / np.sqrt(i)
        parts.append(rng.uniform(-bound, bound, size=o * i))
        parts.append(rng.uniform(-bound, bound, size=o))
    return np.concatenate(parts).astype(np.float32)


def total_loss(parts):
    return parts[0] + 100.0 * (parts[1] + parts[2]) + 10.0 * parts[3]


def train(n_rays=1 << 26, epochs=60, batch=32768, lr=4e-3, seed=0, out=DEFAULT_OUT, log=print):
    from sirius_b200 import abi
    from sirius_b200.engine import Engine

    import torch

    eng = Engine(0)
    t0 = time.time()
    X, Y, Wt = make_dataset(eng, abi, torch, n_rays, seed)
    log(f"dataset: {X.shape[0]} rays in {time.time() - t0:.1f} s, disk-hit fraction {Y[:, 0].mean().item():.3f}")
    n = X.shape[0]
    n_val = max((n // 50) // (SIDE * SIDE), 1) * SIDE * SIDE  # whole frames
    n_train = n - n_val
    if n_train < batch:
        raise ValueError(f"{n_train} training rows hold no batch of {batch}")
    steps_per_epoch = n_train // batch
    cfg = abi.train_config(batch=batch, total_steps=epochs * steps_per_epoch, max_lr=lr, seed=seed)
    eng.train_init(init_params(np.random.default_rng(seed)), cfg)
    xv, yv, wv = X[n_train:], Y[n_train:], Wt[n_train:]
    t0 = time.time()
    for ep in range(epochs):
        eng.train_steps(X.data_ptr(), Y.data_ptr(), Wt.data_ptr(), n_train, steps_per_epoch)
        parts = eng.train_evaluate(xv.data_ptr(), yv.data_ptr(), wv.data_ptr(), n_val)
        log(f"epoch {ep}: validation loss parts (hit bce, r, g, higher) = {[round(float(p), 8) for p in parts]}, "
            f"total {total_loss(parts):.6f}, {time.time() - t0:.1f} s")
    params, steps = eng.train_params()
    assert params.size == abi.SURROGATE_PARAMS and steps == epochs * steps_per_epoch
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.save(out, params)
    log(f"wrote {out} ({params.size} parameters, {steps} optimiser steps)")
    eng.close()
    return params


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rays", type=int, default=1 << 26)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=32768)
    ap.add_argument("--lr", type=float, default=4e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    train(a.rays, a.epochs, a.batch, a.lr, a.seed, a.out, log=lambda m: print(m, flush=True))


if __name__ == "__main__":
    main()

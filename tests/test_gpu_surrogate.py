"""The surrogate MLP on the tensor cores (tcgen05, BF16 operands, FP32
accumulation) against a plain PyTorch FP32 reference of the same network with
the same BF16 roundings of weights and activations (each input feature as two
BF16 terms, bf16(x) + bf16(x - bf16(x))).

Tolerance: the device rounds each hidden activation to BF16 (2^-8 relative)
after an FP32 sum whose order differs from the reference's, and evaluates the
SiLU's sigmoid with the hardware tanh (relative error ~2^-11): an activation
can land one BF16 step away. Outputs agree to 2 % of the output scale at worst
and 0.2 % on average."""
import os

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
    xt = torch.from_numpy(x)
    h = bf(xt) + bf(xt - bf(xt))
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


WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sirius_b200", "data",
                       "surrogate_kerr.npy")


def kerr_frame(side):
    cam = abi.make_camera(r=100.0, theta_deg=60.0, width=side, height=side, fov=30.0)
    return abi.make_frame(abi.make_metric(a=0.9), cam, 0.0, 30.0)


def render_config(prec):
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              initial_step=0.1, escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                              precision=prec, enable_disk=1, enable_volumetric=0, critical_band=0.0)


def test_surrogate_render_against_the_integrator(engine):
    """Surrogate-gated frame vs the same frame fully integrated: the gated and
    audit pixels are the integrator's own values (bit for bit); the rest come
    from the MLP within the surrogate's error budget, which holds for the worst
    pixel too: L-infinity <= 1e-2 and p99 <= 1e-3 of the frame peak (the
    inner-disk gate takes the pixels where the flux rises steeply from the
    inner edge, which the network's radius cannot resolve)."""
    engine.surrogate_load(np.load(WEIGHTS))
    fr = kerr_frame(512)
    engine.configure(render_config(abi.PRECISION_MIXED))
    _, full, _ = engine.trace_frames([fr], results=False)
    img, mimg, gate, st = engine.render_surrogate([fr], mlp_image=True)
    taken = gate != 0
    assert st.rays == full.size and st.integrated == int(taken.sum())
    np.testing.assert_array_equal(img[taken], full[taken])
    np.testing.assert_array_equal(img[~taken], mimg[~taken])
    assert 0.004 < np.mean(gate == 2) < 0.02      # 1 % audit, in runs of 32 pixels
    # the +-0.3 M band around the critical curve and the inner-disk gate
    assert 0.001 < np.mean(gate == 1) < 0.08, np.mean(gate == 1)
    assert st.coarse_rays == 64 * 64  # 8 x 8 pixel cells
    err = np.abs(img.astype(np.float64) - full) / full.max()
    print("surrogate 512^2: L-inf %.3e p99 %.3e mean %.3e gated %.4f" % (err.max(), np.percentile(err, 99), err.mean(),
                                                                           np.mean(gate == 1)))
    assert err.mean() < 1e-4, err.mean()
    assert np.percentile(err, 99) < 1e-3, np.percentile(err, 99)
    assert err.max() < 1e-2, err.max()
    # the audit's judgement in the statistics: the MLP against the integrator on the audit pixels
    a = gate == 2
    d = np.abs(mimg[a].astype(np.float64) - img[a])
    assert st.audit_count == int(a.sum())
    np.testing.assert_allclose(st.audit_rel_l1, d.sum() / img[a].sum(dtype=np.float64), rtol=1e-4)
    np.testing.assert_allclose(st.audit_rel_max, d.max() / img[a].max(), rtol=1e-6)


def test_empty_pixels_skip_the_network(engine):
    """Pixels whose coarse cell and its eight neighbours all predict no disk
    crossing (gate 3) take intensity 0 without the per-pixel MLP, which runs only
    on the pixels it shades and the audit pixels. Every other pixel equals the
    render without the skip bit for bit (the network evaluates each row on its
    own), and the integrator finds no light at the empty pixels (thin disk: a
    ray that never crosses it carries none)."""
    engine.surrogate_load(np.load(WEIGHTS))
    fr = kerr_frame(512)
    engine.configure(render_config(abi.PRECISION_MIXED))
    _, full, _ = engine.trace_frames([fr], results=False)
    img, _, gate, st = engine.render_surrogate([fr])
    ref, _, gate_ref, _ = engine.render_surrogate([fr], config=abi.surrogate_config(empty_skip=-1))
    empty = gate == 3
    assert 0.2 < empty.mean() < 0.8, empty.mean()
    assert not np.any(gate_ref == 3)
    np.testing.assert_array_equal(gate[~empty], gate_ref[~empty])
    np.testing.assert_array_equal(img[~empty], ref[~empty])
    assert np.all(img[empty] == 0.0)
    assert np.abs(full[empty]).max() <= 1e-3 * full.max(), np.abs(full[empty]).max() / full.max()


def test_surrogate_integrates_frames_it_does_not_cover(engine):
    """A Morris-Thorne frame (outside the MLP's training set) is integrated in full."""
    engine.surrogate_load(np.load(WEIGHTS))
    fr = abi.make_frame(abi.make_metric(family=abi.MORRIS_THORNE, b0=1.0),
                        abi.make_camera(r=20.0, theta_deg=80.0, width=64, height=64, fov=40.0), 0.0, 20.0)
    engine.configure(render_config(abi.PRECISION_MIXED))
    _, full, _ = engine.trace_frames([fr], results=False)
    img, _, gate, st = engine.render_surrogate([fr])
    assert np.all(gate == 1) and st.integrated == full.size
    np.testing.assert_array_equal(img, full)


def test_trained_network_gains_over_the_untrained_one(engine):
    """What training buys: the same gated render with the fitted weights and
    with the network's initial (untrained) weights. Both integrate the same
    ~1-2 % of the rays (the gate does not depend on the weights); the fitted
    network brings the other pixels within the error budget, the untrained one
    does not, so without the trained network the whole frame would have to be
    integrated to reach that error."""
    fr = kerr_frame(512)
    engine.configure(render_config(abi.PRECISION_MIXED))
    _, full, _ = engine.trace_frames([fr], results=False)
    scale = full.max()
    errs, fractions, audits = {}, {}, {}
    rng = np.random.default_rng(11)
    # the critical-curve gate alone (the inner-disk gate reads the network's own outputs)
    cfg = abi.surrogate_config(inner_gate=-1.0)
    for name, params in (("trained", np.load(WEIGHTS)), ("untrained", init_params(rng))):
        engine.surrogate_load(params)
        img, _, gate, st = engine.render_surrogate([fr], config=cfg)
        errs[name] = np.abs(img.astype(np.float64) - full) / scale
        fractions[name] = st.integrated / st.rays
        audits[name] = st.audit_rel_l1
    assert fractions["trained"] == fractions["untrained"] < 0.05
    # the 1 % audit sees the difference on its own
    assert audits["untrained"] > 10 * audits["trained"], audits
    assert errs["trained"].mean() < 1e-3 and np.percentile(errs["trained"], 99) < 1e-2
    assert errs["untrained"].mean() > 10 * errs["trained"].mean()
    assert np.percentile(errs["untrained"], 99) > 5 * np.percentile(errs["trained"], 99)


def test_audit_over_budget_renders_again_with_wider_gates(engine):
    """The audit acts: with a budget below the audit's measured error, the frame
    is rendered once more with the critical-curve band and the inner-disk gate
    1.5 times wider; more pixels are integrated, and those are the integrator's."""
    engine.surrogate_load(np.load(WEIGHTS))
    fr = kerr_frame(256)
    engine.configure(render_config(abi.PRECISION_MIXED))
    _, full, _ = engine.trace_frames([fr], results=False)
    img0, _, gate0, st0 = engine.render_surrogate([fr])
    assert st0.rerendered == 0
    img1, _, gate1, st1 = engine.render_surrogate([fr], config=abi.surrogate_config(audit_budget=1e-9))
    assert st1.rerendered == 1
    assert st1.integrated > st0.integrated
    assert np.all(gate1[gate0 == 1] == 1)
    taken = gate1 != 0
    np.testing.assert_array_equal(img1[taken], full[taken])

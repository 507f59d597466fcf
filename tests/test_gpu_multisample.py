"""samples_per_pixel > 1: the image averages a g x g stratified grid of
sub-pixel rays (RenderSession::shadePixel, SNRS001A.cpp:480-530). Checked
against the FP64 oracle tracing the same sub-pixel camera rays (the oracle's
camera is pinned to PinholeCamera::generateRay(x, y, u, v) bit for bit) and
averaging them in the same order. Tolerance: the FP64 path agrees with the
oracle per ray at rounding level; the per-pixel mean adds FP32 summation
rounding (1e-6 of the image scale); a ray whose outcome flips at rounding level
moves its pixel more, so 99 % of the pixels must agree."""
import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def config(spp, prec=abi.PRECISION_FP64):
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              initial_step=0.1, escape_radius=1000.0, horizon_factor=1.01, max_steps=10000,
                              precision=prec, samples_per_pixel=spp)


@pytest.mark.parametrize("spp,g", [(4, 2), (10, 3)])
def test_multisample_image_matches_the_oracle(engine, oracle, spp, g):
    met = abi.make_metric(a=0.9)
    cam = abi.make_camera(r=40.0, theta_deg=75.0, fov=25.0, width=24, height=20)
    fr = abi.make_frame(met, cam, 0.0, 20.0)
    cfg = config(spp)
    engine.configure(cfg)
    _, img, _ = engine.trace_frames([fr], results=False)
    rays = []
    for py in range(cam.height):
        for px in range(cam.width):
            for sy in range(g):
                for sx in range(g):
                    u = (np.float32(sx) + np.float32(0.5)) / np.float32(g)
                    v = (np.float32(sy) + np.float32(0.5)) / np.float32(g)
                    o, d = oracle.camera_ray(cam, px, py, float(u), float(v))
                    ray = abi.CameraRay()
                    ray.origin[:] = list(o)
                    ray.direction[:] = list(d)
                    rays.append(ray)
    out = oracle.trace_rays(met, rays, config(1), disk_inner=0.0, disk_outer=20.0, threads=8)
    ref = out["intensity"].astype(np.float32).reshape(-1, g * g)
    acc = ref[:, 0].copy()
    for k in range(1, g * g):
        acc = acc + ref[:, k]
    ref_img = acc * np.float32(1.0 / (g * g))
    assert ref_img.max() > 0
    err = np.abs(img - ref_img) / ref_img.max()
    assert np.mean(err <= 1e-6) >= 0.99, np.sort(err)[-10:]
    # one sample per pixel differs from the average (the grid is not degenerate)
    engine.configure(config(1))
    _, img1, _ = engine.trace_frames([fr], results=False)
    assert np.abs(img1 - img).max() > 1e-3 * ref_img.max()


def test_multisample_refuses_per_ray_results_and_large_counts(engine):
    from sirius_b200.engine import SiriusError
    fr = abi.make_frame(abi.make_metric(a=0.5), abi.make_camera(r=30.0, width=8, height=8), 0.0, 20.0)
    engine.configure(config(4))
    with pytest.raises(SiriusError) as e:
        engine.trace_frames([fr], results=True)
    assert e.value.code == abi.ERR_INVALID_ARGUMENT
    with pytest.raises(SiriusError):
        engine.configure(config(5000))


def test_mixed_precision_multisample_within_the_image_bar(engine):
    fr = abi.make_frame(abi.make_metric(a=0.9), abi.make_camera(r=60.0, theta_deg=70.0, fov=30.0, width=48,
                                                                   height=48), 0.0, 20.0)
    imgs = {}
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        engine.configure(config(16, prec))
        _, imgs[prec], _ = engine.trace_frames([fr], results=False)
    ref = imgs[abi.PRECISION_FP64]
    assert np.abs(imgs[abi.PRECISION_MIXED] - ref).max() <= 1e-4 * ref.max()

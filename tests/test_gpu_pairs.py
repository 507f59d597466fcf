"""Two rays per thread (rays_per_thread = 2): the mixed-precision Kerr-Schild
kernel whose FP32 attempts run as packed pairs (f32x2).

Each packed operation is the same IEEE operation on each lane, so a ray's
result cannot depend on the ray it shares a thread with: a frame of odd width
traced whole and as row windows pairs its pixels differently (pixel 2i with
2i + 1 of the launch), and must give the same bits. Against the one-ray kernel
and the FP64 oracle the packed kernel meets the mixed-precision bars."""
import os

import numpy as np
import pytest

from oracle import compare
from sirius_b200 import abi

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def config(rays_per_thread, **kw):
    base = dict(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0, initial_step=0.1,
                escape_radius=200.0, horizon_factor=1.01, max_steps=10000, precision=abi.PRECISION_MIXED,
                enable_volumetric=1, n_bins=16, rays_per_thread=rays_per_thread)
    base.update(kw)
    return abi.default_config(**base)


def frame(w, h, **kw):
    cam = abi.make_camera(r=100.0, theta_deg=60.0, width=w, height=h, fov=30.0)
    return abi.make_frame(abi.make_metric(a=0.9), cam, 0.0, 30.0, **kw)


def test_pairing_does_not_change_a_ray(engine):
    engine.configure(config(2))
    full = frame(63, 40)
    res, img, spc = engine.trace_frames([full], spectra=True)
    parts = [engine.trace_frames([frame(63, 40, row_begin=r0, row_count=n)], spectra=True)
             for r0, n in ((0, 3), (3, 18), (21, 19))]
    assert np.concatenate([p[0] for p in parts]).tobytes() == res.tobytes()
    assert np.concatenate([p[1] for p in parts]).tobytes() == img.tobytes()
    assert np.concatenate([p[2] for p in parts]).tobytes() == spc.tobytes()


def test_packed_kernel_against_one_ray_kernel_and_oracle(engine, oracle):
    fr = frame(64, 64)
    engine.configure(config(1))
    _, img1, _ = engine.trace_frames([fr], results=False)
    engine.configure(config(2))
    res2, img2, spc2 = engine.trace_frames([fr], spectra=True)
    scale = img1.max()
    assert np.abs(img2.astype(np.float64) - img1).max() / scale <= 1e-4
    ref, bins = oracle.trace_frame(fr, config(1, precision=abi.PRECISION_FP64), threads=THREADS)
    rep = compare.report(res2, img2, ref, spc2, bins, escape_radius=200.0)
    print(compare.summary(rep))
    assert rep["outcome_agreement"] >= 0.99
    assert rep["image"]["max"] <= 1e-4
    assert rep["null_final"]["max"] <= 1e-8
    assert rep["escape_direction_rad"]["p99"] <= 1e-4


def test_autotuner_times_rays_per_thread(engine):
    engine.configure(config(0))
    cfg = engine.autotune([frame(128, 128)])
    assert cfg.rays_per_thread in (1, 2)
    with pytest.raises(Exception) as e:
        engine.configure(config(3))
    assert "rays_per_thread" in str(e.value)

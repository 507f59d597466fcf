"""CUDA engine vs the CPU oracle, through the C ABI (sm_100a kernels).

Tolerances: FP64 engine vs FP64 oracle — the same algorithm in the same
precision: identical outcomes and step counts except on rays whose histories
split at rounding level, terminal state ~1e-9; mixed precision (FP32 RHS, FP64
state and projection) — image L-infinity <= 1e-4 of the image scale, null
constraint of the returned state <= 1e-8."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def workload(prec, **kw):
    base = dict(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0, initial_step=0.1,
                escape_radius=200.0, horizon_factor=1.01, max_steps=10000, precision=prec)
    base.update(kw)
    return abi.default_config(**base)


def kerr_frame(w=48, h=48, a=0.9, th=60.0, r=100.0, rout=30.0):
    return abi.make_frame(abi.make_metric(a=a), abi.make_camera(r=r, theta_deg=th, width=w, height=h, fov=30.0),
                          0.0, rout)


def compare(res, img, ref, *, agree_min, img_rel, dir_tol):
    agree = res["outcome"] == ref["outcome"]
    assert agree.mean() >= agree_min, f"outcome agreement {agree.mean():.4f}"
    scale = float(ref["intensity"].max())
    err = np.abs(img.astype(np.float64) - ref["intensity"]) / scale
    assert np.percentile(err, 99.5) <= img_rel, f"image p99.5 {np.percentile(err, 99.5):.2e}"
    esc = agree & (ref["outcome"] == abi.ESCAPED)
    if esc.any():
        kg = res["final_k"][esc, 1:].astype(np.float64)
        ko = ref["final_k"][esc, 1:].astype(np.float64)
        kg /= np.linalg.norm(kg, axis=1, keepdims=True)
        ko /= np.linalg.norm(ko, axis=1, keepdims=True)
        d = np.linalg.norm(kg - ko, axis=1)
        assert np.percentile(d, 99) <= dir_tol, f"escape direction p99 {np.percentile(d, 99):.2e}"
    return err


# ------------------------------------------------------------ unit level ----
FAMILIES = [
    abi.make_metric(a=0.0), abi.make_metric(a=0.9), abi.make_metric(a=0.6, Q=0.5),
    abi.make_metric(a=0.7, Lambda=1e-4), abi.make_metric(family=abi.MORRIS_THORNE, b0=1.3),
    abi.make_metric(family=abi.MORRIS_THORNE, b0=0.8, shape=2), abi.make_metric(family=abi.ALCUBIERRE, vs=1.5),
]


def points_for(m, rng, n=256):
    if m.family == abi.MORRIS_THORNE:
        return np.stack([np.zeros(n), rng.uniform(1.2 * m.b0, 40, n), rng.uniform(0.2, np.pi - 0.2, n),
                         rng.uniform(0, 2 * np.pi, n)], 1)
    r = rng.uniform(0.3, 3.0, n) if m.family == abi.ALCUBIERRE else rng.uniform(1.6, 60, n)
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    return np.stack([np.zeros(n), r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], 1)


@pytest.mark.parametrize("mi", range(len(FAMILIES)))
def test_metric_and_dual_derivatives(engine, oracle, mi):
    """IMetric::evaluate on the device: FP64 and FP32 dual-number dg vs the oracle's analytic dg."""
    m = FAMILIES[mi]
    pts = points_for(m, np.random.default_rng(mi))
    g0, dg0 = oracle.metric_evaluate(m, pts)
    g, dg = engine.metric_evaluate(m, pts, abi.PRECISION_FP64)
    np.testing.assert_allclose(g, g0, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(dg, dg0, rtol=1e-10, atol=1e-12)
    gf, dgf = engine.metric_evaluate(m, pts, abi.PRECISION_MIXED)
    scale = np.abs(dg0).max()
    assert np.max(np.abs(dgf - dg0)) / scale < 2e-5
    np.testing.assert_allclose(gf, g0, rtol=2e-5, atol=2e-6)


def test_dp45_step_matches_oracle(engine, oracle):
    """Geodesic::integrateStepRK45 (engine semantics), one attempt per state, FP64."""
    m = abi.make_metric(a=0.9)
    cfg = workload(abi.PRECISION_FP64)
    engine.configure(cfg)
    rng = np.random.default_rng(2)
    states, hs = [], []
    cam = abi.make_camera(r=30.0, theta_deg=70.0, width=64, height=64, fov=60.0)
    for i in range(200):
        o, d = oracle.camera_ray(cam, int(rng.integers(64)), int(rng.integers(64)))
        x, p, _ = oracle.init_state(m, cfg, o, d)
        states.append(np.concatenate([x, p]))
        hs.append(rng.uniform(0.05, 3.0))
    s0, h0, a0, e0 = oracle.dp45_step(m, cfg, states, hs)
    s1, h1, a1, e1 = engine.dp45_step(m, states, hs)
    np.testing.assert_array_equal(a1, a0)
    # the error estimate is a cancelling sum: the two formulations agree to ~1e-6 of it
    np.testing.assert_allclose(e1, e0, rtol=1e-5, atol=1e-8)
    np.testing.assert_allclose(s1, s0, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(h1, h0, rtol=1e-12)


# ------------------------------------------------------------ frame level ---
def test_kerr_frame_fp64_matches_oracle(engine, oracle):
    fr = kerr_frame()
    cfg = workload(abi.PRECISION_FP64)
    engine.configure(cfg)
    res, img, _ = engine.trace_frames([fr])
    ref, _ = oracle.trace_frame(fr, cfg, threads=THREADS)
    compare(res, img, ref, agree_min=0.995, img_rel=1e-8, dir_tol=1e-8)
    assert (res["steps"] == ref["steps"]).mean() >= 0.98
    hit = (res["n_crossings"] > 0) & (ref["n_crossings"] > 0)
    np.testing.assert_allclose(res["disk_r"][hit, 0], ref["disk_r"][hit, 0], rtol=1e-6)
    np.testing.assert_allclose(res["disk_g"][hit, 0], ref["disk_g"][hit, 0], rtol=1e-6)
    assert res["null_final"].max() < 1e-12


def test_kerr_frame_mixed_matches_oracle(engine, oracle):
    """The north-star accuracy bar: image L-inf <= 1e-4 vs the FP64 oracle, null drift <= 1e-8."""
    fr = kerr_frame()
    cfg = workload(abi.PRECISION_MIXED)
    engine.configure(cfg)
    res, img, _ = engine.trace_frames([fr])
    ref, _ = oracle.trace_frame(fr, workload(abi.PRECISION_FP64), threads=THREADS)
    err = compare(res, img, ref, agree_min=0.99, img_rel=1e-4, dir_tol=1e-5)
    assert np.percentile(err, 99) <= 1e-5
    assert res["null_final"].max() <= 1e-8
    dE = np.abs(res["E"] - res["E0"]) / np.abs(res["E0"])
    assert dE.max() <= 1e-6


def test_schwarzschild_tight_tolerance_fp64(engine, oracle):
    """Schwarzschild, r_obs 50, incl 85 deg, rtol = atol = 1e-10, horizon 1.01 r_+, escape 1000 (a crop)."""
    fr = abi.make_frame(abi.make_metric(), abi.make_camera(r=50.0, theta_deg=85.0, width=32, height=32, fov=30.0),
                        6.0, 20.0)
    cfg = workload(abi.PRECISION_FP64, abs_tolerance=1e-10, rel_tolerance=1e-10, escape_radius=1000.0,
                   min_step=1e-12)
    engine.configure(cfg)
    res, img, _ = engine.trace_frames([fr])
    ref, _ = oracle.trace_frame(fr, cfg, threads=THREADS)
    compare(res, img, ref, agree_min=0.995, img_rel=1e-8, dir_tol=1e-8)


def test_volumetric_spectra(engine, oracle):
    fr = kerr_frame(w=24, h=24)
    for prec, tol in ((abi.PRECISION_FP64, 2e-5), (abi.PRECISION_MIXED, 2e-4)):
        cfg = workload(prec, enable_volumetric=1, n_bins=16)
        engine.configure(cfg)
        res, img, spc = engine.trace_frames([fr], spectra=True)
        ref, bins = oracle.trace_frame(fr, workload(abi.PRECISION_FP64, enable_volumetric=1, n_bins=16),
                                       threads=THREADS)
        agree = res["outcome"] == ref["outcome"]
        scale = bins.max(axis=0, keepdims=True)
        err = np.abs(spc[agree] - bins[agree]) / scale
        assert np.percentile(err, 99) <= tol, (prec, np.percentile(err, 99))
        assert bins.max() > 0


@pytest.mark.parametrize("name,metric,cam", [
    ("kerr_newman", abi.make_metric(a=0.6, Q=0.5), dict(r=60.0, theta_deg=75.0)),
    ("kerr_de_sitter", abi.make_metric(a=0.7, Lambda=1e-4), dict(r=60.0, theta_deg=75.0)),
    ("morris_thorne", abi.make_metric(family=abi.MORRIS_THORNE, b0=1.3), dict(r=30.0, theta_deg=80.0)),
    ("alcubierre", abi.make_metric(family=abi.ALCUBIERRE, vs=1.5, sigma=8.0, R=1.0), dict(r=20.0, theta_deg=80.0)),
])
def test_metric_families_fp64(engine, oracle, name, metric, cam):
    fr = abi.make_frame(metric, abi.make_camera(width=24, height=24, fov=40.0, **cam), 0.0, 25.0)
    cfg = workload(abi.PRECISION_FP64)
    engine.configure(cfg)
    res, img, _ = engine.trace_frames([fr])
    ref, _ = oracle.trace_frame(fr, cfg, threads=THREADS)
    agree = res["outcome"] == ref["outcome"]
    assert agree.mean() >= 0.99, name
    same = agree & (res["steps"] == ref["steps"])
    assert same.mean() >= 0.95, name
    np.testing.assert_allclose(res["final_x"][same], ref["final_x"][same], rtol=1e-7, atol=1e-7)
    np.testing.assert_allclose(res["E"], res["E0"], rtol=1e-6)


def test_heterogeneous_batch_equals_separate_frames(engine):
    """Frames of different families and resolutions in one launch give the
    per-frame results bit for bit (per-ray arithmetic is independent of scheduling)."""
    frames = [kerr_frame(w=20, h=20),
              abi.make_frame(abi.make_metric(family=abi.MORRIS_THORNE, b0=1.0), abi.make_camera(r=30, width=16, height=12), 0, 25),
              abi.make_frame(abi.make_metric(a=0.3, Q=0.2), abi.make_camera(r=40, theta_deg=45, width=8, height=24), 0, 25),
              abi.make_frame(abi.make_metric(family=abi.ALCUBIERRE, vs=0.5), abi.make_camera(r=20, width=12, height=12), 0, 25)]
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        engine.configure(workload(prec))
        res, img, _ = engine.trace_frames(frames)
        off = 0
        for f in frames:
            n = f.camera.width * f.camera.height
            r1, i1, _ = engine.trace_frames([f])
            assert r1.tobytes() == res[off:off + n].tobytes()
            assert i1.tobytes() == img[off:off + n].tobytes()
            off += n


def test_impact_parameter_grid_trace_rays(engine, oracle):
    """TSIN006A.cpp:88-130 through the GeodesicTracer::trace batch entry point."""
    m = abi.make_metric(a=0.0)
    rays = []
    for ib in range(10):
        b = 1.0 + 14.0 * ib / 9
        for ip in range(10):
            ph = 2 * math.pi * ip / 10
            rays.append(abi.CameraRay((C.c_double * 4)(0.0, 50.0, math.pi / 2, 0.0),
                                      (C.c_double * 4)(0.0, -1.0, 0.0, b / 50.0 * math.cos(ph))))
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        cfg = workload(prec, min_step=1e-8, max_step=0.1, initial_step=0.01, enable_disk=0, escape_radius=100.0,
                       horizon_factor=1.05)
        engine.configure(cfg)
        res = engine.trace_rays(m, rays, 6.0, 20.0)
        ref = oracle.trace_rays(m, rays, workload(abi.PRECISION_FP64, min_step=1e-8, max_step=0.1,
                                                  initial_step=0.01, enable_disk=0, escape_radius=100.0,
                                                  horizon_factor=1.05), 6.0, 20.0, threads=THREADS)
        np.testing.assert_array_equal(res["outcome"], ref["outcome"])
        esc = ref["outcome"] == abi.ESCAPED
        # |dr/r| < 1e-4 and |dtheta| < 1e-4 rad (TSIN006A.cpp:42-43) on the escape direction
        kg = res["final_k"][esc, 1:].astype(np.float64)
        ko = ref["final_k"][esc, 1:].astype(np.float64)
        ang = np.arccos(np.clip(np.sum(kg * ko, 1) / np.linalg.norm(kg, axis=1) / np.linalg.norm(ko, axis=1), -1, 1))
        assert ang.max() < 1e-4


# ------------------------------------------------------ full-size checks ----
def test_full_size_properties(engine):
    """1024^2 frames: for Schwarzschild the geometry (outcome and crossing
    radius) is symmetric under the left-right mirror of the image (phi -> -phi;
    the disk's rotation breaks the symmetry of the redshift only); repeated
    launches are bit-identical; every ray ends with a valid outcome and a null
    state (size-independent properties of the workload)."""
    fr = abi.make_frame(abi.make_metric(), abi.make_camera(r=100.0, theta_deg=60.0, width=1024, height=1024), 0.0,
                        30.0)
    engine.configure(workload(abi.PRECISION_MIXED))
    res, img, _ = engine.trace_frames([fr])
    res2, img2, _ = engine.trace_frames([fr])
    assert img.tobytes() == img2.tobytes()
    assert res.tobytes() == res2.tobytes()
    assert np.all(np.isin(res["outcome"], [abi.ESCAPED, abi.HORIZON, abi.DISK_HIT]))
    assert res["null_final"].max() <= 1e-8
    out = res["outcome"].reshape(1024, 1024)
    assert (out == out[:, ::-1]).mean() >= 0.999
    r0 = res["disk_r"][:, 0].reshape(1024, 1024)
    both = (r0 > 0) & (r0[:, ::-1] > 0)
    asym = np.abs(r0 - r0[:, ::-1])[both] / r0[both]
    assert np.percentile(asym, 99.9) < 1e-4


def test_kerr_full_frame_vs_fp64_engine(engine):
    """1024^2 Kerr a = 0.9: the mixed-precision image against the FP64 engine (the plain comparator)."""
    fr = kerr_frame(w=1024, h=1024)
    engine.configure(workload(abi.PRECISION_FP64))
    _, img64, _ = engine.trace_frames([fr], results=False)
    engine.configure(workload(abi.PRECISION_MIXED))
    _, img32, _ = engine.trace_frames([fr], results=False)
    err = np.abs(img32.astype(np.float64) - img64) / img64.max()
    assert np.percentile(err, 99.9) <= 1e-4
    assert np.percentile(err, 99) <= 1e-5


# ---------------------------------------------------------- error paths -----
def test_invalid_configuration_is_reported(engine):
    bad = workload(abi.PRECISION_MIXED, n_bins=64, enable_volumetric=1)
    with pytest.raises(Exception) as e:
        engine.configure(bad)
    assert "n_bins" in str(e.value)
    with pytest.raises(Exception):
        engine.configure(workload(abi.PRECISION_FP64, abs_tolerance=-1.0))
    engine.configure(workload(abi.PRECISION_FP64))
    bad_frame = kerr_frame(w=0, h=4)
    with pytest.raises(Exception):
        engine.trace_frames([bad_frame])
    # the handle stays usable
    res, _, _ = engine.trace_frames([kerr_frame(w=4, h=4)])
    assert len(res) == 16


def test_watchdog_bounds_a_launch(engine):
    """A launch that outlives watchdog_ms ends with SIRIUS_ERR_TIMEOUT and the
    context stays usable (the bound is a device-clock check, not a fault)."""
    from sirius_b200.engine import SiriusError
    engine.configure(workload(abi.PRECISION_FP64, watchdog_ms=1))
    with pytest.raises(SiriusError) as e:
        engine.trace_frames([kerr_frame(w=1024, h=1024)], results=False)
    assert e.value.code == abi.ERR_TIMEOUT
    engine.configure(workload(abi.PRECISION_FP64))
    res, _, _ = engine.trace_frames([kerr_frame(w=8, h=8)])
    assert np.all(res["steps"] > 0)


def test_register_budgets_agree(engine):
    """max_registers selects the trace kernel compiled for a register cap (255,
    168 or 128; 0 is the precision's default, 128 mixed and 255 FP64). The cap
    changes spills, not arithmetic: FP64 images are bit-identical; the mixed
    path's FP32 contractions may round differently, so its images agree within
    the FP32 right-hand side's error budget."""
    fr = kerr_frame(w=96, h=96)
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        imgs = {}
        for cap in (0, 255, 168, 128):
            engine.configure(workload(prec, max_registers=cap))
            _, imgs[cap], _ = engine.trace_frames([fr], results=False)
        for cap in (0, 168, 128):
            if prec == abi.PRECISION_FP64:
                np.testing.assert_array_equal(imgs[cap], imgs[255])
            else:
                err = np.abs(imgs[cap].astype(np.float64) - imgs[255]) / imgs[255].max()
                assert err.max() <= 1e-4, err.max()
    with pytest.raises(Exception) as e:
        engine.configure(workload(abi.PRECISION_MIXED, max_registers=5))
    assert "max_registers" in str(e.value)


def test_autotune_and_peaks(engine):
    engine.configure(workload(abi.PRECISION_MIXED))
    cfg = engine.autotune([kerr_frame(w=128, h=128)])
    assert 0 <= cfg.blocks_per_sm <= 4 and 1 <= cfg.refill_threshold <= 32
    assert cfg.max_registers in (0, 255, 168, 128)
    assert engine.fma_peak(1) > 1e13 and engine.fma_peak(0) > 5e12

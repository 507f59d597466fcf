"""Pin the CPU oracle against the reference's own outputs (tests/golden/, made
by tests/golden/make_golden.py from the reference's compiled CPU code) and,
when the compiled reference is present, against fresh runs of it."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden
from sirius_b200 import abi


def compat_config(cfg_tuple):
    """Engine config carrying the reference TracerConfig values of a golden frame."""
    (esc, hf, max_steps, en_disk, din, dout, tin, en_vol, atol, rtol, hmin, hmax, h0, safety, grow, shrink) = cfg_tuple
    c = abi.default_config(escape_radius=esc, horizon_factor=hf, max_steps=int(max_steps), enable_disk=int(en_disk),
                           disk_temperature_inner=tin, enable_volumetric=int(en_vol), abs_tolerance=atol,
                           rel_tolerance=rtol, min_step=hmin, max_step=hmax, initial_step=h0, safety_factor=safety,
                           step_grow_max=grow, step_shrink_min=shrink, compat=1, spiral_check=1)
    return c, din, dout


def test_ks_metric_matches_reference(oracle):
    """KerrSchildFamily::evaluate (PHMT100A.h:248-396): g and the analytic dg."""
    d = golden("ks_metric.npz")
    for i, (M, a, Q, L) in enumerate(d["params"]):
        g, dg = oracle.metric_evaluate(abi.make_metric(M=M, a=a, Q=Q, Lambda=L), d["points"])
        np.testing.assert_allclose(g, d["g"][i], rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(dg, d["dg"][i], rtol=1e-11, atol=1e-13)


def test_camera_matches_reference(oracle):
    """PinholeCamera::generateRay (CMBS001A.h:120-185): float arithmetic reproduced exactly."""
    d = golden("camera.npz")
    for row, (ci, px, py) in enumerate(zip(d["idx"], d["px"], d["py"])):
        r, th, ph, fov, w, h, yaw, pitch, roll = d["cam"][int(ci)]
        cam = abi.Camera(0.0, r, th, ph, yaw, pitch, roll, fov, int(w), int(h), 0, 0)
        o, dd = oracle.camera_ray(cam, int(px), int(py))
        np.testing.assert_array_equal(o, d["origin"][row])
        np.testing.assert_array_equal(dd, d["dir"][row])


def test_rk45_step_matches_reference(oracle):
    """Geodesic::integrateStepRK45 (PHGD001A.cpp:530-641) as written, one call per state."""
    d = golden("rk45_step.npz")
    atol, rtol, hmin, hmax, h0, safety, grow, shrink = d["cfg"]
    cfg = abi.default_config(abs_tolerance=atol, rel_tolerance=rtol, min_step=hmin, max_step=hmax, initial_step=h0,
                             safety_factor=safety, step_grow_max=grow, step_shrink_min=shrink, compat=1)
    met = abi.make_metric(M=float(d["M"]), a=float(d["a"]))
    pos, vel, h, ok, term = oracle.rk45_step_compat(met, cfg, d["pos_in"], d["vel_in"], d["h_in"])
    np.testing.assert_array_equal(ok, d["success"])
    np.testing.assert_array_equal(term, d["terminated"])
    np.testing.assert_array_equal(h, d["h_out"])
    np.testing.assert_array_equal(pos, d["pos_out"])
    np.testing.assert_array_equal(vel, d["vel_out"])


@pytest.mark.parametrize("name", ["kerr_session", "schw_session", "schw_tight", "schw_default", "kerr_volumetric"])
def test_trace_matches_reference(oracle, name):
    """GeodesicTracer::trace (GTRC001A.cpp:139-592) with the reference's semantics, bit for bit."""
    d = golden(f"trace_{name}.npz")
    rec = d["records"]
    r, th, ph, fov, w, h = d["camera"]
    M, a = d["metric"]
    cfg, din, dout = compat_config(d["cfg"])
    cam = abi.Camera(0.0, r, th, ph, 0.0, 0.0, 0.0, fov, int(w), int(h), 0, 0)
    fr = abi.make_frame(abi.make_metric(M=M, a=a), cam, disk_inner=din, disk_outer=dout)
    res, _ = oracle.trace_frame(fr, cfg, threads=4)
    np.testing.assert_array_equal(res["outcome"], rec["outcome"])
    np.testing.assert_array_equal(res["steps"], rec["steps_taken"])
    np.testing.assert_array_equal(res["n_crossings"], rec["num_disk_crossings"])
    np.testing.assert_array_equal(res["equatorial_crossings"], rec["equatorial_crossings"])
    np.testing.assert_array_equal(res["image_order"], rec["image_order"])
    np.testing.assert_array_equal(res["total_phi_change"], rec["total_phi_change"])
    np.testing.assert_array_equal(res["min_radius"], rec["min_radius"])
    np.testing.assert_array_equal(res["magnification"], rec["magnification"])
    np.testing.assert_array_equal(res["impact_parameter"], rec["impact_parameter"])
    np.testing.assert_array_equal((res["flags"] & abi.FLAG_PHOTON_RING) != 0, rec["photon_ring"] != 0)
    n = rec["num_disk_crossings"]
    for j in range(4):
        m = n > j
        np.testing.assert_array_equal(res["disk_r"][m, j], rec["disk_r"][m, j])
        np.testing.assert_array_equal(res["disk_phi"][m, j], rec["disk_phi"][m, j])
        np.testing.assert_array_equal(res["disk_g"][m, j], rec["disk_redshift"][m, j])
    # terminal state of escaped/horizon rays (TraceResult::final_position/direction)
    esc = rec["outcome"] == abi.ESCAPED
    np.testing.assert_array_equal(res["final_x"][esc], rec["final_position"][esc])
    np.testing.assert_array_equal(res["final_k"][esc], rec["final_direction"][esc].astype(np.float32))
    hor = rec["outcome"] == abi.HORIZON
    np.testing.assert_array_equal(res["final_x"][hor], rec["final_position"][hor])
    if name == "kerr_volumetric":
        np.testing.assert_array_equal(res["optical_depth"], rec["optical_depth"])


def test_tight_tolerance_finding(oracle):
    """At rtol = atol = 1e-10 every reference ray stops as MAX_STEPS after a
    rejected first step (GTRC001A.cpp:272-277); the engine semantics retry
    and finish the same rays (the reason the oracle's engine mode exists)."""
    d = golden("trace_schw_tight.npz")
    rec = d["records"]
    assert np.all(rec["outcome"] == abi.MAX_STEPS)
    assert rec["steps_taken"].max() < 10
    r, th, ph, fov, w, h = d["camera"]
    cfg, din, dout = compat_config(d["cfg"])
    cfg.compat = 0
    cfg.spiral_check = 0
    cfg.min_step = 1e-12
    cam = abi.Camera(0.0, r, th, ph, 0.0, 0.0, 0.0, fov, int(w), int(h), 0, 0)
    res, _ = oracle.trace_frame(abi.make_frame(abi.make_metric(), cam, din, dout), cfg, threads=4)
    assert np.all(np.isin(res["outcome"], [abi.ESCAPED, abi.HORIZON, abi.DISK_HIT]))


def test_isco_matches_reference(oracle):
    """AccretionDiskD::computeISCO (PHAD001A.h:88-105)."""
    d = golden("isco.npz")
    for s, v in zip(d["spin"], d["isco"]):
        assert oracle.isco(float(s)) == pytest.approx(float(v), rel=1e-15, abs=1e-15)


def test_live_reference_random_rays(oracle):
    """When the compiled reference is present (it travels with the repository
    snapshot), trace fresh seeded random camera rays through both."""
    from oracle.pyoracle import Reference, ref_available, ref_config_from
    if not ref_available():
        pytest.skip("reference library not built here")
    ref = Reference()
    rng = np.random.default_rng(7)
    for a in (0.0, 0.6, -0.95):
        n = 64
        origins = np.zeros((n, 4))
        origins[:, 1] = rng.uniform(15, 80, n)
        origins[:, 2] = np.radians(rng.uniform(20, 160, n))
        origins[:, 3] = rng.uniform(0, 2 * np.pi, n)
        dirs = rng.normal(size=(n, 4))
        dirs[:, 0] = 0
        dirs[:, 1] = -np.abs(dirs[:, 1]) * 3
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        cfg = abi.default_config(compat=1, spiral_check=1)
        din = oracle.isco(a)
        recs = ref.trace_rays(1.0, a, ref_config_from(cfg, din, 20.0), origins, dirs, threads=4)
        rays = [abi.CameraRay((C.c_double * 4)(*o), (C.c_double * 4)(*dd)) for o, dd in zip(origins, dirs)]
        res = oracle.trace_rays(abi.make_metric(a=a), rays, cfg, din, 20.0, threads=4)
        np.testing.assert_array_equal(res["outcome"], recs["outcome"])
        np.testing.assert_array_equal(res["steps"], recs["steps_taken"])
        esc = recs["outcome"] == abi.ESCAPED
        np.testing.assert_array_equal(res["final_x"][esc], recs["final_position"][esc])


def test_subpixel_camera_matches_reference(oracle):
    """PinholeCamera::generateRay(x, y, u, v) (CMBS001A.h:120) at sub-pixel positions, bit for bit."""
    d = golden("camera_uv.npz")
    r, th, ph, fov, w, h, yaw, pitch, roll = d["cam"]
    cam = abi.Camera(0.0, r, th, ph, yaw, pitch, roll, fov, int(w), int(h), 0, 0)
    for i in range(len(d["px"])):
        o, dd = oracle.camera_ray(cam, int(d["px"][i]), int(d["py"][i]), float(d["u"][i]), float(d["v"][i]))
        np.testing.assert_array_equal(o, d["origin"][i])
        np.testing.assert_array_equal(dd, d["dir"][i])

"""Beams (sirius_cuda_trace_beams): the magnification of each escaped pixel
ray from its two tangent vectors integrated along it, against finite
differences of neighbouring rays traced independently by the FP64 oracle
(pixel offsets of 1e-3 on each side, the camera mapping evaluated in FP64).

Tolerances: the tangents are central differences of the right-hand side
(relative error ~1e-10) integrated with the ray's own steps; the oracle's
neighbours are separate rays at tolerance 1e-11 whose escape directions are
differenced over 2e-3 pixels, good to ~1e-5 relative. Rays grazing the shadow
are strongly magnified and sensitive, so the comparison asks the median and
the 90th percentile."""
import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def config(tol=1e-10):
    return abi.default_config(abs_tolerance=tol, rel_tolerance=tol, min_step=1e-12, max_step=5.0, initial_step=0.1,
                              escape_radius=2000.0, horizon_factor=1.01, max_steps=100000,
                              precision=abi.PRECISION_FP64, enable_disk=0)


def escape_dir(oracle, met, rec):
    g, _ = oracle.metric_evaluate(met, np.asarray(rec["final_x"], dtype=np.float64))
    k = np.linalg.solve(np.asarray(g).reshape(4, 4), np.asarray(rec["final_p"], dtype=np.float64))
    n = k[1:4]
    return n / np.linalg.norm(n)


def fd_magnification(oracle, met, cam, u, v, cfg, h=1e-3):
    rays = []
    for du, dv in ((h, 0), (-h, 0), (0, h), (0, -h), (0, 0)):
        o, d = oracle.camera_ray_exact(cam, u + du, v + dv)
        r = abi.CameraRay()
        r.origin[:] = list(o)
        r.direction[:] = list(d)
        rays.append(r)
    out = oracle.trace_rays(met, rays, cfg, disk_inner=0.0, disk_outer=20.0)
    if not np.all(out["outcome"] == abi.ESCAPED):
        return None
    n = [escape_dir(oracle, met, out[i]) for i in range(5)]
    dn_u, dn_v = (n[0] - n[1]) / (2 * h), (n[2] - n[3]) / (2 * h)
    dd = []
    for du, dv in ((h, 0), (-h, 0), (0, h), (0, -h)):
        dd.append(np.array(oracle.camera_ray_exact(cam, u + du, v + dv)[1][1:4]))
    dd_u, dd_v = (dd[0] - dd[1]) / (2 * h), (dd[2] - dd[3]) / (2 * h)
    d0 = np.array(oracle.camera_ray_exact(cam, u, v)[1][1:4])
    ci, cs = np.cross(dd_u, dd_v), np.cross(dn_u, dn_v)
    mu = np.linalg.norm(ci) / np.linalg.norm(cs)
    parity = np.sign(ci @ d0) * np.sign(cs @ n[4])
    return mu, parity, n[4]


def test_flat_space_has_unit_magnification(engine):
    fr = abi.make_frame(abi.make_metric(M=0.0, a=0.0), abi.make_camera(r=30.0, theta_deg=60.0, fov=50.0, width=16,
                                                                         height=12, yaw=0.2, roll=0.1), 0.0, 20.0)
    engine.configure(config())
    b = engine.trace_beams([fr])
    assert np.all(b["outcome"] == abi.ESCAPED)
    np.testing.assert_allclose(b["magnification"], 1.0, rtol=1e-6)
    assert np.all(b["parity"] == 1.0)


@pytest.mark.parametrize("a", [0.0, 0.9])
def test_magnification_matches_neighbouring_rays(engine, oracle, a):
    met = abi.make_metric(a=a)
    cam = abi.make_camera(r=40.0, theta_deg=80.0, fov=40.0, width=20, height=16)
    fr = abi.make_frame(met, cam, 0.0, 20.0)
    engine.configure(config())
    b = engine.trace_beams([fr])
    ocfg = config(1e-11)
    rel, signs, seen, dirs = [], [], 0, []
    for idx in range(0, cam.width * cam.height, 3):
        if b["outcome"][idx] != abi.ESCAPED:
            continue
        u, v = idx % cam.width + 0.5, idx // cam.width + 0.5
        r = fd_magnification(oracle, met, cam, u, v, ocfg)
        if r is None:
            continue
        seen += 1
        mu, par, n = r
        rel.append(abs(b["magnification"][idx] - mu) / mu)
        signs.append(b["parity"][idx] == par)
        dirs.append(np.abs(b["final_dir"][idx] - n).max())
    assert seen > 40
    rel = np.array(rel)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert np.percentile(rel, 90) < 1e-2, np.percentile(rel, 90)
    assert np.mean(signs) > 0.97
    assert np.median(dirs) < 1e-5


def test_beams_refuse_other_families(engine):
    from sirius_b200.engine import SiriusError
    engine.configure(config())
    mt = abi.make_frame(abi.make_metric(family=abi.MORRIS_THORNE, b0=1.0), abi.make_camera(r=20.0, width=4, height=4),
                        0.0, 20.0)
    with pytest.raises(SiriusError) as e:
        engine.trace_beams([mt])
    assert e.value.code == abi.ERR_UNSUPPORTED

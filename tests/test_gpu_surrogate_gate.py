"""The surrogate's gate against the analytic critical curve, computed on the
CPU independently of the device: every pixel whose celestial coordinates
(alpha, beta) lie within the gate band of the Bardeen (1973) curve is
integrated, and no pixel well outside the band is gated.

The celestial coordinates come from the oracle's initial state of each pixel's
ray (alpha = -L_z / (E sin theta_o), beta = p_theta / E); the curve is the
family of spherical photon orbits, sampled densely in r and resampled at
equal arc length, so that the CPU distance is good to 1e-3 M. The device
gate uses a 256-point polygon of the same curve in FP32; pixels within
`SHELL` of the band edge may fall either way."""
import numpy as np
import pytest

from sirius_b200 import abi

BAND = 0.3
SHELL = 0.01


def spherical_orbit_constants(a, M, r):
    """xi = L/E and eta = Q/E^2 of the spherical photon orbit at radius r."""
    xi = (r * r * (3.0 * M - r) - a * a * (r + M)) / (a * (r - M))
    eta = r ** 3 * (4.0 * a * a * M - r * (r - 3.0 * M) ** 2) / (a * a * (r - M) ** 2)
    return xi, eta


def critical_curve(a, M, theta_o, n=20000, spacing=1e-3):
    """Closed polygon of the critical curve in the (alpha, beta) plane, points
    at most `spacing` apart."""
    so, co = np.sin(theta_o), np.cos(theta_o)
    if abs(a) < 1e-6 * M:
        t = np.linspace(0.0, 2.0 * np.pi, int(2 * np.pi * np.sqrt(27.0) * M / spacing) + 1)
        return np.stack([np.sqrt(27.0) * M * np.cos(t), np.sqrt(27.0) * M * np.sin(t)], axis=1)
    s = min(abs(a) / M, 1.0)
    r_pro = 2.0 * M * (1.0 + np.cos(2.0 / 3.0 * np.arccos(-s)))
    r_ret = 2.0 * M * (1.0 + np.cos(2.0 / 3.0 * np.arccos(s)))
    r = np.linspace(r_pro, r_ret, n)
    xi, eta = spherical_orbit_constants(a, M, r)
    b2 = eta + a * a * co * co - xi * xi * (co / so) ** 2
    ok = b2 >= 0.0
    al, be = -xi[ok] / so, np.sqrt(b2[ok])
    upper = np.stack([al, be], axis=1)
    lower = np.stack([al[::-1], -be[::-1]], axis=1)
    poly = np.concatenate([upper, lower, upper[:1]])
    # resample every edge so that no two consecutive points are more than `spacing` apart
    out = [poly[:1]]
    for p0, p1 in zip(poly[:-1], poly[1:]):
        k = max(1, int(np.ceil(np.hypot(*(p1 - p0)) / spacing)))
        w = np.arange(1, k + 1)[:, None] / k
        out.append(p0 + w * (p1 - p0))
    return np.concatenate(out)


def celestial(oracle, frame, cfg):
    """(alpha, beta) per pixel from the oracle's initial states, and the
    camera's Boyer-Lindquist polar angle."""
    m, cam = frame.metric, frame.camera
    n = cam.width * cam.height
    al, be = np.zeros(n), np.zeros(n)
    theta_o = None
    for idx in range(n):
        o, d = oracle.camera_ray(cam, idx % cam.width, idx // cam.width)
        x, p, _ = oracle.init_state(m, cfg, o, d)
        if theta_o is None:
            X, Y, Z = x[1:4]
            R2m = X * X + Y * Y + Z * Z - m.a * m.a
            rk = np.sqrt(0.5 * (R2m + np.sqrt(R2m * R2m + 4.0 * m.a * m.a * Z * Z)))
            theta_o = np.arccos(np.clip(Z / rk, -1.0, 1.0))
        r, _ = oracle.radial(m, x)
        E, L = -p[0], x[1] * p[2] - x[2] * p[1]
        ct = np.clip(x[3] / r, -1.0, 1.0)
        st = np.sqrt(max(1.0 - ct * ct, 1e-30))
        pth = (ct / st) * (x[1] * p[1] + x[2] * p[2]) - r * st * p[3]
        al[idx] = -L / (E * max(np.sin(theta_o), 1e-6))
        be[idx] = pth / E
    return al, be, theta_o


def test_curve_reduces_to_the_schwarzschild_circle():
    c = critical_curve(0.0, 1.0, 1.0)
    np.testing.assert_allclose(np.hypot(c[:, 0], c[:, 1]), np.sqrt(27.0), rtol=1e-12)
    # Kerr: each orbit is a double root of the radial potential
    # R(r) = (r^2 + a^2 - a xi)^2 - Delta (eta + (xi - a)^2)
    a, M = 0.9, 1.0
    r = np.linspace(1.56, 3.9, 50)
    xi, eta = spherical_orbit_constants(a, M, r)
    R = (r * r + a * a - a * xi) ** 2 - (r * r - 2 * M * r + a * a) * (eta + (xi - a) ** 2)
    dR = 4 * r * (r * r + a * a - a * xi) - (2 * r - 2 * M) * (eta + (xi - a) ** 2)
    scale = (r * r + a * a) ** 2
    assert np.abs(R / scale).max() < 1e-12 and np.abs(dR / scale).max() < 1e-12
    # the inclined curve closes on itself and spans the prograde/retrograde extremes
    k = critical_curve(a, M, np.radians(60.0))
    assert np.hypot(*(k[0] - k[-1])) < 1e-12
    assert np.all(np.hypot(*np.diff(k, axis=0).T) <= 1e-3 + 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("a,theta,fov", [(0.9, 60.0, 15.0), (0.5, 85.0, 15.0), (0.0, 30.0, 15.0),
                                          (-0.7, 75.0, 18.0)])
def test_gate_matches_the_analytic_critical_curve(engine, oracle, a, theta, fov):
    from scipy.spatial import cKDTree
    engine.surrogate_load(np.load(_weights()))
    side = 192
    cam = abi.make_camera(r=100.0, theta_deg=theta, width=side, height=side, fov=fov)
    fr = abi.make_frame(abi.make_metric(a=a), cam, 0.0, 30.0)
    cfg = abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                             initial_step=0.1, escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                             precision=abi.PRECISION_MIXED, enable_disk=1, enable_volumetric=0,
                             critical_band=0.0)
    engine.configure(cfg)
    _, _, gate, st = engine.render_surrogate([fr], config=abi.surrogate_config(gate_band=BAND, audit_fraction=0.0, inner_gate=-1.0))
    al, be, theta_o = celestial(oracle, fr, cfg)
    curve = critical_curve(a, 1.0, theta_o)
    dist, _ = cKDTree(curve).query(np.stack([al, be], axis=1))
    inside, outside = dist < BAND - SHELL, dist > BAND + SHELL
    gated = gate == 1
    assert inside.sum() > 500, inside.sum()
    assert np.all(gated[inside]), np.flatnonzero(inside & ~gated)[:10]
    assert not np.any(gated[outside]), np.flatnonzero(outside & gated)[:10]
    assert not np.any(gate == 2)
    assert st.integrated == int(gated.sum())


def _weights():
    import os
    return os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sirius_b200", "data",
                        "surrogate_kerr.npy")

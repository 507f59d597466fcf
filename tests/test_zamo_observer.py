"""The zero-angular-momentum observer (camera observer SIRIUS_OBSERVER_ZAMO).

CPU: the Bardeen (1972) tetrad restated here in Boyer-Lindquist coordinates
has the properties the reference's FIDO tests check (TSCM005A.cpp:84-311):
rho, Delta, lapse below 1 and tending to 1, no frame dragging without spin,
an orthonormal basis, a subluminal circular-orbit speed.

GPU: every ray of a ZAMO frame starts with the constants of motion of
p = e_(t) + n^i e_(i) built here independently in Boyer-Lindquist
coordinates from the same pixel direction n (E, L_z, Carter Q); disk
redshifts follow g = 1 / (u^t (E - Omega L)) (observer frequency 1); the
mixed-precision image agrees with the FP64 one; the observer is refused where
it is not defined."""
import numpy as np
import pytest

from sirius_b200 import abi


def bl_metric(M, a, Q, r, th):
    rho2 = r * r + a * a * np.cos(th) ** 2
    D = r * r - 2 * M * r + a * a + Q * Q
    s2 = np.sin(th) ** 2
    w = 2 * M * r - Q * Q
    g = np.zeros((4, 4))
    g[0, 0] = -(1 - w / rho2)
    g[0, 3] = g[3, 0] = -a * s2 * w / rho2
    g[1, 1] = rho2 / D
    g[2, 2] = rho2
    g[3, 3] = (r * r + a * a + a * a * s2 * w / rho2) * s2
    return g


def zamo(M, a, Q, r, th):
    """(rho, Delta, alpha, omega, varpi, tetrad rows e_(t), e_(r), e_(theta), e_(phi))."""
    st, ct = np.sin(th), np.cos(th)
    rho = np.sqrt(r * r + a * a * ct * ct)
    D = r * r - 2 * M * r + a * a + Q * Q
    Sig = np.sqrt((r * r + a * a) ** 2 - a * a * D * st * st)
    alpha = rho * np.sqrt(D) / Sig
    omega = a * (2 * M * r - Q * Q) / Sig ** 2
    varpi = Sig * st / rho
    e = np.array([[1 / alpha, 0, 0, omega / alpha], [0, np.sqrt(D) / rho, 0, 0], [0, 0, 1 / rho, 0],
                  [0, 0, 0, 1 / varpi]])
    return rho, D, alpha, omega, varpi, e


def circular_speed(M, a, r, th=np.pi / 2):
    """Prograde circular geodesic speed relative to the ZAMO, (varpi / alpha)(Omega - omega)."""
    _, _, alpha, omega, varpi, _ = zamo(M, a, 0.0, r, th)
    Om = np.sqrt(M) / (r ** 1.5 + a * np.sqrt(M))
    return varpi / alpha * (Om - omega)


def test_fido_quantities_follow_the_reference_checks():
    M = 1.0
    rho, D, alpha, omega, varpi, e = zamo(M, 0.0, 0.0, 10.0, np.pi / 2)
    assert abs(rho - 10.0) < 1e-12 and abs(D - 80.0) < 1e-12 and abs(omega) < 1e-15
    assert abs(alpha - np.sqrt(1 - 2 / 10.0)) < 1e-12
    assert zamo(M, 0.9, 0.0, 6.0, 1.0)[3] > zamo(M, 0.3, 0.0, 6.0, 1.0)[3] > 0
    assert 0 < zamo(M, 0.9, 0.0, 4.0, 1.2)[2] < 1
    assert zamo(M, 0.9, 0.0, 1e4, 1.2)[2] > 0.999
    for a in (0.0, 0.5, 0.99):
        for r, th in ((3.5, 0.7), (12.0, np.pi / 2), (60.0, 2.5)):
            e = zamo(M, a, 0.2, r, th)[5]
            G = e @ bl_metric(M, a, 0.2, r, th) @ e.T
            np.testing.assert_allclose(G, np.diag([-1.0, 1.0, 1.0, 1.0]), atol=1e-12)
    assert -1 < circular_speed(M, 0.9, 6.0) < 1
    assert abs(circular_speed(M, 0.9, 4.0)) > abs(circular_speed(M, 0.9, 40.0))
    assert 0 < circular_speed(M, 0.0, 10.0) < 0.5


def expected_constants(oracle, frame):
    """E, L_z and Carter Q per pixel of p = e_(t) + n^i e_(i) (Boyer-Lindquist)."""
    m, cam = frame.metric, frame.camera
    th = np.clip(cam.theta, 0.01, np.pi - 0.01)
    e = zamo(m.M, m.a, m.Q, cam.r, th)[5]
    g = bl_metric(m.M, m.a, m.Q, cam.r, th)
    out = []
    for py in range(cam.height):
        for px in range(cam.width):
            _, d = oracle.camera_ray(cam, px, py)
            n = np.array(d[1:4])
            pu = e[0] + n[0] * e[1] + n[1] * e[2] + n[2] * e[3]
            p = g @ pu
            E, L, pth = -p[0], p[3], p[2]
            Qc = pth ** 2 + np.cos(th) ** 2 * (L * L / np.sin(th) ** 2 - m.a ** 2 * E * E)
            out.append((E, L, Qc))
    return np.array(out)


def zamo_frame(a=0.9, Q=0.0, r=30.0, theta_deg=70.0, w=40, h=32, fov=40.0, phi=0.4):
    met = abi.make_metric(a=a)
    met.Q = Q
    cam = abi.make_camera(r=r, theta_deg=theta_deg, phi=phi, width=w, height=h, fov=fov,
                          observer=abi.OBSERVER_ZAMO)
    return abi.make_frame(met, cam, 0.0, 20.0)


def config(prec):
    return abi.default_config(abs_tolerance=1e-10, rel_tolerance=1e-10, min_step=1e-9, max_step=2.0,
                              escape_radius=300.0, horizon_factor=1.01, max_steps=20000, precision=prec)


@pytest.mark.gpu
@pytest.mark.parametrize("a,Q", [(0.9, 0.0), (0.6, 0.4), (0.0, 0.0)])
def test_initial_constants_match_the_boyer_lindquist_tetrad(engine, oracle, a, Q):
    fr = zamo_frame(a=a, Q=Q)
    engine.configure(config(abi.PRECISION_FP64))
    res, _, _ = engine.trace_frames([fr], results=True)
    ref = expected_constants(oracle, fr)
    np.testing.assert_allclose(res["E0"], ref[:, 0], rtol=2e-6)
    np.testing.assert_allclose(res["Lz0"], ref[:, 1], rtol=2e-6, atol=2e-6 * np.abs(ref[:, 1]).max())
    np.testing.assert_allclose(res["Carter0"], ref[:, 2], rtol=2e-5, atol=2e-5 * np.abs(ref[:, 2]).max())
    # conserved along the trace, and null
    np.testing.assert_allclose(res["E"], res["E0"], rtol=1e-6)
    assert np.all(res["null_final"] < 1e-8)


@pytest.mark.gpu
def test_disk_redshift_relative_to_the_zamo(engine):
    fr = zamo_frame(a=0.9, r=40.0, theta_deg=80.0, w=48, h=48, fov=30.0)
    engine.configure(config(abi.PRECISION_FP64))
    res, _, _ = engine.trace_frames([fr], results=True)
    hit = res["n_crossings"] >= 1
    assert hit.sum() > 100
    r = res["disk_r"][hit, 0].astype(np.float64)
    E, L = res["E0"][hit].astype(np.float64), res["Lz0"][hit].astype(np.float64)
    a, M = 0.9, 1.0
    Om = np.sqrt(M) / (r ** 1.5 + a * np.sqrt(M))
    ut = (r ** 1.5 + a * np.sqrt(M)) / (r ** 0.75 * np.sqrt(r ** 1.5 - 3 * M * np.sqrt(r) + 2 * a * np.sqrt(M)))
    g = 1.0 / (ut * (E - Om * L))
    np.testing.assert_allclose(res["disk_g"][hit, 0], g, rtol=1e-4)


@pytest.mark.gpu
def test_mixed_precision_image_matches_fp64(engine):
    fr = zamo_frame(a=0.9, r=60.0, theta_deg=75.0, w=64, h=64, fov=30.0)
    imgs = {}
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        engine.configure(config(prec))
        _, imgs[prec], _ = engine.trace_frames([fr], results=False)
    ref = imgs[abi.PRECISION_FP64]
    assert ref.max() > 0
    assert np.abs(imgs[abi.PRECISION_MIXED] - ref).max() <= 1e-4 * ref.max()


@pytest.mark.gpu
def test_observer_is_refused_where_undefined(engine):
    from sirius_b200.engine import SiriusError
    engine.configure(config(abi.PRECISION_FP64))
    mt = abi.make_frame(abi.make_metric(family=abi.MORRIS_THORNE, b0=1.0),
                        abi.make_camera(r=20.0, width=8, height=8, observer=abi.OBSERVER_ZAMO), 0.0, 20.0)
    with pytest.raises(SiriusError) as e:
        engine.trace_frames([mt], results=False)
    assert e.value.code == abi.ERR_UNSUPPORTED
    inside = zamo_frame(a=0.5, r=1.5, w=8, h=8)
    with pytest.raises(SiriusError) as e:
        engine.trace_frames([inside], results=False)
    assert e.value.code == abi.ERR_INVALID_ARGUMENT
    bad = zamo_frame(w=8, h=8)
    bad.camera.observer = 7
    with pytest.raises(SiriusError):
        engine.trace_frames([bad], results=False)

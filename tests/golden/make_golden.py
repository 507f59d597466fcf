"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference's CPU implementation of the path (GeodesicTracer,
Geodesic::integrateStepRK45, KerrSchildFamily::evaluate, PinholeCamera,
AccretionDiskD::computeISCO), compiled from its sources by oracle/Makefile into
oracle/_ref/libsirius_ref.so, on fixed seeded inputs, and stores inputs and
outputs as .npz. The fixtures pin the CPU oracle (oracle/oracle.hpp) in
tests/test_oracle_pin.py; nothing at test time needs the reference sources.

Usage:  make -C oracle && python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Reference, RefTracerConfig  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def ks_points(rng, n):
    # Cartesian points from r ~ 1.2 .. 60 at all angles, plus points near the equator and the axis
    r = np.exp(rng.uniform(np.log(1.2), np.log(60.0), n))
    th = np.arccos(rng.uniform(-1, 1, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    pts = np.stack([rng.uniform(0, 10, n), r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph),
                    r * np.cos(th)], axis=1)
    pts[: n // 8, 3] = rng.uniform(-1e-3, 1e-3, n // 8)  # near the equatorial plane
    return pts


def main():
    ref = Reference()
    rng = np.random.default_rng(20261203)

    # 1. KerrSchildFamily::evaluate over (M, a, Q, Lambda) combinations
    params = np.array([[1.0, 0.0, 0.0, 0.0], [1.0, 0.9, 0.0, 0.0], [1.0, 0.998, 0.0, 0.0], [1.0, 0.5, 0.5, 0.0],
                       [1.0, 0.3, 0.0, 1e-4], [2.0, -0.7, 0.2, 0.0]])
    pts = ks_points(rng, 128)
    G = np.zeros((len(params), len(pts), 4, 4))
    DG = np.zeros((len(params), len(pts), 4, 4, 4))
    for i, (M, a, Q, L) in enumerate(params):
        G[i], DG[i] = ref.ks_evaluate(M, a, Q, L, pts)
    np.savez_compressed(os.path.join(OUT, "ks_metric.npz"), params=params, points=pts, g=G, dg=DG)

    # 2. PinholeCamera::generateRay
    from sirius_b200 import abi
    cams = [abi.make_camera(r=50.0, theta_deg=85.0, fov=30.0, width=256, height=256),
            abi.make_camera(r=100.0, theta_deg=60.0, fov=30.0, width=1024, height=1024),
            abi.make_camera(r=20.0, theta_deg=30.0, fov=45.0, width=320, height=200, yaw=0.1, pitch=-0.2, roll=0.3)]
    cam_rows = []
    for ci, cam in enumerate(cams):
        px = rng.integers(0, cam.width, 64).astype(np.int32)
        py = rng.integers(0, cam.height, 64).astype(np.int32)
        o, d = ref.camera_rays(cam, px, py)
        cam_rows.append((ci, px, py, o, d))
    np.savez_compressed(os.path.join(OUT, "camera.npz"),
                        cam=np.array([[c.r, c.theta, c.phi, c.fov, c.width, c.height, c.yaw, c.pitch, c.roll]
                                      for c in cams]),
                        idx=np.concatenate([np.full(64, r[0]) for r in cam_rows]),
                        px=np.concatenate([r[1] for r in cam_rows]), py=np.concatenate([r[2] for r in cam_rows]),
                        origin=np.concatenate([r[3] for r in cam_rows]), dir=np.concatenate([r[4] for r in cam_rows]))

    # 3. Geodesic::integrateStepRK45: one call from camera-initialised states
    rcfg = RefTracerConfig(200.0, 1.05, 20000, 1, 2.3209, 20.0, 1.0, 0, 5e-6, 5e-6, 1e-5, 2.0, 0.1, 0.9, 2.0, 0.1)
    n = 128
    r = rng.uniform(8.0, 60.0, n)
    th = np.arccos(rng.uniform(-0.95, 0.95, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    pos = np.stack([np.zeros(n), r * np.sin(th) * np.cos(ph), r * np.sin(th) * np.sin(ph), r * np.cos(th)], 1)
    vel = rng.normal(size=(n, 4))
    vel[:, 0] = 0.0
    h = rng.uniform(0.01, 1.0, n).astype(np.float32)
    step_in = dict(pos=pos.copy(), vel=vel.copy(), h=h.copy())
    # velocities are normalised to null by the first step's re-normalisation only if drifted; start null:
    from oracle.pyoracle import Oracle
    orc = Oracle()
    met = abi.make_metric(a=0.9)
    for i in range(n):
        g, _ = orc.metric_evaluate(met, pos[i])
        k = vel[i].copy()
        A = g[0, 0, 0]
        B = 2 * g[0, 0, 1:] @ k[1:]
        Cc = k[1:] @ g[0, 1:, 1:] @ k[1:]
        k[0] = (-B - math.sqrt(B * B - 4 * A * Cc)) / (2 * A)
        vel[i] = k
    step_in = dict(pos=pos.copy(), vel=vel.copy(), h=h.copy())
    p2, v2, h2, ok, term = ref.rk45_step(1.0, 0.9, rcfg, pos, vel, h)
    np.savez_compressed(os.path.join(OUT, "rk45_step.npz"), M=1.0, a=0.9,
                        cfg=np.array([5e-6, 5e-6, 1e-5, 2.0, 0.1, 0.9, 2.0, 0.1]), pos_in=step_in["pos"],
                        vel_in=step_in["vel"], h_in=step_in["h"], pos_out=p2, vel_out=v2, h_out=h2, success=ok,
                        terminated=term)

    # 4. GeodesicTracer::trace on small frames (the reference's semantics as written)
    frames = {
        # RenderSession tracer settings (SNRS001A.cpp:103-129), Kerr a = 0.9, r_obs = 100, incl 60 deg
        "kerr_session": dict(M=1.0, a=0.9, r=100.0, th=60.0, fov=30.0, w=24, h=24,
                             cfg=(200.0, 1.05, 20000, 1, 2.3208830, 20.0, 1.0, 0, 5e-6, 5e-6, 1e-5, 2.0, 0.1, 0.9,
                                  2.0, 0.1)),
        # Schwarzschild r_obs = 50, incl 85 deg, RenderSession tolerances
        "schw_session": dict(M=1.0, a=0.0, r=50.0, th=85.0, fov=30.0, w=24, h=24,
                             cfg=(200.0, 1.05, 20000, 1, 6.0, 20.0, 1.0, 0, 5e-6, 5e-6, 1e-5, 2.0, 0.1, 0.9, 2.0,
                                  0.1)),
        # the tight-tolerance configuration (rtol = atol = 1e-10, 10k steps, escape 1000, horizon 1.01)
        "schw_tight": dict(M=1.0, a=0.0, r=50.0, th=85.0, fov=30.0, w=16, h=16,
                           cfg=(1000.0, 1.01, 10000, 1, 6.0, 20.0, 1.0, 0, 1e-10, 1e-10, 1e-9, 2.0, 0.1, 0.9, 2.0,
                                0.1)),
        # the default TracerConfig (GTRC001A.h:162-196)
        "schw_default": dict(M=1.0, a=0.0, r=50.0, th=85.0, fov=30.0, w=12, h=12,
                             cfg=(100.0, 1.05, 5000, 1, 6.0, 20.0, 1.0, 0, 1e-6, 1e-6, 1e-6, 0.1, 0.01, 0.9, 2.0,
                                  0.1)),
        # volumetric gray march on (enable_volumetric)
        "kerr_volumetric": dict(M=1.0, a=0.5, r=40.0, th=75.0, fov=35.0, w=16, h=16,
                                cfg=(200.0, 1.05, 20000, 1, 4.233, 20.0, 1.0, 1, 5e-6, 5e-6, 1e-5, 2.0, 0.1, 0.9, 2.0,
                                     0.1)),
    }
    for name, f in frames.items():
        cam = abi.make_camera(r=f["r"], theta_deg=f["th"], fov=f["fov"], width=f["w"], height=f["h"])
        rc = RefTracerConfig(*f["cfg"])
        rec = ref.trace_frame(f["M"], f["a"], rc, cam, threads=8)
        np.savez_compressed(os.path.join(OUT, f"trace_{name}.npz"), records=rec,
                            camera=np.array([f["r"], math.radians(f["th"]), 0.0, f["fov"], f["w"], f["h"]]),
                            metric=np.array([f["M"], f["a"]]), cfg=np.array(f["cfg"], dtype=np.float64))

    # 5. AccretionDiskD::computeISCO
    spins = np.array([0.0, 0.5, 0.9, 0.998, -0.5, -0.998])
    np.savez_compressed(os.path.join(OUT, "isco.npz"), spin=spins, isco=np.array([ref.isco(s) for s in spins]))
    camera_subpixel(ref)
    print("golden fixtures written to", OUT)


def camera_subpixel(ref):
    """6. PinholeCamera::generateRay(x, y, u, v) at the stratified sub-pixel positions
    RenderSession::shadePixel uses ((s + 0.5) / g for g = 2, 3, 8) and at random (u, v)."""
    from sirius_b200 import abi
    rng = np.random.default_rng(20261204)
    cam = abi.make_camera(r=20.0, theta_deg=30.0, fov=45.0, width=320, height=200, yaw=0.1, pitch=-0.2, roll=0.3)
    px = rng.integers(0, cam.width, 256).astype(np.int32)
    py = rng.integers(0, cam.height, 256).astype(np.int32)
    grid = []
    for g in (2, 3, 8):
        s = np.arange(g, dtype=np.float32)
        grid.append((s + np.float32(0.5)) / np.float32(g))
    pool = np.concatenate(grid)
    u = np.concatenate([rng.choice(pool, 128), rng.uniform(0, 1, 128)]).astype(np.float32)
    v = np.concatenate([rng.choice(pool, 128), rng.uniform(0, 1, 128)]).astype(np.float32)
    o, d = ref.camera_rays_uv(cam, px, py, u, v)
    np.savez_compressed(os.path.join(OUT, "camera_uv.npz"),
                        cam=np.array([cam.r, cam.theta, cam.phi, cam.fov, cam.width, cam.height, cam.yaw, cam.pitch,
                                      cam.roll]), px=px, py=py, u=u, v=v, origin=o, dir=d)


if __name__ == "__main__":
    main()

"""The GPU engine against the reference's own CPU tracer (oracle/_ref, its
GeodesicTracer compiled from its sources), a statistical cross-check that ties
the device to the reference itself and not only to the restatement.

The two follow the same algorithm on rays the reference traces to the end: at
RenderSession's tolerances (5e-6) a ray the reference does not stop on a
rejected step (it reports those as MAX_STEPS, GTRC001A.cpp:272-277) takes the
same Dormand-Prince path up to the reference's float roundings of the
right-hand side and state (PHGD001A.cpp:176,199,549-571) and its null
renormalisation (MTTN001A.cpp:171-237). So on those rays: the same outcome, the
same disk-crossing radius to the reference's crossing interpolation (its
radius is the cylindrical sqrt(x^2 + y^2) = sqrt(r^2 + a^2) of the engine's
Boyer-Lindquist r at the equator, GTRC001A.h:420), and the same escape
direction up to the difference between the reference's final dx/dlambda and
the engine's final covariant momentum at the escape sphere (O(M / r))."""
import os

import numpy as np
import pytest

from oracle import pyoracle
from sirius_b200 import abi

pytestmark = pytest.mark.gpu

FRAMES = [
    ("schwarzschild", 0.0, dict(r=30.0, theta_deg=80.0), 6.0, 20.0),
    ("kerr_0.5", 0.5, dict(r=30.0, theta_deg=75.0), 0.0, 20.0),
    ("kerr_0.9", 0.9, dict(r=50.0, theta_deg=60.0), 0.0, 20.0),
]


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("name,a,cam,d_in,d_out", FRAMES, ids=[f[0] for f in FRAMES])
def test_gpu_engine_against_the_reference_tracer(engine, name, a, cam, d_in, d_out):
    ref = pyoracle.Reference()
    camera = abi.make_camera(width=128, height=128, fov=40.0, **cam)
    frame = abi.make_frame(abi.make_metric(a=a), camera, d_in, d_out)
    cfg = abi.default_config(precision=abi.PRECISION_FP64)  # RenderSession's tracer settings
    engine.configure(cfg)
    res, _, _ = engine.trace_frames([frame])
    rcfg = pyoracle.ref_config_from(cfg, d_in if d_in > 0 else ref.isco(a), d_out)
    rec = ref.trace_frame(1.0, a, rcfg, camera, threads=os.cpu_count() or 1)
    full = rec["outcome"] != abi.MAX_STEPS
    agree = (res["outcome"] == rec["outcome"])[full].mean()
    both = full & (rec["outcome"] == abi.DISK_HIT) & (res["outcome"] == abi.DISK_HIT)
    rho = np.sqrt(res["disk_r"][both, 0].astype(np.float64) ** 2 + a * a)
    dr = np.abs(rho - rec["disk_r"][both, 0]) / rec["disk_r"][both, 0]
    esc = full & (rec["outcome"] == abi.ESCAPED) & (res["outcome"] == abi.ESCAPED)
    v1, v2 = rec["final_direction"][esc, 1:4], res["final_p"][esc, 1:4]
    ang = np.arccos(np.clip(np.sum(v1 * v2, axis=1) / np.linalg.norm(v1, axis=1) / np.linalg.norm(v2, axis=1),
                            -1.0, 1.0))
    print(f"{name}: {full.sum()} rays traced to the end by the reference, outcome agreement {agree:.4f}; "
          f"{both.sum()} disk hits, radius median {np.median(dr):.1e} p99 {np.percentile(dr, 99):.1e}; "
          f"{esc.sum()} escapes, direction median {np.median(ang):.1e} rad")
    assert full.sum() > 2000, full.sum()
    assert agree >= 0.99
    assert both.sum() > 500 and np.median(dr) <= 1e-3 and np.percentile(dr, 99) <= 2e-2
    assert esc.sum() > 200 and np.median(ang) <= 5e-3

"""The symplectic integrator on the device vs the oracle's (the stress
configuration's physics on a small equirectangular crop): Kerr-Newman
a = 0.998, Q = 0.05 from r = 15, Yoshida-4 at d-lambda = 0.01 (shrunk near the
horizon), FP64 re-projection every 8 steps, thin disk + 32-bin volumetric transfer."""
import os

import numpy as np
import pytest

from oracle import compare
from sirius_b200 import abi

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def stress_config(prec, **kw):
    base = dict(integrator=abi.INTEGRATOR_SYMPLECTIC, symplectic_order=4, symplectic_step=0.01,
                projection_period=8, max_steps=50000, escape_radius=60.0, horizon_factor=1.01, min_step=1e-9,
                enable_volumetric=1, n_bins=32, precision=prec)
    base.update(kw)
    return abi.default_config(**base)


def stress_frame(w=32, h=16):
    cam = abi.make_camera(r=15.0, theta_deg=80.0, width=w, height=h, projection=abi.CAMERA_EQUIRECTANGULAR)
    return abi.make_frame(abi.make_metric(a=0.998, Q=0.05), cam, 0.0, 30.0)


def test_equirectangular_camera_rays(engine, oracle):
    """The sky-map camera: device-generated rays equal the oracle's (a ray per pixel over 4 pi)."""
    fr = stress_frame(16, 8)
    engine.configure(abi.default_config(max_steps=1, enable_disk=0))
    res, _, _ = engine.trace_frames([fr])
    ref, _ = oracle.trace_frame(fr, abi.default_config(max_steps=1, enable_disk=0), threads=THREADS)
    np.testing.assert_allclose(res["E0"], ref["E0"], rtol=1e-6)
    np.testing.assert_allclose(res["Lz0"], ref["Lz0"], rtol=1e-5, atol=1e-6)


# (precision, image L-infinity bar over the rays whose histories agree, spectra bar)
@pytest.mark.parametrize("prec,img_max,spec_max", [(abi.PRECISION_FP64, 1e-7, 5e-4),
                                                   (abi.PRECISION_MIXED, 1e-5, 5e-4)])
def test_symplectic_frame_matches_oracle(engine, oracle, prec, img_max, spec_max):
    """A 64 x 32 crop of the sky map: per-output errors against the FP64 oracle
    (the same Yoshida-4 scheme in FP64), maxima over the rays whose histories
    agree. The spectra accumulate in FP32 on the device in both precision modes.
    The null constraint and L_z drift are the scheme's own (the reference's
    leapfrog drifts with dH/dp at the old position, PHSI001A.h:430-455, and the
    re-projection runs every 8 steps): the device's returned states carry the
    oracle's values of both."""
    fr = stress_frame(64, 32)
    engine.configure(stress_config(prec))
    res, img, spc = engine.trace_frames([fr], spectra=True)
    ref, bins = oracle.trace_frame(fr, stress_config(abi.PRECISION_FP64), threads=THREADS)
    rep = compare.report(res, img, ref, spc, bins, escape_radius=60.0)
    print("symplectic", prec)
    print(compare.summary(rep))
    assert rep["outcome_agreement"] >= 0.98
    assert rep["image"]["max"] <= img_max, rep["image"]
    assert rep["spectra"]["max"] <= spec_max, rep["spectra"]
    assert rep["E"]["drift"]["max"] <= 1e-12
    assert rep["Lz"]["vs_oracle"]["max"] <= 1e-5 and rep["Carter"]["vs_oracle"]["max"] <= 1e-5
    # re-projection every 8 steps: the returned state is at most 7 steps past one,
    # and its null value is the oracle's
    oracle_null = float(np.abs(ref["null_final"]).max())
    assert rep["null_final"]["max"] <= 1.01 * oracle_null + 1e-12, (rep["null_final"], oracle_null)


def test_symplectic_rejects_bad_order(engine):
    with pytest.raises(Exception):
        engine.configure(stress_config(abi.PRECISION_MIXED, symplectic_order=5))
    engine.configure(stress_config(abi.PRECISION_MIXED))

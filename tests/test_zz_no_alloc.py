"""The allocation-free device entry point, sirius_cuda_trace_frames_static,
against sirius_cuda_trace_frames_device on the same frames: two calls in a row
give the same image, spectra and per-ray records, bit for bit, and a call with
more frames than the static scratch holds is rejected before any launch.

The file sorts last so that the check also runs after every other GPU test
has used the device (and the library's own allocations) in this process."""
import ctypes as C

import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def batch():
    """A Kerr frame (thin disk + 16-bin volumetric) and a Schwarzschild frame."""
    f0 = abi.make_frame(abi.make_metric(a=0.9), abi.make_camera(r=100.0, theta_deg=60.0, width=40, height=32,
                                                                fov=30.0), 0.0, 30.0)
    f1 = abi.make_frame(abi.make_metric(a=0.0), abi.make_camera(r=50.0, theta_deg=85.0, width=24, height=24,
                                                                fov=30.0), 0.0, 20.0)
    f1.ray_offset = 40 * 32
    return [f0, f1]


def config():
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                              precision=abi.PRECISION_MIXED, enable_volumetric=1, n_bins=16)


def run(engine, entry, frames):
    import torch
    dev = torch.device("cuda", 0)
    arr = (abi.Frame * len(frames))(*frames)
    d_frames = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
    total = sum(f.camera.width * f.camera.height for f in frames)
    rsize = abi.result_dtype().itemsize
    d_res = torch.zeros(total * rsize, dtype=torch.uint8, device=dev)
    d_img = torch.zeros(total, dtype=torch.float32, device=dev)
    d_spc = torch.zeros(total * 16, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    entry(d_frames.data_ptr(), len(frames), total, d_res.data_ptr(), d_img.data_ptr(), d_spc.data_ptr(),
          stream.cuda_stream)
    torch.cuda.synchronize()
    return d_res.cpu().numpy().tobytes(), d_img.cpu().numpy(), d_spc.cpu().numpy()


def test_static_entry_matches_device_entry_twice(engine):
    engine.configure(config())
    frames = batch()
    ref = run(engine, engine.trace_frames_device, frames)
    assert np.all(np.isfinite(ref[1])) and ref[1].max() > 0
    for _ in range(2):
        got = run(engine, engine.trace_frames_static, frames)
        assert got[0] == ref[0]
        np.testing.assert_array_equal(got[1], ref[1])
        np.testing.assert_array_equal(got[2], ref[2])


def test_static_entry_rejects_too_many_frames(engine):
    import torch
    from sirius_b200.engine import SiriusError
    engine.configure(config())
    n = abi.STATIC_MAX_FRAMES + 1
    frames = []
    for i in range(n):
        f = abi.make_frame(abi.make_metric(a=0.5), abi.make_camera(r=50.0, theta_deg=80.0, width=1, height=1,
                                                                   fov=30.0), 0.0, 20.0)
        f.ray_offset = i
        frames.append(f)
    arr = (abi.Frame * n)(*frames)
    dev = torch.device("cuda", 0)
    d_frames = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
    d_img = torch.zeros(n, dtype=torch.float32, device=dev)
    with pytest.raises(SiriusError) as e:
        engine.trace_frames_static(d_frames.data_ptr(), n, n, None, d_img.data_ptr(), None,
                                   torch.cuda.current_stream(dev).cuda_stream)
    assert e.value.code == abi.ERR_INVALID_ARGUMENT
    # the handle stays usable
    got = run(engine, engine.trace_frames_static, batch())
    assert np.all(np.isfinite(got[1]))

"""The allocation-free device entry point, sirius_cuda_trace_frames_static.

Some hosts cannot let a plugin allocate device memory: their own allocator
already holds the memory they hand out, or their frame loop cannot take the
device-wide synchronisation of cudaMalloc/cudaFree. This entry point serves
them by keeping its launch scratch in a static device array of the library.
The tests check that it allocates nothing (device free memory is unchanged
across calls on a freshly created handle, whose own scratch buffers were never
allocated), that it gives what sirius_cuda_trace_frames_device gives on the same
frames, bit for bit, on two calls in a row, and that a call with more frames
than the static scratch holds is rejected before any launch.

The file sorts last so that the check also runs after every other GPU test
has used the device (and the library's own allocations) in this process."""
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


class Buffers:
    """Device copies of the frames and output buffers, allocated once by torch."""

    def __init__(self, frames):
        import torch
        dev = torch.device("cuda", 0)
        arr = (abi.Frame * len(frames))(*frames)
        self.n = len(frames)
        self.frames = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
        self.total = sum(abi.frame_rays(f) for f in frames)
        self.res = torch.zeros(self.total * abi.result_dtype().itemsize, dtype=torch.uint8, device=dev)
        self.img = torch.zeros(self.total, dtype=torch.float32, device=dev)
        self.spc = torch.zeros(self.total * 16, dtype=torch.float32, device=dev)
        self.stream = torch.cuda.current_stream(dev).cuda_stream
        torch.cuda.synchronize()

    def call(self, entry):
        entry(self.frames.data_ptr(), self.n, self.total, self.res.data_ptr(), self.img.data_ptr(),
              self.spc.data_ptr(), self.stream)

    def read(self):
        import torch
        torch.cuda.synchronize()
        return self.res.cpu().numpy().tobytes(), self.img.cpu().numpy(), self.spc.cpu().numpy()


def test_static_entry_allocates_nothing_and_matches_device_entry(engine):
    import torch

    from sirius_b200.engine import Engine
    frames = batch()
    # one static call on the shared handle first: the CUDA modules of the library
    # load (lazily, on first use), and the static scratch address is resolved
    engine.configure(config())
    warm = Buffers(frames)
    warm.call(engine.trace_frames_static)
    warm.read()
    fresh = Engine(0)
    try:
        fresh.configure(config())
        buf = Buffers(frames)
        free0 = torch.cuda.mem_get_info(0)[0]
        got = []
        for _ in range(2):
            buf.call(fresh.trace_frames_static)
            got.append(buf.read())
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
        # the same frames through the device entry point, which allocates its own scratch
        ref = Buffers(frames)
        ref.call(fresh.trace_frames_device)
        want = ref.read()
    finally:
        fresh.close()
    assert np.all(np.isfinite(want[1])) and want[1].max() > 0
    for g in got:
        assert g[0] == want[0]
        np.testing.assert_array_equal(g[1], want[1])
        np.testing.assert_array_equal(g[2], want[2])


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
    buf = Buffers(batch())
    buf.call(engine.trace_frames_static)
    assert np.all(np.isfinite(buf.read()[1]))

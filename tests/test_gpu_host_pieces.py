"""The host entry point into page-locked buffers traces a large one-frame launch
in pieces of tile rows on two streams and copies each piece to the host while
the next ones trace. Per-ray results, image and spectra are bit for bit those of
the single launch (pageable buffers) and of the device entry point, on a frame
whose width and height are multiples of the 16 x 8 tile and on a ragged one."""
import ctypes as C

import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def kerr_frame(width, height):
    cam = abi.make_camera(r=100.0, theta_deg=60.0, width=width, height=height, fov=30.0)
    return abi.make_frame(abi.make_metric(a=0.9), cam, 0.0, 30.0)


@pytest.mark.parametrize("width,height", [(512, 512), (520, 500)])
def test_pieces_equal_the_single_launch(engine, width, height):
    import torch
    engine.configure(abi.default_config(precision=abi.PRECISION_MIXED, enable_disk=1, enable_volumetric=1,
                                        n_bins=16, abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9,
                                        horizon_factor=1.01, max_steps=10000))
    fr = kerr_frame(width, height)
    total = width * height
    # pageable numpy buffers: one launch, then the copies
    res, img, spc = engine.trace_frames([fr], results=True, image=True, spectra=True)
    single = engine.stats()
    # page-locked buffers: the piecewise launch
    h_res = torch.zeros(total * abi.result_dtype().itemsize, dtype=torch.uint8, pin_memory=True)
    h_img = torch.full((total,), float("nan"), dtype=torch.float32, pin_memory=True)
    h_spc = torch.full((total * 16,), float("nan"), dtype=torch.float32, pin_memory=True)
    arr = (abi.Frame * 1)(fr)
    engine.trace_frames_into(C.addressof(arr), 1, h_res.data_ptr(), h_img.data_ptr(), h_spc.data_ptr())
    pieces = engine.stats()
    assert single.kernel_launches <= 2 < pieces.kernel_launches  # the trace (+ the flux table) vs the pieces
    np.testing.assert_array_equal(h_img.numpy(), img)
    np.testing.assert_array_equal(h_spc.numpy().reshape(total, 16), spc)
    assert h_res.numpy().tobytes() == res.tobytes()
    assert pieces.accepted_steps == single.accepted_steps and pieces.rejected_steps == single.rejected_steps
    # the device entry point
    dev = torch.device("cuda", 0)
    d_fr = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(dev)
    d_img = torch.empty(total, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    engine.trace_frames_device(d_fr.data_ptr(), 1, total, None, d_img.data_ptr(), None, stream.cuda_stream)
    stream.synchronize()
    np.testing.assert_array_equal(d_img.cpu().numpy(), img)

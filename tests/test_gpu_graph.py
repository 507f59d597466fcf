"""Prepared frames (sirius_cuda_prepare_frames / _launch_prepared): the launch
is device work only, so it can be captured in a CUDA graph; replays of the
graph give the same image, bit for bit, as the ordinary entry point, also
after other calls on the handle have uploaded other frames."""
import numpy as np
import pytest

from sirius_b200 import abi

pytestmark = pytest.mark.gpu


def frames():
    f0 = abi.make_frame(abi.make_metric(a=0.9), abi.make_camera(r=60.0, theta_deg=70.0, width=40, height=32,
                                                                fov=30.0), 0.0, 25.0)
    f1 = abi.make_frame(abi.make_metric(a=0.0), abi.make_camera(r=40.0, theta_deg=85.0, width=24, height=24,
                                                                fov=35.0), 0.0, 20.0)
    return [f0, f1]


@pytest.mark.parametrize("prec", [abi.PRECISION_MIXED, abi.PRECISION_FP64])
def test_graph_replays_match_the_direct_trace(engine, prec):
    import torch
    cfg = abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                             escape_radius=500.0, horizon_factor=1.01, max_steps=20000, precision=prec,
                             enable_volumetric=1, n_bins=8)
    engine.configure(cfg)
    fr = frames()
    _, ref, ref_spc = engine.trace_frames(fr, results=False, image=True, spectra=True)
    total = engine.prepare_frames(fr)
    assert total == ref.size
    dev = torch.device("cuda", 0)
    d_img = torch.zeros(total, dtype=torch.float32, device=dev)
    d_spc = torch.zeros(total * 8, dtype=torch.float32, device=dev)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # an ordinary (uncaptured) launch first
        engine.launch_prepared(None, d_img.data_ptr(), d_spc.data_ptr(), side.cuda_stream)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_img.cpu().numpy(), ref)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        engine.launch_prepared(None, d_img.data_ptr(), d_spc.data_ptr(), torch.cuda.current_stream().cuda_stream)
    # other work on the handle in between, with other frames
    other = abi.make_frame(abi.make_metric(a=0.5), abi.make_camera(r=30.0, width=64, height=64), 0.0, 20.0)
    engine.trace_frames([other], results=False)
    for _ in range(3):
        d_img.zero_()
        d_spc.zero_()
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d_img.cpu().numpy(), ref)
        np.testing.assert_array_equal(d_spc.cpu().numpy(), ref_spc.ravel())
    del g


def test_prepared_frames_refuse_multisample(engine):
    from sirius_b200.engine import SiriusError
    engine.configure(abi.default_config(samples_per_pixel=4))
    with pytest.raises(SiriusError) as e:
        engine.prepare_frames(frames())
    assert e.value.code == abi.ERR_UNSUPPORTED

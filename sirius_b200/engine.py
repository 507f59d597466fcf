"""Python binding of the C ABI (include/sirius_cuda.h) via ctypes.

This is a thin host-side mirror for scripts and tests; the product boundary is
the C ABI itself. The library must have been built (sirius_b200.build.build());
there is no fallback of any kind when it is missing or no CUDA device exists.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsirius_b200.so")

_P = C.POINTER

# Every symbol include/sirius_cuda.h declares (checked by tests/test_abi.py).
EXPORTS = [
    "sirius_cuda_abi_version", "sirius_cuda_default_config", "sirius_cuda_create", "sirius_cuda_destroy",
    "sirius_cuda_get_last_error", "sirius_cuda_configure", "sirius_cuda_trace_frames",
    "sirius_cuda_trace_frames_device", "sirius_cuda_trace_rays", "sirius_cuda_metric_evaluate",
    "sirius_cuda_dp45_step", "sirius_cuda_last_stats", "sirius_cuda_autotune", "sirius_cuda_measure_fma_peak",
    "sirius_cuda_flop_count", "sirius_cuda_trace_frames_static", "sirius_cuda_surrogate_load",
    "sirius_cuda_surrogate_infer", "sirius_cuda_surrogate_features", "sirius_cuda_render_surrogate",
    "sirius_cuda_render_surrogate_device", "sirius_cuda_default_train_config", "sirius_cuda_train_init",
    "sirius_cuda_train_steps", "sirius_cuda_train_evaluate", "sirius_cuda_train_gradient", "sirius_cuda_train_params",
    "sirius_cuda_write_png", "sirius_cuda_write_exr", "sirius_cuda_write_pfm", "sirius_cuda_write_ppm",
    "sirius_cuda_trace_beams", "sirius_cuda_prepare_frames", "sirius_cuda_launch_prepared",
]


class SiriusError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"sirius_cuda error {code}: {msg}")
        self.code = code


def load_library(path=LIB_PATH):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = C.CDLL(path)
    L.sirius_cuda_abi_version.restype = C.c_int
    L.sirius_cuda_default_config.argtypes = [_P(abi.TraceConfig)]
    L.sirius_cuda_create.argtypes = [C.c_int, _P(C.c_void_p)]
    L.sirius_cuda_destroy.argtypes = [C.c_void_p]
    L.sirius_cuda_get_last_error.argtypes = [C.c_void_p]
    L.sirius_cuda_get_last_error.restype = C.c_char_p
    L.sirius_cuda_configure.argtypes = [C.c_void_p, _P(abi.TraceConfig)]
    L.sirius_cuda_trace_frames.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.sirius_cuda_trace_frames_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_void_p]
    L.sirius_cuda_trace_frames_static.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_void_p]
    L.sirius_cuda_surrogate_load.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.sirius_cuda_surrogate_infer.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.sirius_cuda_surrogate_features.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _P(abi.SurrogateConfig),
                                                 C.c_void_p, C.c_void_p, C.c_void_p]
    L.sirius_cuda_render_surrogate.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _P(abi.SurrogateConfig),
                                               C.c_void_p, C.c_void_p, C.c_void_p, _P(abi.SurrogateStats)]
    L.sirius_cuda_render_surrogate_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _P(abi.SurrogateConfig),
                                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                      _P(abi.SurrogateStats)]
    L.sirius_cuda_trace_rays.argtypes = [C.c_void_p, _P(abi.Metric), C.c_double, C.c_double, C.c_void_p,
                                         C.c_int64, C.c_void_p]
    L.sirius_cuda_metric_evaluate.argtypes = [C.c_void_p, _P(abi.Metric), C.c_void_p, C.c_int64, C.c_int32,
                                              C.c_void_p, C.c_void_p]
    L.sirius_cuda_dp45_step.argtypes = [C.c_void_p, _P(abi.Metric), C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int64]
    L.sirius_cuda_last_stats.argtypes = [C.c_void_p, _P(abi.LaunchStats)]
    L.sirius_cuda_autotune.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _P(abi.TraceConfig)]
    L.sirius_cuda_measure_fma_peak.argtypes = [C.c_void_p, C.c_int32, _P(C.c_double)]
    L.sirius_cuda_flop_count.argtypes = [_P(abi.Metric), _P(C.c_double), _P(C.c_double), _P(C.c_double)]
    L.sirius_cuda_default_train_config.argtypes = [_P(abi.TrainConfig)]
    L.sirius_cuda_default_train_config.restype = None
    L.sirius_cuda_train_init.argtypes = [C.c_void_p, C.c_void_p, _P(abi.TrainConfig)]
    L.sirius_cuda_train_steps.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                          _P(C.c_float)]
    L.sirius_cuda_train_evaluate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.sirius_cuda_train_gradient.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p]
    L.sirius_cuda_train_params.argtypes = [C.c_void_p, C.c_void_p, _P(C.c_int64)]
    L.sirius_cuda_trace_beams.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    L.sirius_cuda_prepare_frames.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, _P(C.c_int64)]
    L.sirius_cuda_launch_prepared.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    for name in ("sirius_cuda_write_png", "sirius_cuda_write_exr"):
        getattr(L, name).argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    for name in ("sirius_cuda_write_pfm", "sirius_cuda_write_ppm"):
        getattr(L, name).argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_void_p]
    return L


def flop_count(metric, lib=None):
    """(rhs, attempt, accepted step) algorithmic operation counts of the kernels' formulation."""
    lib = lib or load_library()
    a, b, c = C.c_double(), C.c_double(), C.c_double()
    rc = lib.sirius_cuda_flop_count(C.byref(metric), C.byref(a), C.byref(b), C.byref(c))
    if rc != abi.OK:
        raise SiriusError(rc, "sirius_cuda_flop_count failed")
    return a.value, b.value, c.value


def write_image(path, pixels, fmt=None, lib=None):
    """Write an (height, width, 3 or 4) float image (top row first) as PNG, EXR,
    PFM or PPM (by `fmt` or the file extension) with the library's writers."""
    lib = lib or load_library()
    px = np.ascontiguousarray(pixels, dtype=np.float32)
    if px.ndim != 3 or px.shape[2] not in (3, 4):
        raise ValueError("pixels must be (height, width, 3) or (height, width, 4)")
    h, w, c = px.shape
    fmt = (fmt or os.path.splitext(path)[1].lstrip(".")).lower()
    p = os.fsencode(path)
    if fmt in ("png", "exr"):
        rc = getattr(lib, f"sirius_cuda_write_{fmt}")(p, w, h, c, px.ctypes.data)
    elif fmt in ("pfm", "ppm"):
        if c != 3:
            raise ValueError(f"{fmt} takes RGB pixels")
        rc = getattr(lib, f"sirius_cuda_write_{fmt}")(p, w, h, px.ctypes.data)
    else:
        raise ValueError(f"unknown image format {fmt!r}")
    if rc != abi.OK:
        raise SiriusError(rc, f"writing {path}")


def frames_array(frames):
    """Pack frames into a ctypes array, assigning contiguous ray offsets."""
    arr = (abi.Frame * len(frames))(*frames)
    off = 0
    for f in arr:
        f.ray_offset = off
        off += abi.frame_rays(f)
    return arr, off


class Engine:
    """One handle on one CUDA device (mirrors the lifecycle of sirius_optix_*)."""

    def __init__(self, device=0, config=None, lib=None):
        self.lib = lib or load_library()
        h = C.c_void_p()
        rc = self.lib.sirius_cuda_create(device, C.byref(h))
        if rc != abi.OK:
            raise SiriusError(rc, "sirius_cuda_create failed (no sm_100 device or CUDA error)")
        self.h = h
        self.config = config or abi.default_config()
        self.configure(self.config)

    def close(self):
        if self.h:
            self.lib.sirius_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != abi.OK:
            raise SiriusError(rc, self.lib.sirius_cuda_get_last_error(self.h).decode())

    def configure(self, cfg):
        self._check(self.lib.sirius_cuda_configure(self.h, C.byref(cfg)))
        self.config = cfg

    def trace_frames(self, frames, results=True, image=True, spectra=False):
        arr, total = frames_array(frames)
        nb = self.config.n_bins if self.config.enable_volumetric else 0
        res = np.zeros(total, dtype=abi.result_dtype()) if results else None
        img = np.zeros(total, dtype=np.float32) if image else None
        spc = np.zeros((total, max(nb, 1)), dtype=np.float32) if (spectra and nb) else None
        self._check(self.lib.sirius_cuda_trace_frames(
            self.h, C.addressof(arr), len(frames), res.ctypes.data if res is not None else None,
            img.ctypes.data if img is not None else None, spc.ctypes.data if spc is not None else None))
        return res, img, (spc[:, :nb] if spc is not None else None)

    def trace_frames_into(self, frames_arr, n_frames, results_ptr, image_ptr, spectra_ptr):
        """Host entry point with caller-owned host buffers (raw addresses, e.g. pinned memory)."""
        self._check(self.lib.sirius_cuda_trace_frames(self.h, frames_arr, n_frames, results_ptr, image_ptr,
                                                      spectra_ptr))

    def trace_frames_device(self, d_frames, n_frames, total, d_results, d_image, d_spectra, stream):
        """Device entry point: all pointers are device addresses; stream is a cudaStream_t address."""
        self._check(self.lib.sirius_cuda_trace_frames_device(self.h, d_frames, n_frames, total, d_results, d_image,
                                                             d_spectra, stream))

    def trace_frames_static(self, d_frames, n_frames, total, d_results, d_image, d_spectra, stream):
        """As trace_frames_device, with the launch scratch in the library's static
        device array: no device allocation (at most SIRIUS_STATIC_MAX_FRAMES frames)."""
        self._check(self.lib.sirius_cuda_trace_frames_static(self.h, d_frames, n_frames, total, d_results, d_image,
                                                             d_spectra, stream))

    def surrogate_load(self, params):
        """Surrogate MLP weights: SURROGATE_PARAMS floats, nn.Linear order (W1 b1 ... W5 b5)."""
        p = np.ascontiguousarray(params, dtype=np.float32).ravel()
        self._check(self.lib.sirius_cuda_surrogate_load(self.h, p.ctypes.data, p.size))

    def surrogate_infer(self, d_features, n, d_out, stream=None):
        """MLP on n x 5 device features into n x 4 device outputs."""
        self._check(self.lib.sirius_cuda_surrogate_infer(self.h, d_features, n, d_out, stream))

    def prepare_frames(self, frames):
        """Upload the frames for launch_prepared; returns the number of rays (pixels)."""
        arr, _ = frames_array(frames)
        total = C.c_int64()
        self._check(self.lib.sirius_cuda_prepare_frames(self.h, C.addressof(arr), len(frames), C.byref(total)))
        return total.value

    def launch_prepared(self, d_results, d_image, d_spectra, stream):
        """The trace of the prepared frames as stream work only (capturable in a CUDA graph)."""
        self._check(self.lib.sirius_cuda_launch_prepared(self.h, d_results, d_image, d_spectra, stream))

    def trace_beams(self, frames):
        """Beams around every pixel ray of the frames: a structured array of BeamResult
        (outcome, steps, magnification, parity, final_dir)."""
        arr, total = frames_array(frames)
        out = (abi.BeamResult * total)()
        self._check(self.lib.sirius_cuda_trace_beams(self.h, C.addressof(arr), len(frames), C.addressof(out)))
        dt = np.dtype([("outcome", "<i4"), ("steps", "<i4"), ("magnification", "<f4"), ("parity", "<f4"),
                       ("final_dir", "<f4", (3,)), ("reserved", "<i4")])
        return np.frombuffer(bytes(out), dtype=dt).copy()

    def train_init(self, params, config):
        """Start training from params (SURROGATE_PARAMS floats): FP32 master weights, zero Adam moments."""
        p = np.ascontiguousarray(params, dtype=np.float32).ravel()
        if p.size != abi.SURROGATE_PARAMS:
            raise ValueError(f"expected {abi.SURROGATE_PARAMS} parameters, got {p.size}")
        self._check(self.lib.sirius_cuda_train_init(self.h, p.ctypes.data, C.byref(config)))

    def train_steps(self, d_features, d_targets, d_weights, n_rows, n_steps):
        """n_steps optimiser steps over the device-resident rows [0, n_rows); returns their device time (ms)."""
        ms = C.c_float()
        self._check(self.lib.sirius_cuda_train_steps(self.h, d_features, d_targets, d_weights, n_rows, n_steps,
                                                     C.byref(ms)))
        return ms.value

    def train_evaluate(self, d_features, d_targets, d_weights, n_rows):
        """Loss parts (BCE, l_r, l_g, l_h) of the current weights over rows [0, n_rows)."""
        out = np.zeros(4, dtype=np.float32)
        self._check(self.lib.sirius_cuda_train_evaluate(self.h, d_features, d_targets, d_weights, n_rows,
                                                        out.ctypes.data))
        return out

    def train_gradient(self, d_features, d_targets, d_weights, n_rows):
        """(loss parts, gradient) of one batch of rows [0, n_rows); no update."""
        parts = np.zeros(4, dtype=np.float32)
        grad = np.zeros(abi.SURROGATE_PARAMS, dtype=np.float32)
        self._check(self.lib.sirius_cuda_train_gradient(self.h, d_features, d_targets, d_weights, n_rows,
                                                        parts.ctypes.data, grad.ctypes.data))
        return parts, grad

    def train_params(self):
        """(FP32 master weights, optimiser steps taken)."""
        p = np.zeros(abi.SURROGATE_PARAMS, dtype=np.float32)
        steps = C.c_int64()
        self._check(self.lib.sirius_cuda_train_params(self.h, p.ctypes.data, C.byref(steps)))
        return p, steps.value

    def surrogate_features(self, frames, d_features, d_gate=None, config=None, stream=None):
        """Features (n x 5) and gate (n bytes) of every pixel of the frames, into device buffers."""
        arr, _ = frames_array(frames)
        cfg = config or abi.surrogate_config()
        self._check(self.lib.sirius_cuda_surrogate_features(self.h, C.addressof(arr), len(frames), C.byref(cfg),
                                                            d_features, d_gate, stream))

    def render_surrogate(self, frames, config=None, mlp_image=False):
        """Surrogate-gated image (host): returns (image, mlp_image or None, gate, stats)."""
        arr, total = frames_array(frames)
        cfg = config or abi.surrogate_config()
        img = np.zeros(total, dtype=np.float32)
        mimg = np.zeros(total, dtype=np.float32) if mlp_image else None
        gate = np.zeros(total, dtype=np.uint8)
        st = abi.SurrogateStats()
        self._check(self.lib.sirius_cuda_render_surrogate(
            self.h, C.addressof(arr), len(frames), C.byref(cfg), img.ctypes.data,
            mimg.ctypes.data if mimg is not None else None, gate.ctypes.data, C.byref(st)))
        return img, mimg, gate, st

    def render_surrogate_device(self, frames, d_image, d_image_mlp=None, d_gate=None, config=None, stream=None):
        """Surrogate-gated image into device buffers; returns the stage statistics."""
        arr, _ = frames_array(frames)
        cfg = config or abi.surrogate_config()
        st = abi.SurrogateStats()
        self._check(self.lib.sirius_cuda_render_surrogate_device(self.h, C.addressof(arr), len(frames), C.byref(cfg),
                                                                 d_image, d_image_mlp, d_gate, stream, C.byref(st)))
        return st

    def trace_rays(self, metric, rays, disk_inner=0.0, disk_outer=20.0):
        n = len(rays)
        arr = (abi.CameraRay * n)(*rays)
        out = np.zeros(n, dtype=abi.result_dtype())
        self._check(self.lib.sirius_cuda_trace_rays(self.h, C.byref(metric), disk_inner, disk_outer,
                                                    C.addressof(arr), n, out.ctypes.data))
        return out

    def metric_evaluate(self, metric, pos, precision=abi.PRECISION_FP64):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 4)
        n = len(pos)
        g = np.zeros((n, 4, 4))
        dg = np.zeros((n, 4, 4, 4))
        self._check(self.lib.sirius_cuda_metric_evaluate(self.h, C.byref(metric), pos.ctypes.data, n, precision,
                                                         g.ctypes.data, dg.ctypes.data))
        return g, dg

    def dp45_step(self, metric, state, h):
        s = np.array(state, dtype=np.float64).reshape(-1, 8).copy()
        hh = np.array(h, dtype=np.float64).reshape(-1).copy()
        acc = np.zeros(len(s), dtype=np.int32)
        err = np.zeros(len(s))
        self._check(self.lib.sirius_cuda_dp45_step(self.h, C.byref(metric), s.ctypes.data, hh.ctypes.data,
                                                   acc.ctypes.data, err.ctypes.data, len(s)))
        return s, hh, acc, err

    def stats(self):
        st = abi.LaunchStats()
        self._check(self.lib.sirius_cuda_last_stats(self.h, C.byref(st)))
        return st

    def autotune(self, frames):
        arr, _ = frames_array(frames)
        out = abi.TraceConfig()
        self._check(self.lib.sirius_cuda_autotune(self.h, C.addressof(arr), len(frames), C.byref(out)))
        self.config = out
        return out

    def fma_peak(self, precision):
        v = C.c_double()
        self._check(self.lib.sirius_cuda_measure_fma_peak(self.h, precision, C.byref(v)))
        return v.value

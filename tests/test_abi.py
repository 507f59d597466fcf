"""The C ABI library loads without a GPU and exports every entry point the
header declares; the Python mirror of the structs matches the C layout."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from sirius_b200 import abi
from sirius_b200.engine import EXPORTS, LIB_PATH, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sirius_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sirius_cuda_\w+)\s*\(", text)))


def test_header_declarations_match_binding_list():
    assert declared_functions() == sorted(EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = load_library()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} not exported by {LIB_PATH}"


def test_abi_version():
    lib = load_library()
    assert lib.sirius_cuda_abi_version() == abi.ABI_VERSION


def test_struct_layouts_match_c(oracle):
    # the oracle is compiled against the same header
    assert C.sizeof(abi.RayResult) == oracle.lib.oracle_sizeof_result()
    assert C.sizeof(abi.TraceConfig) == oracle.lib.oracle_sizeof_config()
    assert C.sizeof(abi.Frame) == oracle.lib.oracle_sizeof_frame()
    # static_asserts in engine.cu
    assert C.sizeof(abi.Metric) == 80
    assert C.sizeof(abi.Camera) == 64
    assert C.sizeof(abi.Frame) == 176
    assert C.sizeof(abi.RayResult) == 256
    assert C.sizeof(abi.CameraRay) == 64
    assert C.sizeof(abi.SurrogateConfig) == 40
    assert C.sizeof(abi.SurrogateStats) == 56
    assert C.sizeof(abi.TrainConfig) == 64
    dt = abi.result_dtype()
    for name, _ in abi.RayResult._fields_:
        assert dt.fields[name][1] == getattr(abi.RayResult, name).offset, name


def test_default_config_matches_render_session():
    """sirius_cuda_default_config == the tracer settings RenderSession applies (SNRS001A.cpp:103-129)."""
    lib = load_library()
    c = abi.TraceConfig()
    assert lib.sirius_cuda_default_config(C.byref(c)) == abi.OK
    py = abi.default_config()
    for name, _ in abi.TraceConfig._fields_:
        a, b = getattr(c, name), getattr(py, name)
        if name == "reserved":
            assert list(a) == list(b)
        else:
            assert a == b, name
    assert (c.escape_radius, c.horizon_factor, c.max_steps) == (200.0, 1.05, 20000)
    assert (c.initial_step, c.max_step, c.min_step, c.abs_tolerance) == (0.1, 2.0, 1e-5, 5e-6)


def test_default_train_config_matches_python_mirror():
    lib = load_library()
    c = abi.TrainConfig()
    lib.sirius_cuda_default_train_config(C.byref(c))
    py = abi.train_config()
    for name, _ in abi.TrainConfig._fields_:
        a, b = getattr(c, name), getattr(py, name)
        assert (list(a) == list(b)) if name == "reserved" else (a == b), name


def test_null_handle_and_bad_arguments_are_errors_not_crashes():
    lib = load_library()
    assert lib.sirius_cuda_get_last_error(None) == b"invalid handle"
    assert lib.sirius_cuda_destroy(None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_configure(None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_trace_frames(None, None, 0, None, None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_default_config(None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_train_init(None, None, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_train_steps(None, None, None, None, 0, 0, None) == abi.ERR_INVALID_ARGUMENT
    assert lib.sirius_cuda_train_gradient(None, None, None, None, 128, None, None) == abi.ERR_INVALID_ARGUMENT
    h = C.c_void_p()
    rc = lib.sirius_cuda_create(999, C.byref(h))
    assert rc in (abi.ERR_NO_DEVICE, abi.ERR_INVALID_ARGUMENT)
    assert h.value is None


def test_frames_array_assigns_contiguous_offsets():
    from sirius_b200.engine import frames_array
    fr = [abi.make_frame(abi.make_metric(), abi.make_camera(width=w, height=h)) for w, h in ((4, 3), (5, 5), (2, 7))]
    arr, total = frames_array(fr)
    assert [f.ray_offset for f in arr] == [0, 12, 37]
    assert total == 51


def test_engine_fails_loudly_without_library(tmp_path):
    with pytest.raises(FileNotFoundError):
        load_library(str(tmp_path / "missing.so"))


def test_result_dtype_roundtrip():
    r = abi.RayResult()
    r.outcome = abi.DISK_HIT
    r.final_x[2] = 3.5
    r.disk_g[1] = 0.25
    r.flags = 3
    arr = np.frombuffer(bytes(r), dtype=abi.result_dtype())
    assert arr["outcome"][0] == abi.DISK_HIT and arr["final_x"][0, 2] == 3.5
    assert arr["disk_g"][0, 1] == np.float32(0.25) and arr["flags"][0] == 3

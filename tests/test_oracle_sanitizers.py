"""The oracle and its C ABI under AddressSanitizer and UndefinedBehaviorSanitizer.

A small driver is compiled together with oracle/oracle_capi.cpp with
-fsanitize=address,undefined (any UB report aborts) and traces a set of frames
and configurations written by the test: DP45 in engine and compat semantics with
the thin disk and volumetric bins, long double precision, the symplectic
integrator on an equirectangular crop, Morris-Thorne and Alcubierre frames, a row
window, and several host threads. The frames' outputs must also be finite."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from sirius_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r'''
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include "sirius_cuda.h"
extern "C" int oracle_trace_frame(const sirius_frame*, const sirius_trace_config*, int64_t, int64_t,
                                  sirius_ray_result*, double*, int, int);
int main(int argc, char** argv) {
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) return 2;
    int32_t n = 0;
    if (std::fread(&n, 4, 1, fp) != 1) return 3;
    long long total_steps = 0;
    for (int i = 0; i < n; ++i) {
        sirius_frame f;
        sirius_trace_config c;
        int32_t threads = 1, precision = 0;
        if (std::fread(&f, sizeof f, 1, fp) != 1 || std::fread(&c, sizeof c, 1, fp) != 1 ||
            std::fread(&threads, 4, 1, fp) != 1 || std::fread(&precision, 4, 1, fp) != 1) return 4;
        const int64_t rows = f.row_count > 0 ? f.row_count : f.camera.height;
        const int64_t count = rows * int64_t(f.camera.width);
        std::vector<sirius_ray_result> out(count);
        std::vector<double> bins(count * (c.enable_volumetric ? (c.n_bins > 0 ? c.n_bins : 1) : 1), 0.0);
        if (oracle_trace_frame(&f, &c, 0, count, out.data(), bins.data(), threads, precision) != 0) return 5;
        for (const auto& r : out) {
            total_steps += r.steps;
            if (!std::isfinite(r.intensity) || !std::isfinite(r.final_x[1])) { std::printf("non-finite\n"); return 6; }
        }
        for (double b : bins) if (!std::isfinite(b)) { std::printf("non-finite bin\n"); return 7; }
        std::printf("case %d: %lld rays\n", i, (long long)count);
    }
    std::printf("steps %lld\n", total_steps);
    return 0;
}
'''


def cases():
    kerr = abi.make_frame(abi.make_metric(a=0.9), abi.make_camera(r=60.0, theta_deg=70.0, width=12, height=10,
                                                                  fov=30.0), 0.0, 20.0)
    base = dict(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0, escape_radius=100.0,
                horizon_factor=1.01, max_steps=4000)
    out = [(kerr, abi.default_config(enable_volumetric=1, n_bins=8, **base), 2, 0),
           (kerr, abi.default_config(compat=1), 1, 0),
           (kerr, abi.default_config(**base), 1, 1)]
    window = abi.make_frame(kerr.metric, kerr.camera, 0.0, 20.0, row_begin=3, row_count=4)
    out.append((window, abi.default_config(**base), 2, 0))
    cam = abi.make_camera(r=15.0, theta_deg=80.0, width=8, height=4, projection=abi.CAMERA_EQUIRECTANGULAR)
    kn = abi.make_frame(abi.make_metric(a=0.998, Q=0.05), cam, 0.0, 30.0)
    out.append((kn, abi.default_config(integrator=abi.INTEGRATOR_SYMPLECTIC, symplectic_order=4,
                                       symplectic_step=0.05, projection_period=8, max_steps=3000,
                                       escape_radius=60.0, horizon_factor=1.01, enable_volumetric=1, n_bins=4), 2, 0))
    mt = abi.make_frame(abi.make_metric(family=abi.MORRIS_THORNE, b0=1.3),
                        abi.make_camera(r=30.0, theta_deg=80.0, width=6, height=6, fov=40.0), 0.0, 25.0)
    alc = abi.make_frame(abi.make_metric(family=abi.ALCUBIERRE, vs=1.5, sigma=8.0, R=1.0),
                         abi.make_camera(r=20.0, theta_deg=80.0, width=6, height=6, fov=40.0), 0.0, 25.0)
    out += [(mt, abi.default_config(**base), 1, 0), (alc, abi.default_config(**base), 1, 0)]
    return out


def test_oracle_under_address_and_ub_sanitizers(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    drv = tmp_path / "driver.cpp"
    drv.write_text(DRIVER)
    exe = tmp_path / "oracle_asan"
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "oracle", "oracle_capi.cpp"), str(drv), "-o", str(exe), "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr and "cannot find" in r.stderr:
        pytest.skip("sanitizer runtime not installed")
    assert r.returncode == 0, r.stderr[-3000:]
    data = bytearray(np.int32(len(cases())).tobytes())
    for fr, cfg, threads, prec in cases():
        data += bytes(fr) + bytes(cfg) + np.int32(threads).tobytes() + np.int32(prec).tobytes()
    inp = tmp_path / "cases.bin"
    inp.write_bytes(bytes(data))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    run = subprocess.run([str(exe), str(inp)], capture_output=True, text=True, timeout=600, env=env)
    assert run.returncode == 0, (run.stdout + run.stderr)[-4000:]
    assert "ERROR: AddressSanitizer" not in run.stderr and "runtime error" not in run.stderr, run.stderr[-4000:]
    assert f"case {len(cases()) - 1}:" in run.stdout

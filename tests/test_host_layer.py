"""Builds tests/cpp/test_host_layer.cpp against include/sirius_b200.hpp and
libsirius_b200.so and runs it: CPU checks here, device checks under -m gpu."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_host_layer.cpp")
LIBDIR = os.path.join(ROOT, "sirius_b200")


@pytest.fixture(scope="module")
def binary(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "test_host_layer")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
                    "-L", LIBDIR, "-lsirius_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return out


def test_host_layer_cpu(binary):
    r = subprocess.run([binary], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_host_layer_gpu(binary):
    r = subprocess.run([binary, "--gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

"""The reference-side adapter compiles against the reference's own IAccelerator
header and links against the library.

The adapter (CUDAAccelerator in sirius_b200/host/reference_adapter/RDCA001A.h,
the class a maintainer adds beside the reserved BackendType::CUDA slot,
src/Sirius.Render/Acceleration/Backend/ACIB001A.h:27,148-189) is built as it
stands against the real ACIB001A.h of a reference checkout and linked against
libsirius_b200.so. Without a GPU the
program checks that initialise() fails cleanly (no CUDA device) rather than
crashing. Skipped where no reference checkout is present (the checkout is read at
build and test time only)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MAIN = r'''
#include "CUDA/RDCA001A.h"
#include <cstdio>
#include <memory>
using namespace Sirius::Acceleration;
int main() {
    std::unique_ptr<IAccelerator> acc = std::make_unique<CUDA::CUDAAccelerator>();
    if (acc->getType() != BackendType::CUDA) return 2;
    const bool ok = acc->initialise(64, 48);
    if (ok) {
        LaunchConfig lc;
        lc.width = 64; lc.height = 48; lc.blackHoleSpin = 0.9f; lc.observerDistance = 100.0f;
        acc->launch(lc);
        if (!acc->getLastError().empty()) { std::printf("launch: %s\n", acc->getLastError().c_str()); return 3; }
        if (acc->getFrameBufferSize() != size_t(64) * 48 * 4 * sizeof(float)) return 4;
        std::printf("traced %zu bytes\n", acc->getFrameBufferSize());
    } else {
        std::printf("initialise: %s\n", acc->getLastError().c_str());
    }
    acc->cleanup();
    return 0;
}
'''


def reference_root():
    from __graft_entry__ import REFERENCE_ROOT
    return os.environ.get("SIRIUS_REFERENCE_ROOT", REFERENCE_ROOT)


def adapter_source():
    with open(os.path.join(ROOT, "sirius_b200", "host", "reference_adapter", "RDCA001A.h")) as f:
        return f.read()


def test_adapter_compiles_against_the_reference_interface(tmp_path):
    acib = os.path.join(reference_root(), "src", "Sirius.Render", "Acceleration", "Backend", "ACIB001A.h")
    if not os.path.exists(acib):
        pytest.skip("no reference checkout on this host")
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    from sirius_b200.engine import LIB_PATH, load_library
    load_library()  # builds the library if needed
    (tmp_path / "CUDA").mkdir()
    (tmp_path / "Backend").mkdir()
    # the adapter includes "../Backend/ACIB001A.h"; that name forwards to the reference's file
    (tmp_path / "Backend" / "ACIB001A.h").write_text(f'#include "{acib}"\n')
    (tmp_path / "CUDA" / "RDCA001A.h").write_text(adapter_source())
    (tmp_path / "main.cpp").write_text(MAIN)
    exe = tmp_path / "adapter"
    libdir = os.path.dirname(LIB_PATH)
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-I", str(tmp_path), "-I", os.path.join(ROOT, "include"),
           str(tmp_path / "main.cpp"), "-o", str(exe), "-L", libdir, "-lsirius_b200", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "initialise:" in run.stdout or "traced" in run.stdout

"""Without a GPU the library refuses loudly: there is no CPU fallback.

The Python virtual grid raises on creation, and the C++ drop-in's Decomp
raises std::runtime_error from its device selection (the reference's
src/runtime.cpp:149-231 does the same for a rank without a device), rather
than running the path anywhere else.  Skipped where a GPU is visible."""
import os
import shutil
import subprocess

import pytest

import dsdecompx_b200 as dsx
from dsdecompx_b200 import _build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def gpu_visible():
    import torch
    return torch.cuda.is_available()


pytestmark = pytest.mark.skipif(gpu_visible(), reason="a GPU is visible")


def test_virtual_grid_refuses_without_a_device():
    with pytest.raises(RuntimeError, match="(?i)cuda"):
        dsx.VirtualGrid(8, (2, 2, 2), "manual", (0, 0, 0), (10, 10, 10), halo_width=1.0,
                        particles=100)


PROGRAM = r"""
#include <dsdecompx.hpp>
#include <cstdio>
#include <cstring>
#include <stdexcept>

int main(int argc, char** argv) {
    int provided = 0;
    MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
    dsdecompx::Config config;
    config.domain.upper = {10.0, 10.0, 10.0};
    config.halo.width = 1.5;
    int rc = 1;
    try {
        dsdecompx::Decomp decomp(MPI_COMM_WORLD, config);
        std::puts("constructed");
    } catch (const std::runtime_error& e) {
        std::puts(e.what());
        rc = std::strstr(e.what(), "could not select a CUDA device") ? 0 : 1;
    } catch (const std::exception& e) {
        std::printf("other: %s\n", e.what());
    }
    MPI_Finalize();
    return rc;
}
"""


def test_dropin_decomp_refuses_without_a_device(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    lib = dsx.library_path()
    src = tmp_path / "no_device.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "no_device"
    subprocess.run([cxx, "-std=c++17", "-I", _build.INCLUDE, "-I", _build.MPI_STUB, "-o", str(exe),
                    str(src), "-L", os.path.dirname(lib), "-ldsx",
                    "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "could not select a CUDA device" in run.stdout

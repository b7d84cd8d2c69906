"""A C program against include/bbjd.h and include/bbjd_gpu.h, linked with
libbbjd_gpu.so and run in its own process (no Python or PyTorch in it):
device operators and the reference's host-callback interface both return
the eigenpairs nearest sigma (tests/c/solve_device.c checks them)."""
import os
import subprocess

import pytest

from bbjd_b200 import _lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_c_caller_device_and_callback_solves(tmp_path):
    _lib.load()                                   # builds the library if needed
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "solve_device"
    subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "solve_device.c"), "-o", str(exe),
                    f"-L{libdir}", "-lbbjd_gpu", f"-Wl,-rpath,{libdir}", "-lm"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(out.stdout, out.stderr)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().endswith("ok")

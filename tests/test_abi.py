"""The C-ABI library loads and exports every symbol include/*.h declares, and
the ctypes structs match the C layouts (checked against a C program compiled
from the headers).  CPU only: no compute call is made."""
import os
import re
import subprocess
import tempfile

import ctypes
import pytest

from bbjd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def _declared_functions():
    names = set()
    for h in ("bbjd.h", "bbjd_gpu.h"):
        src = open(os.path.join(INCLUDE, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        src = re.sub(r"typedef[^;]*;", "", src, flags=re.S)
        for m in re.finditer(r"\b(bbjd_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_library_builds_and_loads():
    lib = _lib.load()
    assert b"sm_100a" in lib.bbjd_gpu_version()


@pytest.mark.parametrize("name", _declared_functions())
def test_symbol_exported(name):
    lib = _lib.load()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "bbjd_gpu.h"
#define P(T, F) printf(#T "." #F " %zu\n", offsetof(T, F))
int main(void) {
    printf("params %zu\nresult %zu\nworkspace %zu\next %zu\n", sizeof(bbjd_params),
           sizeof(bbjd_result), sizeof(bbjd_workspace), sizeof(bbjd_device_ext));
    P(bbjd_params, sigma); P(bbjd_params, target); P(bbjd_params, tol); P(bbjd_params, v0);
    P(bbjd_params, matvec_A); P(bbjd_params, precond); P(bbjd_params, op_data); P(bbjd_params, verbose);
    P(bbjd_result, eigenvectors); P(bbjd_result, iters); P(bbjd_result, status);
    P(bbjd_workspace, MA); P(bbjd_workspace, nlock); P(bbjd_workspace, gmres_V);
    P(bbjd_workspace, inner_maxiter); P(bbjd_workspace, swap_nm); P(bbjd_workspace, h_work);
    P(bbjd_device_ext, evec_layout); P(bbjd_device_ext, ritz_estimate);
    P(bbjd_device_ext, seconds_total); P(bbjd_device_ext, kernel_launches);
    P(bbjd_device_ext, duplicates); P(bbjd_device_ext, ritz_refinements);
    P(bbjd_device_ext, ritz_fallbacks); P(bbjd_device_ext, host_overlap);
    P(bbjd_device_ext, conv_iters); P(bbjd_device_ext, seconds_qz_exposed);
    P(bbjd_device_ext, guess_hits); P(bbjd_device_ext, guess_misses);
    P(bbjd_device_ext, kernel_ms); P(bbjd_device_ext, kernel_calls);
    return 0;
}
"""

PYMAP = {"params": _lib.Params, "result": _lib.Result, "workspace": _lib.Workspace,
         "ext": _lib.DeviceExt}
STRUCTS = {"bbjd_params": _lib.Params, "bbjd_result": _lib.Result,
           "bbjd_workspace": _lib.Workspace, "bbjd_device_ext": _lib.DeviceExt}


def test_struct_layouts_match_c():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(PROBE)
        subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    for line in out.strip().splitlines():
        key, val = line.split()
        val = int(val)
        if "." in key:
            sname, field = key.split(".")
            assert getattr(STRUCTS[sname], field).offset == val, key
        else:
            assert ctypes.sizeof(PYMAP[key]) == val, key


def test_reference_header_layout_is_kept():
    """The reference's own header compiles against our struct sizes: the
    fields the reference declares (include/bbjd.h:114-224 there) keep their
    order; our header only appends enum values."""
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.c")
        open(src, "w").write('#include "bbjd.h"\nint main(void){bbjd_params p; bbjd_params_init(&p); return 0;}\n')
        subprocess.run(["gcc", "-std=c11", "-c", "-I", INCLUDE, src, "-o", os.path.join(d, "p.o")],
                       check=True)

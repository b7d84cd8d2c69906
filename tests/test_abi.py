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


REF_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "bbjd.h"
#define P(T, F) printf(#T "." #F " %zu\n", offsetof(T, F))
int main(void) {
    printf("params %zu\nresult %zu\nworkspace %zu\n", sizeof(bbjd_params), sizeof(bbjd_result),
           sizeof(bbjd_workspace));
    P(bbjd_params, n); P(bbjd_params, nev); P(bbjd_params, sigma); P(bbjd_params, target);
    P(bbjd_params, tol); P(bbjd_params, maxiter); P(bbjd_params, maxsub); P(bbjd_params, minsub);
    P(bbjd_params, inner_maxiter); P(bbjd_params, inner_tol); P(bbjd_params, matvec_A);
    P(bbjd_params, matvec_B); P(bbjd_params, precond); P(bbjd_params, op_data);
    P(bbjd_params, verbose); P(bbjd_params, v0);
    P(bbjd_result, nconv); P(bbjd_result, eigenvalues); P(bbjd_result, eigenvectors);
    P(bbjd_result, residuals); P(bbjd_result, iters); P(bbjd_result, status);
    P(bbjd_workspace, n); P(bbjd_workspace, maxsub); P(bbjd_workspace, nev);
    P(bbjd_workspace, V); P(bbjd_workspace, W); P(bbjd_workspace, AV); P(bbjd_workspace, BV);
    P(bbjd_workspace, MA); P(bbjd_workspace, MB); P(bbjd_workspace, SA); P(bbjd_workspace, SB);
    P(bbjd_workspace, ZA); P(bbjd_workspace, ZB); P(bbjd_workspace, nlock); P(bbjd_workspace, kdim);
    P(bbjd_workspace, gmres_V); P(bbjd_workspace, gmres_H); P(bbjd_workspace, gmres_cs);
    P(bbjd_workspace, gmres_sn); P(bbjd_workspace, gmres_g); P(bbjd_workspace, inner_maxiter);
    P(bbjd_workspace, tmp1); P(bbjd_workspace, tmp4); P(bbjd_workspace, swap_nm);
    P(bbjd_workspace, Q_right); P(bbjd_workspace, Q_left); P(bbjd_workspace, h_work);
    printf("BBJD_SUCCESS %d BBJD_MAX_ITER %d BBJD_ERR_ALLOC %d BBJD_ERR_INVALID %d "
           "BBJD_ERR_CALLBACK %d BBJD_ERR_LAPACK %d BBJD_ERR_BREAKDOWN %d\n",
           BBJD_SUCCESS, BBJD_MAX_ITER, BBJD_ERR_ALLOC, BBJD_ERR_INVALID, BBJD_ERR_CALLBACK,
           BBJD_ERR_LAPACK, BBJD_ERR_BREAKDOWN);
    printf("targets %d %d %d %d %d %d %d\n", BBJD_TARGET_NEAREST, BBJD_TARGET_LARGEST_MAG,
           BBJD_TARGET_SMALLEST_MAG, BBJD_TARGET_LARGEST_REAL, BBJD_TARGET_SMALLEST_REAL,
           BBJD_TARGET_LARGEST_IMAG, BBJD_TARGET_SMALLEST_IMAG);
    return 0;
}
"""


def _probe(include_dir):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(src, "w").write(REF_PROBE)
        subprocess.run(["gcc", "-std=c11", "-I", include_dir, src, "-o", exe], check=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout


REFERENCE = os.environ.get("BBJD_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "include", "bbjd.h")),
                    reason="the reference checkout is not on this machine ($BBJD_REFERENCE)")
def test_layouts_identical_to_the_reference_header():
    """The same probe compiled against the reference's own include/bbjd.h
    and against ours: every size, offset and enum value the reference
    declares is identical (its include/bbjd.h:61-224)."""
    assert _probe(os.path.join(REFERENCE, "include")) == _probe(INCLUDE)


def test_reference_probe_compiles_against_our_header():
    """Without the reference checkout (the GPU box), the probe of the
    reference's declarations still compiles and runs against our header."""
    out = _probe(INCLUDE)
    assert "params" in out and "BBJD_ERR_BREAKDOWN -5" in out

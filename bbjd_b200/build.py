"""Build libbbjd_gpu.so (sm_100a) in-tree with nvcc.

The library is compiled from ``bbjd_b200/csrc/*.cu`` for ``sm_100a`` only
and linked against the LAPACK the reference itself links (scipy's bundled
OpenBLAS, symbol prefix ``scipy_``) for the small projected QZ.  Output:
``bbjd_b200/_build/libbbjd_gpu.so``.
"""
from __future__ import annotations

import glob
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libbbjd_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def openblas() -> tuple[str, str]:
    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
    if not cands:
        raise RuntimeError(f"scipy's bundled OpenBLAS not found under {libdir}")
    return libdir, os.path.basename(cands[0])


def torch_lib_dir() -> str | None:
    """Directory of PyTorch's shared libraries (its bundled MKL, inside
    libtorch_cpu.so, gives the engine a faster ZGEEV), found without
    importing torch; None when torch is not installed."""
    import importlib.util
    spec = importlib.util.find_spec("torch")
    if not spec or not spec.submodule_search_locations:
        return None
    d = os.path.join(list(spec.submodule_search_locations)[0], "lib")
    return d if os.path.exists(os.path.join(d, "libtorch_cpu.so")) else None


def defines() -> list[str]:
    d = torch_lib_dir()
    return [f'-DBBJD_TORCH_LIB="{d}"'] if d else []


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
            sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    h.update(" ".join(ARCH + defines()).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    stamp = os.path.join(OUT_DIR, "libbbjd_gpu.sha256")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == dig:
                return LIB
    libdir, blas = openblas()
    objs = []
    for src in sources():
        obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", *defines(),
               "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, f"-L{libdir}", f"-l:{blas}", "-ldl",
           "-Xlinker", f"-rpath={libdir}"]
    subprocess.run(cmd, check=True)
    with open(stamp, "w") as f:
        f.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

"""Build recipe of the native library ``libns3d_b200.so`` (in-tree, sm_100a).

Translation units and their floating-point contracts:

* ``ns3d_fp64.cu``  -- FP64 stencil kernels, ``-fmad=false`` (no FMA contraction,
  the reference's rounding sequence).
* ``ns3d_fp32.cu``  -- FP32-stencil kernels, FMA contraction on, approximate
  float division/sqrt, denormals flushed.
* ``ns3d_api.cu``   -- C ABI, transfers, reductions, spectrum; ``-fmad=false``.
* ``ns3d_params.cpp`` -- solver.in parser (host only).
* ``ns3d_io.cpp``   -- Tecplot field, residual, spectrum and statistics files (host only).
* ``ns3d_run.cpp``  -- time_advance with its monitor and output (host only).

Run ``python -m ns3d_cpp_b200.build`` (or ``build()``); objects go to
``ns3d_cpp_b200/_build/`` and the library next to this file.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libns3d_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(_nvcc())))


COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}",
          "-ccbin", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"]

UNITS = {
    "ns3d_fp64.cu": ["--fmad=false"],
    "ns3d_fp32.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "ns3d_api.cu": ["--fmad=false"],
    "ns3d_noalloc.cu": ["--fmad=false"],
    "ns3d_adjoint.cu": ["--fmad=true"],
    "ns3d_params.cpp": [],
    "ns3d_io.cpp": [],
    "ns3d_run.cpp": [],
}


def _sources():
    out = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".cpp")):
                out.append(os.path.join(d, f))
    return out


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources())


def _compile(unit: str, extra: list, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    if unit.endswith(".cpp"):
        cmd = ["/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++", "-O2", "-std=c++17",
               "-fPIC", f"-I{INCLUDE}", "-c", src, "-o", obj]
    else:
        cmd = [_nvcc(), *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile of {unit} failed:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every translation unit for sm_100a and link the shared library."""
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    libdir = os.path.join(_cuda_home(), "lib64")
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcufft", "-Xlinker",
           f"-rpath={libdir}"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build the native parts of the B200 path tracer in place.

Outputs (next to this file):
  liblucid_cuda.so                         C ABI (include/lucid_cuda.h), sm_100a kernels
  lucidrenderer.<python-ext-suffix>        pybind11 module with the reference's surface

Run:  python build_ext.py  [--force]
Requires nvcc (CUDA 12.8+ for sm_100a), g++, pybind11 and nlohmann/json
headers.  The CUDA runtime is linked statically so the library loads on any
machine with a recent driver.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wno-unused-function"]

LIB = os.path.join(HERE, "liblucid_cuda.so")
EXT = os.path.join(HERE, "lucidrenderer" + sysconfig.get_config_var("EXT_SUFFIX"))


def nlohmann_include() -> str:
    import site
    for s in site.getsitepackages() + [site.getusersitepackages()]:
        c = os.path.join(s, "include", "cudnn_frontend", "thirdparty")
        if os.path.exists(os.path.join(c, "nlohmann", "json.hpp")):
            return c
    for c in ("/usr/include", "/usr/local/include"):
        if os.path.exists(os.path.join(c, "nlohmann", "json.hpp")):
            return c
    raise RuntimeError("nlohmann/json.hpp not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build(force: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(REPO, "include", "lucid_cuda.h")]
    inc = ["-I" + CSRC, "-I" + os.path.join(REPO, "include"), "-I" + nlohmann_include(),
           "-I" + os.path.join(CUDA_HOME, "include")]
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            _run([NVCC] + ARCH + NVCC_FLAGS + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))):
        if os.path.basename(src) == "pybind_module.cpp":
            continue
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + headers):
            _run([CXX] + CXX_FLAGS + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                                                 "-lpthread"])
    # pybind11 module
    import pybind11
    src = os.path.join(CSRC, "pybind_module.cpp")
    if os.path.exists(src) and (force or _stale(EXT, [src, LIB] + headers)):
        py_inc = sysconfig.get_paths()["include"]
        _run([CXX] + CXX_FLAGS + ["-shared", "-I" + pybind11.get_include(), "-I" + py_inc] + inc +
             [src, "-o", EXT, "-L" + HERE, "-llucid_cuda", "-Wl,-rpath,$ORIGIN"])


if __name__ == "__main__":
    build(force="--force" in sys.argv)

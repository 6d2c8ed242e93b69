"""Build recipe for the in-tree native libraries (sm_100a only).

* ``gp5_b200/libgp5cu.so``   CUDA kernels + the C ABI of include/gp5cu.h (nvcc)
* ``gp5_b200/gpCpp*.so``     pybind11 module mirroring the reference's ``gpCpp``
                              (src/gpCpp.cpp:327-371), a C++ client of the C ABI

Objects are compiled in parallel and relinked only when a source is newer than the target.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgp5cu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["gp5cu_f64.cu", "gp5cu_f32.cu", "gp5cu_host.cu", "gp5cu_batch.cu", "gp5cu_noalloc.cu", "mlp.cu",
              "gp5cu_cluster.cu", "gp5cu_h5.cpp"]
HEADERS = ["common.cuh", "fft_line.cuh", "passes.cuh", "ops.cuh", "ring.cuh", "launch_impl.cuh", "plan.hpp"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def pybind_ext_path() -> str:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.join(HERE, "gpCpp" + suffix)


def build_lib(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "gp5cu.h")]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", s, "-o", o])
    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            outs = list(ex.map(_run, jobs))
        if verbose or ptxas_info:
            for o in outs:
                sys.stdout.write(o)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    return LIB


def build_pybind(verbose: bool = False) -> str:
    import pybind11

    out = pybind_ext_path()
    src = os.path.join(CSRC, "gpCpp.cpp")
    if not _newer(out, [src, LIB, os.path.join(ROOT, "include", "gp5cu.h")]):
        return out
    inc = sysconfig.get_paths()["include"]
    cmd = ["g++", "-O2", "-shared", "-fPIC", "-std=c++17", "-I" + pybind11.get_include(), "-I" + inc,
           "-I" + os.path.join(ROOT, "include"), src, "-o", out, "-L" + HERE, "-lgp5cu",
           "-Wl,-rpath,$ORIGIN"]
    _run(cmd)
    return out


def build(verbose: bool = False) -> None:
    build_lib(verbose)
    if os.path.exists(os.path.join(CSRC, "gpCpp.cpp")):
        build_pybind(verbose)


if __name__ == "__main__":
    build(verbose=True)
    print("built", LIB)

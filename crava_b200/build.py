"""Build the CUDA library in-tree: crava_b200/libcrava_gpu.so (sm_100a).

    python -m crava_b200.build          # build if sources are newer than the library
    python -m crava_b200.build --force
"""
from __future__ import annotations

import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcrava_gpu.so")
SOURCES = ["crava_api.cu", "kernels.cu", "fft4.cu", "fft4_p1.cu", "fft4_p2.cu", "fft4_p3.cu", "fft4_p4.cu", "fft4_p5.cu", "fft4_p6.cu", "zpass.cu", "zpass_n12.cu", "zpass_n34.cu", "zpass_n56.cu", "zpass_n78.cu", "pencil.cu", "pencil_s1.cu", "pencil_s2.cu", "pencil_s3.cu", "localnoise.cu", "gridio.cu", "facies.cu", "thick.cu", "prior.cu", "segy.cu"]
HEADERS = ["fft_core.cuh", "fft2.cuh", "fft4.cuh", "kernels.cuh", "pencil_common.cuh", "pencil.cuh", "zpass.cuh", "facies.cuh", "fft4_facies.cuh", "ibm_float.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "crava_gpu.h")]
    if not force and not _newer(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    shared = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "crava_gpu.h")]

    def compile_one(s):
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        # an object is reused when it is newer than its source and every shared header
        if not force and not ptxas_info and not _newer(obj, [src] + shared):
            return s, obj, None
        cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        return s, obj, subprocess.run(cmd, capture_output=True, text=True)

    objs = []
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        for s, obj, r in ex.map(compile_one, SOURCES):
            if r is not None and r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {s}:\n{r.stdout}\n{r.stderr}")
            if r is not None and ptxas_info:
                sys.stderr.write(r.stderr)
            objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


HOST = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libcrava_host.so")
HOST_DEMO = os.path.join(HOST, "avo_host_demo")
CXX = os.environ.get("CXX", "g++")


def build_host(force: bool = False, verbose: bool = False) -> str:
    """The C++ host layer (FFTGrid / AVOInversion over the C ABI) and its demo driver."""
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + HOST]
    steps = [
        (HOST_LIB, [os.path.join(HOST, "crava_host.cpp"), os.path.join(HOST, "crava_host.h"), LIB],
         [CXX, "-std=c++17", "-O2", "-fPIC", "-Wall", "-shared"] + inc +
         [os.path.join(HOST, "crava_host.cpp"), "-L" + HERE, "-lcrava_gpu", "-Wl,-rpath,$ORIGIN", "-o", HOST_LIB]),
        (HOST_DEMO, [os.path.join(HOST, "avo_host_demo.cpp"), os.path.join(HOST, "crava_host.h"), HOST_LIB],
         [CXX, "-std=c++17", "-O2", "-Wall"] + inc +
         [os.path.join(HOST, "avo_host_demo.cpp"), "-L" + HERE, "-lcrava_host", "-lcrava_gpu",
          "-Wl,-rpath,$ORIGIN/..", "-o", HOST_DEMO]),
    ]
    for target, deps, cmd in steps:
        if not force and not _newer(target, deps):
            continue
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"host build failed for {target}:\n{r.stdout}\n{r.stderr}")
    return HOST_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    build_host(force="--force" in sys.argv, verbose=True)
    print(LIB)

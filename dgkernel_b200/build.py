"""Build libdgk.so in-tree for sm_100a (nvcc + g++), so the library travels with the repository."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdgk.so")
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
CUDA_INC = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(NVCC))), "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INC = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
CXXFLAGS = ["-O3", "-std=c++17"]

CU = ["kernels.cu", "kernels_tma.cu", "setup.cu", "ops.cu", "noalloc.cu", "mixed.cu", "av.cu", "tcm.cu", "oz.cu", "exchange.cu", "lsens.cu"]
CPP = ["runner.cpp", "element.cpp", "mesh.cpp", "gambit.cpp", "abi.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _obj(src):
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _stale(src, obj):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "dgk.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    jobs = []
    for src in CU:
        extra = ["-Xptxas", "-v"] if ptxas_info else []
        jobs.append((src, [NVCC, *ARCH, "-lineinfo", *CXXFLAGS, "-Xcompiler", "-fPIC", *INC, *extra, "-c",
                           os.path.join(CSRC, src), "-o", _obj(src)]))
    for src in CPP:
        jobs.append((src, [CXX, *CXXFLAGS, "-fPIC", *INC, "-I" + CUDA_INC, "-c", os.path.join(CSRC, src), "-o",
                           _obj(src)]))
    todo = [(s, c) for s, c in jobs if _stale(s, _obj(s)) or ptxas_info]
    logs = []
    with ThreadPoolExecutor(max_workers=min(8, len(todo) or 1)) as ex:
        for out in ex.map(lambda sc: _run(sc[1]), todo):
            logs.append(out)
    if todo or not os.path.exists(LIB):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *[_obj(s) for s, _ in jobs], "-lcudart"])
    if verbose:
        sys.stdout.write("".join(logs))
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)

"""Build libpumatch_b200.so and the `test` CLI in-tree for sm_100a.

    python -m pumatch_b200.build        (or pumatch_b200.build.build())

Outputs: pumatch_b200/lib/libpumatch_b200.so, pumatch_b200/bin/test.
Objects go to pumatch_b200/_build/ (ignored by git).  Rebuilds only what is
older than its sources.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libpumatch_b200.so")
CLI = os.path.join(PKG, "bin", "test")
CONVERT = os.path.join(PKG, "bin", "convert")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["pm_device.cu", "pm_paging.cu", "pm_learn.cu", "pm_gen.cu"]
CPP_SOURCES = ["pm_host.cpp", "pm_parts.cpp"]
HEADERS = ["pm_common.h", "pm_device.cuh"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INC, "pumatch.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp",
                   "-I", INC, "-I", CSRC, "-c", "-o", o, s]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd)
            if verbose or ptxas_info:
                sys.stderr.write(r.stderr)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            _run(["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function",
                  "-I", INC, "-I", CSRC, f"-I{CUDA}/include", "-c", "-o", o, s])
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    cli_src = os.path.join(CSRC, "pm_cli.cpp")
    if _stale(CLI, [cli_src, LIB, os.path.join(INC, "pumatch.h")]):
        _run(["g++", "-O2", "-std=c++17", "-I", INC, "-o", CLI, cli_src,
              "-L", os.path.dirname(LIB), "-lpumatch_b200",
              "-Wl,-rpath,$ORIGIN/../lib"])
    conv_src = os.path.join(CSRC, "pm_convert_cli.cpp")
    if _stale(CONVERT, [conv_src, LIB, os.path.join(INC, "pumatch.h")]):
        _run(["g++", "-O2", "-std=c++17", "-I", INC, "-o", CONVERT, conv_src,
              "-L", os.path.dirname(LIB), "-lpumatch_b200", "-Wl,-rpath,$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)

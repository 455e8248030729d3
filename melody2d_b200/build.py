"""Builds libmelgpu.so (the C-ABI library of include/melgpu.h) in-tree for sm_100a.

    python -m melody2d_b200.build            # library only
    python -m melody2d_b200.build --all      # library + oracle checkers (oracle/Makefile)

The FP64 kernels are compiled with -fmad=false so that every multiply and add rounds as in the
reference (x86-64 SSE2 arithmetic); see the operation-order notes in csrc/mel_kernels.cu."""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmelgpu.so")
EXE = os.path.join(HERE, "melody_gpu")
BUILD = os.path.join(HERE, "_build")

CU_SOURCES = ["mel_kernels.cu", "mel_prox.cu", "mel_model.cu", "mel_noalloc.cu", "mel_monitor.cu", "mel_mls.cu"]
CPP_SOURCES = ["mel_loader.cpp", "mel_chunks.cpp", "mel_material.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "melgpu.h"))
    objs = []
    common = ["-O3", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-Xcompiler", "-fPIC"]
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + headers):
            cmd = [nvcc()] + ARCH + common + ["-lineinfo", "-fmad=false", "-Xptxas", "-warn-spills", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _newer(o, [s] + headers):
            cmd = [nvcc()] + ARCH + common + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(o)
    if force or _newer(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    main_src = os.path.join(CSRC, "melody_gpu_main.cpp")
    if force or _newer(EXE, [main_src, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), main_src, "-o", EXE,
               "-L" + HERE, "-lmelgpu", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all"], check=True)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--all", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(force=a.force, verbose=a.verbose)
    if a.all:
        build_oracle()
    return 0


if __name__ == "__main__":
    sys.exit(main())

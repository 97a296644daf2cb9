"""Build recipe for the native parts of perft_gpu_2026_b200.

    python -m perft_gpu_2026_b200.build            # library + CLI
    python -m perft_gpu_2026_b200.build --oracle   # also the test oracle (and the
                                                   # reference binary when
                                                   # PERFT_REFERENCE_DIR is set)

Outputs (in-tree, git-ignored, shipped with the repository snapshot):
  perft_gpu_2026_b200/libperftb200.so   CUDA kernels for sm_100a + host driver + C ABI
  perft_gpu_2026_b200/perft_gpu         the command line (links the library)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libperftb200.so")
CLI = os.path.join(PKG, "perft_gpu")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared"] + ARCH


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources():
    out = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".inc", ".h"))]
    out.append(os.path.join(ROOT, "include", "perft_b200.h"))
    return out


def build_library(force: bool = False, extra=()) -> str:
    if force or _newer(LIB, _sources()):
        cmd = [_nvcc()] + NVCC_FLAGS + list(extra) + ["-o", LIB, os.path.join(CSRC, "pb_engine.cu")]
        subprocess.run(cmd, check=True)
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "perft_cli.cpp")
    if force or _newer(CLI, [src, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", "-o", CLI, src, "-L" + PKG, "-lperftb200", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return CLI


def build_oracle(reference_dir: str | None = None) -> None:
    """The checker: oracle/liboracle.so, and oracle/_ref/perft_gpu_ref when a
    directory holding the reference sources is given (argument, else the
    PERFT_REFERENCE_DIR environment variable)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    ref = reference_dir or os.environ.get("PERFT_REFERENCE_DIR")
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + ref], check=True)


def build_all(force: bool = False, oracle: bool = True, reference_dir: str | None = None) -> None:
    build_library(force)
    build_cli(force)
    if oracle:
        build_oracle(reference_dir)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, oracle="--oracle" in sys.argv)

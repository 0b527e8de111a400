"""Build recipe for the native libraries (in-tree, sm_100a).

    python -m lda_sc20_b200.build            # product library + oracle

Products:
  lda_sc20_b200/liblda_b200.so   CUDA kernels, C ABI, host corpus code, ezlda_compat CLI
  lda_sc20_b200/ezlda_compat     EZLDA-style command-line driver
  oracle/liblda_oracle.so        CPU oracle (test infrastructure; built here, never linked
                                 into the product)
"""
from __future__ import annotations

import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lda_sc20_b200")
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-I" + INC]
# extra nvcc flags for tuning builds (e.g. LDA_NVFLAGS="-DLDA_SAMPLE_TILE=256")
NVFLAGS += os.environ.get("LDA_NVFLAGS", "").split()

LIB_SOURCES = ["trainer.cu", "serving.cu", "batch.cu", "corpus.cpp"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False) -> str:
    out = os.path.join(PKG, "liblda_b200.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INC, "lda_b200.h")]
    if force or _stale(out, deps):
        _run([NVCC] + NVFLAGS + ["-shared", "-o", out] + [os.path.join(CSRC, s) for s in LIB_SOURCES])
    cli = os.path.join(PKG, "ezlda_compat")
    cli_src = os.path.join(CSRC, "ezlda_compat.cpp")
    if os.path.exists(cli_src) and (force or _stale(cli, [cli_src, out])):
        _run(["g++", "-O2", "-std=c++17", "-I" + INC, "-o", cli, cli_src, "-L" + PKG, "-llda_b200",
              "-Wl,-rpath,$ORIGIN"])
    return out


def build_oracle(force: bool = False) -> str:
    odir = os.path.join(ROOT, "oracle")
    out = os.path.join(odir, "liblda_oracle.so")
    src = [os.path.join(odir, "lda_oracle.c"), os.path.join(odir, "lda_oracle.h")]
    if force or _stale(out, src):
        # -ffp-contract=off: every float operation is a separate IEEE operation, as in the kernels
        _run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", out,
              src[0], "-lm", "-lpthread"])
    return out


def build_all(force: bool = False) -> None:
    build_library(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)

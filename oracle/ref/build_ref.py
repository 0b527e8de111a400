"""Builds the reference harness into oracle/_ref/ from the reference's own sources.

TEST INFRASTRUCTURE ONLY.  Compiles every EZLDA/*.cu of the reference except
mainKernel.cu (whose main() oracle/ref/ref_harness.cu replaces) for sm_100a, with
oracle/ref/legacy_shim.h force-included so the pre-Volta warp intrinsics resolve.  The
sources are read where they lie; nothing is copied into this repository.  The EZLDA
source directory is passed as an argument (or in EZLDA_SRC); with neither, nothing is
built.  GPU machines have no reference checkout and use the prebuilt binary.

    python oracle/ref/build_ref.py <reference checkout>/EZLDA [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
REF_SOURCES = ["utility.cu", "DTUpdateKernel.cu", "WTUpdateKernel.cu", "WTDenUpdateKernel.cu", "WTAddKernel.cu",
               "SamplingKernel.cu", "Doc.cu", "DataChunk.cu", "DT.cu", "WT.cu", "WTChunk.cu", "WTDense.cu"]


def build(src: str | None = None, force: bool = False) -> str | None:
    REF_EZLDA = src or os.environ.get("EZLDA_SRC", "")
    if not REF_EZLDA or not os.path.isdir(REF_EZLDA):
        return None
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, "ref_harness")
    srcs = [os.path.join(REF_EZLDA, s) for s in REF_SOURCES] + [os.path.join(HERE, "ref_harness.cu")]
    deps = srcs + [os.path.join(HERE, "legacy_shim.h")]
    if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    objs = []
    for s in srcs:
        o = os.path.join(OUT_DIR, os.path.basename(s).replace(".cu", ".o"))
        cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14", "-w",
               "-include", os.path.join(HERE, "legacy_shim.h"), "-I" + REF_EZLDA, "-c", s, "-o", o]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(o)
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out] + objs, check=True)
    for o in objs:
        os.remove(o)
    return out


if __name__ == "__main__":
    pos = [a for a in sys.argv[1:] if not a.startswith("--")]
    print(build(pos[0] if pos else None, force="--force" in sys.argv))

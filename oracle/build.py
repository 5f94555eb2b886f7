"""TEST INFRASTRUCTURE: builds the CPU oracle and, where the reference's
sources are present, the reference's own C++ filter kernel.

  oracle/_build/librefcpu.so  — oracle/refcpu.cpp (C++17, -O3 -ffp-contract=off)
  oracle/_ref/libreffilter.so — bench/simd_filter/cpp/filter_kernel.cpp of the
                                vexq repository, compiled from where it lies
                                (-O3 -mavx2, the flags of bench/simd_filter/Makefile)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the vexq checkout: VEXQ_REFERENCE_ROOT, else a directory named "reference"
# beside this repository (absent on machines that only run the prebuilt files)
REF_ROOT = os.environ.get("VEXQ_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
REF_FILTER_SRC = os.path.join(REF_ROOT, "bench", "simd_filter", "cpp", "filter_kernel.cpp")
ORACLE_SO = os.path.join(HERE, "_build", "librefcpu.so")
REF_FILTER_SO = os.path.join(HERE, "_ref", "libreffilter.so")


def _newer(target: str, *sources: str) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "refcpu.cpp")
    hdrs = [os.path.join(HERE, "refcpu.h"), os.path.join(HERE, "..", "include", "vexq_cuda.h")]
    if not force and _newer(ORACLE_SO, src, *hdrs):
        return ORACLE_SO
    os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
    tmp = ORACLE_SO + ".tmp"
    subprocess.check_call(["g++", "-std=c++17", "-O3", "-ffp-contract=off", "-fPIC", "-shared",
                           "-Wall", "-o", tmp, src, "-lpthread"])
    os.replace(tmp, ORACLE_SO)
    return ORACLE_SO


def build_ref_filter(force: bool = False) -> str | None:
    """Compiles the reference's AVX2 filter kernel when its source is here."""
    if not os.path.exists(REF_FILTER_SRC):
        return REF_FILTER_SO if os.path.exists(REF_FILTER_SO) else None
    if not force and _newer(REF_FILTER_SO, REF_FILTER_SRC):
        return REF_FILTER_SO
    os.makedirs(os.path.dirname(REF_FILTER_SO), exist_ok=True)
    tmp = REF_FILTER_SO + ".tmp"
    subprocess.check_call(["g++", "-std=c++17", "-O3", "-mavx2", "-fPIC", "-shared",
                           "-o", tmp, REF_FILTER_SRC])
    os.replace(tmp, REF_FILTER_SO)
    return REF_FILTER_SO


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_ref_filter(force))

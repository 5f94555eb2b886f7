"""Builds libvexqcuda.so in-tree for sm_100a.

The CUDA sources compile with nvcc (-gencode arch=compute_100a,code=sm_100a);
the device prelude used by the query-specialised kernels (kparams.h +
device_common.cuh) is embedded as a string for NVRTC. cudart is linked
statically and NVRTC dynamically (rpath to the CUDA toolkit), so the library
loads on a host without a GPU driver.

    python -m vexq_b200.build [--force]
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libvexqcuda.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

SOURCES = ["table.cu", "run.cu", "compile.cpp", "jit.cpp", "abi.cpp", "serve.cpp", "noalloc.cu", "batch.cu", "vxq.cu",
           "select.cu", "shard.cpp", "tune.cpp"]
HEADERS = ["internal.h", "plan.h", "kparams.h", "device_common.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-fno-strict-aliasing",
         "-I", os.path.join(HERE, "..", "include")]


def _prelude() -> str:
    parts = []
    for name in ("kparams.h", "device_common.cuh"):
        with open(os.path.join(CSRC, name)) as f:
            txt = f.read().replace("#pragma once", "")
        parts.append(f"// ---- {name} ----\n{txt}")
    return "\n".join(parts)


def _write_prelude_source() -> str:
    src = _prelude()
    out = os.path.join(BUILD, "prelude.cpp")
    body = ('// generated by vexq_b200/build.py from kparams.h + device_common.cuh\n'
            'namespace vq {\nconst char* prelude_source() {\n    return R"VQPRELUDE(\n'
            + src + '\n)VQPRELUDE";\n}\n}  // namespace vq\n')
    if not os.path.exists(out) or open(out).read() != body:
        with open(out, "w") as f:
            f.write(body)
    return out


def _stamp(paths) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as f:
            h.update(f.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    prelude = _write_prelude_source()
    srcs = [os.path.join(CSRC, s) for s in SOURCES] + [prelude]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "vexq_cuda.h")]
    stamp = _stamp(srcs + hdrs)
    stamp_file = os.path.join(BUILD, "lib.stamp")
    if not force and os.path.exists(LIB) and os.path.exists(stamp_file) and open(stamp_file).read() == stamp:
        return LIB
    objs = []
    procs = []
    for s in srcs:
        obj = os.path.join(BUILD, os.path.basename(s) + ".o")
        cmd = [NVCC] + ARCH + FLAGS + ["-c", s, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((s, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    tmp = LIB + ".tmp"
    link = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + [
        "-cudart", "static", "-lnvrtc", "-L", os.path.join(CUDA, "lib64"),
        "-Xlinker", "-rpath," + os.path.join(CUDA, "lib64"), "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(link))
    subprocess.check_call(link)
    os.replace(tmp, LIB)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

"""Builds libkdb_b200.so (in-tree) with nvcc for sm_100a.

The device runtime header (csrc/device_runtime.cuh) is embedded into the
library as a string: NVRTC prepends it to every generated pipeline kernel.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libkdb_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["kernels.cu", "batch.cu", "engine.cc", "codegen.cc", "capi.cc", "server.cc", "join_prior.cu",
           "operators.cu", "capi_ops.cc"]
HEADERS = ["engine.h", "plan.h", "json.h", "host_result.h", "capi_internal.h", "join_prior.h", "device_runtime.cuh",
           "operators.h"]


def _embed_runtime():
    src = open(os.path.join(CSRC, "device_runtime.cuh")).read()
    out = os.path.join(CSRC, "device_runtime.inc")
    # split into chunks to stay under compiler string-literal limits
    chunks = [src[i:i + 12000] for i in range(0, len(src), 12000)]
    body = "\n".join('R"KDBRT(' + c + ')KDBRT"' for c in chunks)
    old = open(out).read() if os.path.exists(out) else None
    if old != body:
        with open(out, "w") as f:
            f.write(body)


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = SOURCES + HEADERS + ["../build.py", "../../include/kdb_b200.h"]
    return any(os.path.getmtime(os.path.join(CSRC, d)) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    _embed_runtime()
    if not force and not _stale():
        return LIB
    cmd = [NVCC, "-shared", "-Xcompiler", "-fPIC", "-std=c++17", "-O3", "-lineinfo",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I" + CSRC, "-I" + os.path.join(HERE, "..", "include"),
           "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES] + [
           "-lnvrtc", "-cudart", "static",
           "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)

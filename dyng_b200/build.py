"""Build the dyng_b200 CUDA library in-tree: dyng_b200/libdyngb200.so (sm_100a).

    python -m dyng_b200.build [--debug]

nvcc cross-compiles without a GPU.  The library is a plain shared object with the C ABI of
include/dyngb200.h; Python (dyng_b200/__init__.py) binds it with ctypes and the C++17 shim
(include/dyng/*.hpp) links it directly.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdyngb200.so")
SOURCES = ["memory.cu", "graph.cu", "sssp.cu", "operators.cu", "mlp.cu", "capi.cu", "serve.cu", "mosp.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def flags(debug=False):
    f = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"] + ARCH
    if debug:
        f += ["-DDYNGB200_DEBUG=1"]
    return f


def newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(debug=False, force=False, verbose=False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES]
    deps += [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".hpp"))]
    deps += [os.path.join(ROOT, "include", "dyngb200.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest(deps):
        return LIB
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    procs = []
    for s in SOURCES:
        obj = os.path.join(build_dir, s.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [NVCC, "-c", os.path.join(CSRC, s), "-o", obj] + flags(debug)
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose:
            sys.stdout.write(out.decode())
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, "-shared", "-o", tmp] + objs + ARCH + ["-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(debug="--debug" in sys.argv, force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)

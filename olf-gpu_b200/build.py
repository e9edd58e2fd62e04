"""Builds the engine's shared library ``lib/libolfgpu_b200.so`` for sm_100a with nvcc (in-tree, no JIT cache)."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
LIB = os.path.join(OUT, "libolfgpu_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-Xptxas", "-O3"]
SOURCES = ["structure.cpp", "kernels.cu", "persistent.cu", "coop.cu", "front.cu", "region.cu", "engine.cu", "noalloc.cu", "gnn.cu", "violations.cu",
           "capi.cu"]


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OUT, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".hpp", ".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "olfgpu_b200.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps if os.path.exists(d)):
        return obj
    lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
    cmd = [NVCC] + ARCH + FLAGS + lang + ["-c", path, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return obj


JNI_SRC = os.path.join(HERE, "jni", "olfgpu_jni.cpp")
JNI_LIB = os.path.join(OUT, "libolfgpu.so")


def _build_jni(verbose: bool) -> str:
    """The JNI layer (lib/libolfgpu.so, the library name the Java side loads): plain C++ over the engine's C ABI,
    linked against lib/libolfgpu_b200.so (found next to it at run time); only the JNI symbols are exported."""
    deps = [JNI_SRC, os.path.join(HERE, "jni", "jni.h"), os.path.join(HERE, "..", "include", "olfgpu_b200.h"), LIB]
    if os.path.exists(JNI_LIB) and all(os.path.getmtime(JNI_LIB) >= os.path.getmtime(d) for d in deps):
        return JNI_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden", "-Wall", "-o", JNI_LIB, JNI_SRC,
           "-L" + OUT, "-lolfgpu_b200", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return JNI_LIB


def build(verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    _build_jni(verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

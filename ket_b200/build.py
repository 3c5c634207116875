"""Build the engine's shared library, ket_b200/libket_sv.so, with nvcc for sm_100a.

Each translation unit in ket_b200/csrc is compiled separately (in parallel)
and linked into one C-ABI shared library whose exported symbols are exactly the
functions of include/ket_sv.h.  The library is built in-tree so that it ships
with the repository snapshot to the GPU host.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libket_sv.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
          "-I", os.path.join(HERE, "..", "include"), "-I", BUILD]


# Device headers compiled into the run-time pass kernels (jit.cpp), embedded
# in the library as strings.
JIT_HEADERS = ["fused_abi.h", "common.cuh", "fused_ops.cuh", "jit_ops.cuh"]
JIT_INC = os.path.join(BUILD, "jit_sources.inc")


def write_jit_sources() -> None:
    parts = ["// Written by ket_b200/build.py from the headers it names: do not edit.",
             "struct JitHeader { const char* name; const char* text; };",
             "static const JitHeader kJitHeaders[] = {"]
    for h in JIT_HEADERS:
        text = open(os.path.join(CSRC, h)).read()
        if ")KETJIT\"" in text:
            raise RuntimeError(f"{h} holds the raw-string delimiter")
        parts.append(f'  {{"{h}", R"KETJIT({text})KETJIT"}},')
    parts.append("};")
    data = "\n".join(parts) + "\n"
    if not os.path.exists(JIT_INC) or open(JIT_INC).read() != data:
        with open(JIT_INC, "w") as f:
            f.write(data)


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "ket_sv.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    path = os.path.join(CSRC, src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(path), headers_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, "-c", path, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu", *ARCH, *COMMON, "-c", path, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    write_jit_sources()
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
